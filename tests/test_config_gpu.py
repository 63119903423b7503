"""Every schedule gives the same exact product.

All candidate configurations the autotuner considers (prime count, transform
length, four-step row length, basecase route) are run on the device and
compared limb for limb with GMP (mpn) or with the default schedule and the
Python restatement (integer polynomials).
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O
from flint_b200 import tuner

pytestmark = pytest.mark.gpu

MPN = [(1, 1), (2, 1), (31, 30), (64, 64), (1000, 3), (1024, 1024), (3000, 1024), (100000, 7),
       (5000, 4999), (70000, 65537), (1 << 20, 1 << 14), (1 << 21, 300)]


@pytest.mark.parametrize("an,bn", MPN)
def test_mpn_every_candidate_exact(ctx, an, bn):
    torch = pytest.importorskip("torch")
    a = O.rand_limbs(an + 7, an)
    b = O.rand_limbs(bn + 9, bn)
    want = O.gmp_mpn_mul(a, b)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty(an + bn, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    for c in tuner.candidates((0, an, bn)):
        dz.fill_(-1)
        ctx.mpn_mul_device_config(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, c,
                                  s.cuda_stream)
        s.synchronize()
        assert (dz.cpu().numpy().view(np.uint64) == want).all(), c


def _valid_logC(logM):
    """Row lengths the validator accepts for a transform of 2^logM points."""
    lo = max(5, logM - 11)
    if logM < 14:
        lo = max(lo, logM - 4)
    return list(range(lo, min(logM, 14) + 1))


@pytest.mark.parametrize("logM", list(range(5, 18)) + [20, 22])
def test_mpn_every_row_length_exact(ctx, logM):
    """Every (transform length, row length, row-pass width) a caller may
    configure -- not only the tuner's candidates -- gives the exact product;
    row lengths just outside the rule are rejected."""
    torch = pytest.importorskip("torch")
    an = (1 << (logM - 1)) - 3 if logM > 5 else 9
    bn = max(1, (1 << (logM - 1)) - an + 7) if logM > 5 else 7
    assert FB.mpn_mul_plan(an, bn)[1] <= logM
    a = O.rand_limbs(an + logM, an)
    b = O.rand_limbs(bn + 3 * logM, bn)
    want = O.gmp_mpn_mul(a, b)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty(an + bn, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    for logC in _valid_logC(logM):
        # the row pass's width by the launch rule, and forced to 16 and 32
        # points per thread
        for fl in (0, FB.FLAG_ROWS16, FB.FLAG_ROWS32) if logC >= 9 else (0, FB.FLAG_ROWS32):
            c = FB.resolve_config(0, an, bn, FB.MulConfig(FB.ROUTE_NTT, 0, logM, logC, fl))
            dz.fill_(-1)
            ctx.mpn_mul_device_config(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, c,
                                      s.cuda_stream)
            s.synchronize()
            assert (dz.cpu().numpy().view(np.uint64) == want).all(), c
    lo = _valid_logC(logM)[0]
    if lo > 5:
        with pytest.raises(FB.GpuFftSmallError):
            FB.resolve_config(0, an, bn, FB.MulConfig(FB.ROUTE_NTT, 0, logM, lo - 1))


def test_basecase_all_ones_and_operand_order(ctx):
    torch = pytest.importorskip("torch")
    s = torch.cuda.current_stream()
    bc = FB.MulConfig(FB.ROUTE_BASECASE, 0, 0, 0)
    for an, bn in [(1024, 1024), (7, 5000), (1, 1), (50000, 1024), (4096, 4096), (3000, 2000),
                   (300000, 4000), (1, 4096)]:
        a = np.full(an, (1 << 64) - 1, dtype=np.uint64)
        b = np.full(bn, (1 << 64) - 1, dtype=np.uint64)
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = torch.from_numpy(b.view(np.int64)).cuda()
        dz = torch.empty(an + bn, dtype=torch.int64, device="cuda")
        ctx.mpn_mul_device_config(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, bc,
                                  s.cuda_stream)
        s.synchronize()
        assert (dz.cpu().numpy().view(np.uint64) == O.gmp_mpn_mul(a, b)).all()


@pytest.mark.parametrize("an,bn", [(129, 257), (128, 256), (4095, 4096), (4096, 2049), (10 ** 6, 4096),
                                   (255, 3), (5000, 4096)])
def test_basecase_split_blocks_exact(ctx, an, bn):
    """The single-product basecase (column sums split over positions and
    short-operand chunks, added atomically) at block-boundary shapes, random
    limbs, against GMP."""
    torch = pytest.importorskip("torch")
    a = O.rand_limbs(an + 5, an)
    b = O.rand_limbs(bn + 11, bn)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.mpn_mul_device_config(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn,
                              FB.MulConfig(FB.ROUTE_BASECASE, 0, 0, 0), s.cuda_stream)
    s.synchronize()
    assert (dz.cpu().numpy().view(np.uint64) == O.gmp_mpn_mul(a, b)).all()


@pytest.mark.parametrize("r", [(1, 300, 200, 2, 2), (1, 4000, 3000, 3, 1), (1, 256, 256, 65, 65)])
def test_fmpz_every_candidate_exact(ctx, r):
    torch = pytest.importorskip("torch")
    _, an, bn, aw, bw = r
    a = O.rand_fmpz_raw(an, an, 64 * aw - 1)
    b = O.rand_fmpz_raw(bn, bn, 64 * bw - 1)
    zw = aw + bw + 1
    zn = an + bn - 1
    want = ctx.fmpz_poly_mul_mid(0, zn, a, b, zw)
    if an * bn <= 300 * 200:
        assert O.raw_to_ints(want) == O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty((zn, zw), dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    for c in tuner.candidates(r):
        dz.fill_(-1)
        ctx.fmpz_poly_mul_device_config(dz.data_ptr(), zw, 0, zn, da.data_ptr(), aw, an,
                                        db.data_ptr(), bw, bn, c, s.cuda_stream)
        s.synchronize()
        assert (dz.cpu().numpy().view(np.uint64) == want).all(), c


def test_time_config_reports_positive_times(ctx):
    for r in [(0, 100, 100), (0, 1 << 16, 1 << 16), (1, 500, 500, 3, 3)]:
        kind, an, bn = r[:3]
        aw, bw = (r[3], r[4]) if kind else (1, 1)
        for c in tuner.candidates(r)[:3]:
            ms = ctx.time_config(kind, an, bn, c, aw, bw, reps=2)
            assert 0.0 < ms < 1000.0
