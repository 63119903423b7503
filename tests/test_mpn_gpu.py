"""GPU parity of the integer product (mpn_ctx_mpn_mul) through the C ABI.

Every output is compared limb for limb: against the golden fixtures made by
the reference itself, against GMP's mpn_mul and the C restatement of the
reference on fresh seeded inputs, and -- at the full 2^24-limb sizes --
against GMP plus residue fingerprints (a*b mod q == z mod q for independent
61-bit primes q).  Edge cases follow the reference's tests
(src/fft_small/test/t-mul.c): unbalanced operands, squaring, all-ones limbs
(longest carry chains), zero limbs, lengths around powers of two.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O
from tests.golden.make_golden import mpn_inputs

pytestmark = pytest.mark.gpu

Q61 = [2305843009213693951, 2305843009213693921, 2305843009213693907]


def _check_record(rec, z):
    if "full" in rec:
        assert ["%016x" % int(v) for v in z] == rec["full"]
    else:
        assert len(z) == rec["len"]
        assert O.digest(z) == rec["digest"]


@pytest.mark.parametrize("name", [
    "1x1", "2x1", "7x5", "32x32", "300x3", "1000x999", "ones_100x57", "ones_4096x4096",
    "square_5000", "40000x40001_np2_edge", "config1_2^16x2^16", "2^20x2^12"])
def test_golden_mpn(ctx, golden, name):
    case = next(c for c in golden["mpn"] if c["name"] == name)
    a, b = mpn_inputs(case)
    _check_record(case, ctx.mpn_mul(a, b))


@pytest.mark.parametrize("name", ["config2_2^24x2^24", "config2b_2^24x2^20"])
def test_golden_mpn_full_size(ctx, golden, name):
    case = next(c for c in golden["mpn"] if c["name"] == name)
    a, b = mpn_inputs(case)
    z = ctx.mpn_mul(a, b)
    _check_record(case, z)
    ai, bi, zi = O.to_int(a), O.to_int(b), O.to_int(z)
    for q in Q61:
        assert (ai % q) * (bi % q) % q == zi % q


def test_full_size_vs_gmp(ctx):
    a = O.rand_limbs(77, 1 << 24)
    b = O.rand_limbs(78, (1 << 24) - 12345)
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


@pytest.mark.parametrize("an,bn", [((1 << 25) - 4095, 4096), (1 << 25, 1)])
def test_longest_transform_vs_gmp(ctx, an, bn):
    """an + bn - 1 = 2^25 coefficients: the longest cyclic transform, no slack."""
    a = O.rand_limbs(an % 1000 + 3, an)
    b = O.rand_limbs(bn % 1000 + 4, bn)
    assert FB.mpn_mul_plan(an, bn)[1] == 25
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


SIZES = [(1, 1), (1, 2), (2, 2), (3, 1), (15, 17), (16, 16), (17, 16), (255, 257),
         (1000, 1), (1, 1000), (4096, 4095), (8191, 8193), (10000, 20000),
         (65536, 1), (65537, 65535), (131072, 3), (100000, 99999), (300000, 5000)]


@pytest.mark.parametrize("an,bn", SIZES)
def test_random_vs_gmp(ctx, an, bn):
    a = O.rand_limbs(an * 7 + bn, an)
    b = O.rand_limbs(bn * 11 + an, bn)
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


@pytest.mark.parametrize("an,bn", [(1, 1), (9, 4), (700, 650), (5000, 3)])
def test_random_vs_restatement(ctx, an, bn):
    a = O.rand_limbs(an + 5, an)
    b = O.rand_limbs(bn + 9, bn)
    assert (ctx.mpn_mul(a, b) == O.port_mpn_mul(a, b)).all()


@pytest.mark.parametrize("n", [1, 2, 100, 4096, 70000])
def test_all_ones_carry_chains(ctx, n):
    ones = np.full(n, (1 << 64) - 1, dtype=np.uint64)
    z = ctx.mpn_mul(ones, ones)
    assert (z == O.gmp_mpn_mul(ones, ones)).all()
    # (2^64n - 1)^2 = 2^128n - 2^(64n+1) + 1
    assert z[0] == 1 and (z[1:n] == 0).all()


def test_zeros_and_sparse(ctx):
    a = np.zeros(3000, dtype=np.uint64)
    a[-1] = 1
    b = O.rand_limbs(5, 2000)
    z = ctx.mpn_mul(a, b)
    assert (z[:2999] == 0).all() and (z[2999:2999 + 2000] == b).all()
    z = ctx.mpn_mul(np.zeros(10, np.uint64), b)
    assert (z == 0).all()


def test_squaring(ctx):
    a = O.rand_limbs(31, 50000)
    assert (ctx.mpn_mul(a, a) == O.gmp_mpn_mul(a, a)).all()


def test_repeated_calls_and_order(ctx):
    """Back-to-back calls of different sizes on one context (scratch reuse,
    look-back epochs) stay exact."""
    for k, (an, bn) in enumerate([(50000, 50000), (10, 3), (70000, 200), (50000, 50000)]):
        a, b = O.rand_limbs(900 + k, an), O.rand_limbs(950 + k, bn)
        assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


def test_range_window(ctx):
    a, b = O.rand_limbs(61, 3000), O.rand_limbs(62, 2500)
    full = O.gmp_mpn_mul(a, b)
    for lo, hi in [(0, 5500), (0, 10), (100, 4000), (5490, 5500), (5400, 6000), (6000, 6010)]:
        w = ctx.mpn_mul_range(lo, hi, a, b)
        want = np.zeros(hi - lo, dtype=np.uint64)
        top = min(hi, 5500)
        if top > lo:
            want[:top - lo] = full[lo:top]
        assert (w == want).all(), (lo, hi)


def test_default_context_entry_point():
    import ctypes
    a, b = O.rand_limbs(3, 4000), O.rand_limbs(4, 1000)
    z = np.zeros(5000, dtype=np.uint64)
    FB.lib().gpu_mpn_mul_default_mpn_ctx(z.ctypes.data, a.ctypes.data, 4000, b.ctypes.data, 1000)
    assert (z == O.gmp_mpn_mul(a, b)).all()
    assert FB.lib().gpu_get_default_mpn_ctx() is not None
    # cleanup releases the thread's context; the next call makes a new one
    FB.lib().gpu_default_mpn_ctx_cleanup()
    FB.lib().gpu_default_mpn_ctx_cleanup()
    z[:] = 0
    FB.lib().gpu_mpn_mul_default_mpn_ctx(z.ctypes.data, a.ctypes.data, 4000, b.ctypes.data, 1000)
    assert (z == O.gmp_mpn_mul(a, b)).all()
    del ctypes


def test_device_pointer_entry_point(ctx):
    torch = pytest.importorskip("torch")
    a, b = O.rand_limbs(13, 123456), O.rand_limbs(14, 65432)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.mpn_mul_device(dz.data_ptr(), da.data_ptr(), len(a), db.data_ptr(), len(b),
                       s.cuda_stream)
    s.synchronize()
    z = dz.cpu().numpy().view(np.uint64)
    assert (z == O.gmp_mpn_mul(a, b)).all()


def test_errors_are_reported(ctx):
    with pytest.raises(FB.GpuFftSmallError) as e:
        ctx.mpn_mul(np.zeros(0, np.uint64), np.ones(3, np.uint64))
    assert e.value.code == FB.EINVAL
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.mpn_mul_plan(1 << 25, (1 << 25) + 1)
    assert e.value.code == FB.ETOOBIG
    # the context stays usable after an error
    a = O.rand_limbs(1, 100)
    assert (ctx.mpn_mul(a, a) == O.gmp_mpn_mul(a, a)).all()


def test_butterfly_rate_calibration(ctx):
    """The integer-pipe calibration runs and reports a plausible rate (148 SMs
    at up to ~2 GHz, nine instructions per butterfly from registers)."""
    r = ctx.butterfly_rate()
    assert 5e11 < r < 2e13
