"""GPU parity of the nmod window product (_nmod_poly_mul_mid_mpn_ctx).

Mirrors src/fft_small/test/t-nmod_poly_mul.c: random windows, 1..64-bit
moduli, squaring, windows beyond the product length; checked against the
reference's golden fixtures, the C restatement and Python integers.
"""
import numpy as np
import pytest

import oracle as O
from tests.golden.make_golden import nmod_inputs

pytestmark = pytest.mark.gpu


def _check_record(rec, z):
    if "full" in rec:
        assert ["%016x" % int(v) for v in z] == rec["full"]
    else:
        assert len(z) == rec["len"]
        assert O.digest(z) == rec["digest"]


@pytest.mark.parametrize("name", ["nmod_small_62", "nmod_window_64bit", "nmod_tiny_mod",
                                  "nmod_square", "nmod_beyond_zn", "config3_2^20_mulmid"])
def test_golden_nmod(ctx, golden, name):
    case = next(c for c in golden["nmod"] if c["name"] == name)
    n, a, b = nmod_inputs(case)
    assert int(case["modulus"], 16) == n
    _check_record(case, ctx.nmod_poly_mul_mid(case["zl"], case["zh"], a, b, n))


@pytest.mark.parametrize("seed", range(12))
def test_random_windows_vs_restatement(ctx, seed):
    rng = np.random.default_rng(seed)
    an, bn = int(rng.integers(1, 3000)), int(rng.integers(1, 3000))
    bits = int(rng.integers(1, 65))
    n = (int(O.rand_limbs(seed + 3, 1, False)[0]) >> (64 - bits)) | (1 << (bits - 1))
    a, b = O.rand_below(seed, an, n), O.rand_below(seed + 77, bn, n)
    zl = int(rng.integers(0, an + bn))
    zh = zl + int(rng.integers(1, an + bn + 10))
    got = ctx.nmod_poly_mul_mid(zl, zh, a, b, n)
    assert (got == O.port_nmod_mul_mid(zl, zh, a, b, n)).all()


def test_small_vs_python(ctx):
    n = 1000003
    a, b = O.rand_below(1, 40, n), O.rand_below(2, 33, n)
    for zl, zh in [(0, 72), (10, 20), (70, 80), (0, 1)]:
        got = ctx.nmod_poly_mul_mid(zl, zh, a, b, n)
        top = min(zh, 72)
        want = np.zeros(zh - zl, np.uint64)
        if top > zl:
            want[:top - zl] = O.nmod_mul_mid_python(zl, top, a, b, n)
        assert (got == want).all()


def test_modulus_one_and_two(ctx):
    a = O.rand_below(5, 100, 2)
    assert (ctx.nmod_poly_mul_mid(0, 199, a, a, 1) == 0).all()
    got = ctx.nmod_poly_mul_mid(0, 199, a, a, 2)
    assert (got == O.port_nmod_mul_mid(0, 199, a, a, 2)).all()


def test_wraparound_window(ctx):
    """A middle product whose window tolerates cyclic wrap-around uses a
    shorter transform (plan.c:56-72) and stays exact."""
    n = (1 << 62) + 135
    # zn = 7999: the window [3910, 4096) fits a cyclic length of 4096
    a, b = O.rand_below(8, 4000, n), O.rand_below(9, 4000, n)
    got = ctx.nmod_poly_mul_mid(3910, 4096, a, b, n)
    assert (got == O.port_nmod_mul_mid(3910, 4096, a, b, n)).all()
    # an operand longer than the transform is folded cyclically on input
    a, b = O.rand_below(10, 6000, n), O.rand_below(11, 2000, n)
    got = ctx.nmod_poly_mul_mid(3905, 4096, a, b, n)
    assert (got == O.port_nmod_mul_mid(3905, 4096, a, b, n)).all()


def _device_mul_mid(ctx, zl, zh, a, b, n, fill=0x5A5A5A5A5A5A5A5A):
    torch = pytest.importorskip("torch")
    da = torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()
    db = da if b is a else torch.from_numpy(np.ascontiguousarray(b, np.uint64).view(np.int64)).cuda()
    dz = torch.full((max(zh - zl, 1),), fill - (1 << 64) if fill >= 1 << 63 else fill,
                    dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.nmod_poly_mul_mid_device(dz.data_ptr(), zl, zh, da.data_ptr(), len(a), db.data_ptr(), len(b), n,
                                 s.cuda_stream)
    s.synchronize()
    return dz.cpu().numpy().view(np.uint64)[:zh - zl]


@pytest.mark.parametrize("seed", range(6))
def test_device_twin_matches_host_call(ctx, seed):
    """gpu_nmod_poly_mul_mid_device gives the host call's coefficients,
    windows beyond the product zero-filled (the output starts as garbage)."""
    rng = np.random.default_rng(100 + seed)
    an, bn = int(rng.integers(1, 5000)), int(rng.integers(1, 5000))
    bits = int(rng.integers(2, 65))
    n = (int(O.rand_limbs(seed + 50, 1, False)[0]) >> (64 - bits)) | (1 << (bits - 1)) | 1
    a, b = O.rand_below(seed + 1, an, n), O.rand_below(seed + 2, bn, n)
    zl = int(rng.integers(0, an + bn))
    zh = zl + int(rng.integers(1, an + bn + 20))
    assert (_device_mul_mid(ctx, zl, zh, a, b, n) == ctx.nmod_poly_mul_mid(zl, zh, a, b, n)).all()


def test_device_twin_edges(ctx, golden):
    # the 2^20 window product of the golden fixtures, squaring, modulus 1,
    # a window entirely beyond the product, and an empty window
    case = next(c for c in golden["nmod"] if c["name"] == "config3_2^20_mulmid")
    n, a, b = nmod_inputs(case)
    _check_record(case, _device_mul_mid(ctx, case["zl"], case["zh"], a, b, n))
    a2 = O.rand_below(3, 3000, n)
    assert (_device_mul_mid(ctx, 100, 6100, a2, a2, n) == ctx.nmod_poly_mul_mid(100, 6100, a2, a2, n)).all()
    assert (_device_mul_mid(ctx, 0, 500, a2, a2, 1) == 0).all()
    assert (_device_mul_mid(ctx, 7000, 7010, a2, a2, n) == 0).all()
    assert len(_device_mul_mid(ctx, 5, 5, a2, a2, n)) == 0
