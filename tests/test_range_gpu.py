"""Windowed products (_mpn_ctx_mpn_mul_range / flint_mpn_mulmid_fft_small).

The reference's contract (src/fft_small/test/t-mpn_mulmid.c): limbs [lo, hi)
of a b, exact for lo = 0; for lo > 0 a lower approximation of
floor(a b / 2^(64 lo)) with deficit <= min(an, bn, lo) 2^64; a window [lo, hi)
agrees with the maximal-top window [lo, an + bn) on every limb, and is zero
past the product.  Both this implementation and the reference's own (through
the compiled reference) are checked against that contract on the same inputs;
the middle-product windows here run a shorter cyclic transform.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


def _windows(rng, zn):
    los = [0, 1, 2, 3, int(rng.integers(0, zn)), max(0, zn - 1 - int(rng.integers(0, 4))),
           int(rng.integers(0, max(1, zn // 2)))]
    return sorted(set(lo for lo in los if lo < zn))


@pytest.mark.parametrize("an,bn,seed", [(2, 1, 1), (40, 33, 2), (1000, 999, 3), (3000, 1500, 4),
                                        (20000, 10000, 5), (65536, 65536, 6), (100000, 7, 7)])
def test_contract_random(ctx, an, bn, seed):
    rng = np.random.default_rng(seed)
    a, b = O.rand_limbs(seed * 11, an), O.rand_limbs(seed * 13, bn)
    zn = an + bn
    for lo in _windows(rng, zn):
        top = ctx.mpn_mul_range(lo, zn, a, b)
        d = O.check_mul_range_contract(a, b, lo, top)
        assert d <= 2
        for hi in [lo + 1, lo + 1 + int(rng.integers(0, zn - lo)), zn + 3, zn]:
            w = ctx.mpn_mul_range(lo, hi, a, b)
            want = np.zeros(hi - lo, dtype=np.uint64)
            k = min(hi, zn) - lo
            want[:k] = top[:k]
            assert (w == want).all(), (lo, hi)


def test_middle_product_windows_and_carry_extremes(ctx):
    """Newton-style middle products (a of 2n limbs, b of n, window [n, 2n)) go
    through the shorter transform; all-ones operands make the dropped carry
    as large as it gets."""
    for n in (1000, 1 << 14, 100000):
        a, b = O.rand_limbs(n + 1, 2 * n), O.rand_limbs(n + 2, n)
        w = ctx.mpn_mul_range(n, 2 * n, a, b)
        top = ctx.mpn_mul_range(n, 3 * n, a, b)
        assert (w == top[:n]).all()
        O.check_mul_range_contract(a, b, n, top)
        ones = np.full(2 * n, (1 << 64) - 1, dtype=np.uint64)
        top1 = ctx.mpn_mul_range(n, 3 * n, ones, ones[:n])
        assert O.check_mul_range_contract(ones, ones[:n], n, top1) <= 2


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn,lo", [(3000, 1500, 1500), (5000, 4000, 7), (20000, 19999, 15000)])
def test_reference_satisfies_the_same_contract(ctx, an, bn, lo):
    a, b = O.rand_limbs(an + 5, an), O.rand_limbs(bn + 6, bn)
    zn = an + bn
    ours = ctx.mpn_mul_range(lo, zn, a, b)
    theirs = O.ref_mpn_mul_range(lo, zn, a, b)
    O.check_mul_range_contract(a, b, lo, ours)
    O.check_mul_range_contract(a, b, lo, theirs)


def test_device_window_and_mulmid_entry(ctx):
    torch = pytest.importorskip("torch")
    import ctypes
    n = 30000
    a, b = O.rand_limbs(71, 2 * n), O.rand_limbs(72, n)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty(n, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.mpn_mul_range_device(dz.data_ptr(), n, 2 * n, da.data_ptr(), 2 * n, db.data_ptr(), n,
                             s.cuda_stream)
    s.synchronize()
    want = ctx.mpn_mul_range(n, 2 * n, a, b)
    assert (dz.cpu().numpy().view(np.uint64) == want).all()
    z = np.zeros(n, dtype=np.uint64)
    FB.lib().gpu_mpn_mulmid_default_mpn_ctx(z.ctypes.data, a.ctypes.data, 2 * n, b.ctypes.data, n,
                                            n, 2 * n)
    assert (z == want).all()
