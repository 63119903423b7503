"""Products on transforms of 3 2^k points (the truncated lengths).

A whole product whose length L = an + bn - 1 lies in (2^(m-1), 3 2^(m-2)]
runs a 3 2^(m-2)-point transform (a radix-3 column stage) instead of a
2^m-point one -- the counterpart of the reference's truncated transforms
(src/fft_small/sd_fft.c:1230-1274, sd_ifft.c:1503-1533).  Every column
length the kernels instantiate (3 2^5 .. 3 2^10 points, transforms of
3 2^18 .. 3 2^23 points) is checked limb for limb against GMP, squarings
included, and the two sizes just above 2^24 coefficients also against the
reference's own product (the compiled fft_small).
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu

# (an, bn, expected transform points)
CASES = [
    ((1 << 18) + 100, (1 << 18) + 7, 3 << 18),       # columns of 3 2^5
    (700000, 600000, 3 << 19),                        # 3 2^6
    (1600000, 1400000, 3 << 20),                      # 3 2^7
    (3500000, 2500000, 3 << 21),                      # 3 2^8
    (6000000, 5500000, 3 << 22),                      # 3 2^9
    ((1 << 23) + (1 << 20), (1 << 23) + (1 << 20), 3 << 23),   # 3 2^10
    (3 << 22, 3 << 22, 3 << 23),                      # L = 3 2^23 - 1, the longest
]


def _device_product(torch, ctx, a, b, square=False):
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = da if square else torch.from_numpy(b.view(np.int64)).cuda()
    n = len(a) + len(b)
    dz = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.mpn_mul_device(dz.data_ptr(), da.data_ptr(), len(a), db.data_ptr(), len(b), s.cuda_stream)
    s.synchronize()
    return dz.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("an,bn,points", CASES)
def test_three_length_products_exact(ctx, an, bn, points):
    torch = pytest.importorskip("torch")
    assert FB.mpn_mul_transform_points(an, bn) == points
    a = O.rand_limbs(an + 11, an)
    b = O.rand_limbs(bn + 13, bn)
    z = _device_product(torch, ctx, a, b)
    assert (z == O.gmp_mpn_mul(a, b)).all()
    if an >= (1 << 23) and O.have_ref():
        assert (z == O.ref_mpn_mul(a, b)).all()


@pytest.mark.parametrize("n", [700001, 3000000, (1 << 23) + 12345])
def test_three_length_squaring_exact(ctx, n):
    torch = pytest.importorskip("torch")
    assert FB.mpn_mul_transform_points(n, n, square=True) % 3 == 0
    a = O.rand_limbs(n + 5, n)
    z = _device_product(torch, ctx, a, a, square=True)
    assert (z == O.gmp_mpn_mul(a, a)).all()


def test_three_length_host_pointer_and_boundaries(ctx):
    """The host-pointer entry point takes the same route; lengths just above
    3 2^(m-2) go back to the power of two, and both sides of the boundary are
    exact."""
    k = 19
    for L, pts in [(3 << k, 3 << k), ((3 << k) + 1, 1 << (k + 2))]:
        an = L // 2 + 1
        bn = L + 1 - an
        assert FB.mpn_mul_transform_points(an, bn) == pts
        a = O.rand_limbs(L + 1, an)
        b = O.rand_limbs(L + 2, bn)
        assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()
