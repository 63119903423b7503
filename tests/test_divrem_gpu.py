"""Division with remainder of nmod polynomials (_nmod_poly_divrem_mpn_ctx).

Quotient and remainder are unique (b's leading coefficient a unit), so the
GPU result is compared with schoolbook division in Python at small sizes and,
at large sizes, with the identity a = q b + r checked through the reference's
own multiplication."""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("an,bn,n", [(2, 2, 7), (50, 20, 1000003), (300, 299, (1 << 62) + 135),
                                     (1000, 33, (1 << 63) + 29), (700, 2, 5), (4097, 2049, 2 ** 61 - 1)])
def test_divrem_vs_schoolbook(ctx, an, bn, n):
    a, b = O.rand_below(an + 1, an, n), O.rand_below(bn + 2, bn, n)
    b[-1] = max(int(b[-1]), 1)
    if n == 5 or n == 7:
        b[-1] = 1
    q, r = ctx.nmod_poly_divrem(a, b, n)
    q2, r2 = O.nmod_divrem_python(a, b, n)
    assert [int(x) for x in q] == q2
    assert [int(x) for x in r] == r2


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn", [(1 << 18, 1 << 17), (200000, 3000), (100000, 99990)])
def test_divrem_large_identity(ctx, an, bn):
    n = (1 << 62) + 135
    a, b = O.rand_below(an + 5, an, n), O.rand_below(bn + 6, bn, n)
    b[-1] = 1 + int(b[-1]) % (n - 1)
    q, r = ctx.nmod_poly_divrem(a, b, n)
    assert O.check_nmod_divrem(a, b, n, q, r)


def test_divrem_rejects_non_unit_leading_coefficient(ctx):
    a = np.arange(1, 20, dtype=np.uint64)
    b = np.array([1, 2, 6], dtype=np.uint64)          # 6 is not a unit mod 12
    with pytest.raises(FB.GpuFftSmallError) as e:
        ctx.nmod_poly_divrem(a, b, 12)
    assert e.value.code == FB.EINVAL


def _unit_leading(seed, bn, n):
    """A divisor whose leading coefficient is a unit mod n."""
    import math
    b = O.rand_below(seed, bn, n)
    k = 0
    while math.gcd(int(b[-1]), n) != 1:
        k += 1
        b[-1] = (int(b[-1]) + k) % n
    return b


# seeded draws in the shape of the reference's own test
# (src/fft_small/test/t-nmod_poly_divrem.c: bn in [2, 5002), qn in [1, 5001),
# moduli of 2 to 64 bits), plus larger quotients and divisors
REF_CASES = [(an_, bn_, bits) for (an_, bn_, bits) in [
    (2, 2, 2), (12, 11, 3), (300, 7, 17), (5000, 2, 31), (5001, 5000, 40), (9999, 5001, 62),
    (4200, 3100, 63), (7000, 123, 64), (20000, 9000, 61), (1 << 17, 1 << 15, 64)]]


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn,bits", REF_CASES)
def test_divrem_equals_reference(ctx, an, bn, bits):
    """Quotient and remainder equal the reference's own
    _nmod_poly_divrem_mpn_ctx (src/fft_small/nmod_poly_mul.c:1248-1277) on the
    same seeded inputs, coefficient for coefficient."""
    n = int(O.rand_limbs(an * 7 + bits, 1)[0]) >> (64 - bits) | (1 << (bits - 1))
    if n < 2:
        n = 3
    a = O.rand_below(an + bits, an, n)
    b = _unit_leading(bn + 3 * bits, bn, n)
    q, r = ctx.nmod_poly_divrem(a, b, n)
    qr, rr = O.ref_nmod_divrem(a, b, n)
    assert np.array_equal(np.asarray(q, dtype=np.uint64), qr)
    assert np.array_equal(np.asarray(r, dtype=np.uint64), rr)
