"""GPU parity of the precomputed-transform products and division
(_mul_precomp_init / _nmod_poly_mul_mid_precomp / _nmod_poly_divrem_precomp_*)
through the C ABI.

As the reference's test (src/fft_small/test/t-nmod_poly_divrem.c:27-90):
moduli of 2..64 bits, bn in [2, 5000], qn in [1, 5000], precision qn plus up
to 200; quotient and remainder compared with the library's own division
(which the divrem tests pin to schoolbook division and to the reference's
multiplication) and, for small sizes, with schoolbook division in Python.
Window products are compared with the plain window product; one precomp is
reused across several operands, as its users do.
"""
import math

import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


def _modulus(rng, bits):
    return int(rng.integers(1 << (bits - 1), (1 << bits) - 1, dtype=np.uint64, endpoint=True)) \
        if bits < 64 else int(rng.integers(1 << 62, 1 << 63)) * 2 + 1


def _poly(seed, n, mod):
    return O.rand_below(seed, n, mod)


def _unit_lead(b, n, seed):
    k = 0
    while math.gcd(int(b[-1]), n) != 1:
        b[-1] = O.rand_below(seed + 7919 * (k + 1), 1, n)[0]
        k += 1
    return b


@pytest.mark.parametrize("seed", range(8))
def test_divrem_precomp_matches_division(ctx, seed):
    rng = np.random.default_rng(100 + seed)
    bits = int(rng.integers(2, 65))
    n = _modulus(rng, bits)
    if n < 2:
        n = 3
    bn = int(rng.integers(2, 5001))
    qn = int(rng.integers(1, 5001))
    prec = qn + int(rng.integers(0, 200))
    b = _unit_lead(_poly(10 * seed + 1, bn, n), n, seed)
    with FB.DivremPrecomp(ctx, b, prec, n) as D:
        for k, q_len in enumerate((qn, max(1, qn // 3), prec)):
            a = _poly(10 * seed + 2 + k, bn + q_len - 1, n)
            q, r = D.divrem(a)
            q2, r2 = ctx.nmod_poly_divrem(a, b, n)
            assert (q == q2).all() and (r == r2).all(), (bits, bn, q_len)
            if (bn + q_len) * min(bn, q_len) < 2e6:
                qs, rs = O.nmod_divrem_python(a, b, n)
                assert [int(v) for v in q] == qs and [int(v) for v in r] == rs


def test_divrem_precomp_small_cases(ctx):
    for n in (2, 3, 5, 1 << 32, (1 << 64) - 59):
        for bn, qn in ((2, 1), (2, 7), (3, 1), (17, 17), (300, 1), (257, 300)):
            b = _unit_lead(_poly(bn * 31 + qn, bn, n), n, bn)
            a = _poly(bn * 37 + qn, bn + qn - 1, n)
            with FB.DivremPrecomp(ctx, b, qn, n) as D:
                q, r = D.divrem(a)
            qs, rs = O.nmod_divrem_python(a, b, n)
            assert [int(v) for v in q] == qs and [int(v) for v in r] == rs, (n, bn, qn)


def test_divrem_precomp_quotient_beyond_precision(ctx):
    n = 1000003
    b = _unit_lead(_poly(5, 100, n), n, 5)
    with FB.DivremPrecomp(ctx, b, 50, n) as D:
        assert D.divrem(_poly(6, 100 + 50 - 1, n)) is not None
        assert D.divrem(_poly(6, 100 + 51 - 1, n)) is None


def test_divrem_precomp_large_device(ctx):
    torch = pytest.importorskip("torch")
    n = (1 << 62) + 135
    bn, qn = 1 << 16, 1 << 18
    b = _unit_lead(_poly(41, bn, n), n, 41)
    a = _poly(42, bn + qn - 1, n)
    with FB.DivremPrecomp(ctx, b, qn, n) as D:
        da = torch.from_numpy(a.view(np.int64)).cuda()
        dq = torch.empty(qn, dtype=torch.int64, device="cuda")
        dr = torch.empty(bn - 1, dtype=torch.int64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        for _ in range(2):                       # reuse
            D.divrem_device(dq.data_ptr(), dr.data_ptr(), da.data_ptr(), len(a), st)
        q = dq.cpu().numpy().view(np.uint64)
        r = dr.cpu().numpy().view(np.uint64)
    q2, r2 = ctx.nmod_poly_divrem(a, b, n)
    assert (q == q2).all() and (r == r2).all()


@pytest.mark.parametrize("bits,bn,depth", [(62, 1000, 12), (64, 4096, 13), (3, 777, 11), (40, 1, 5),
                                           (50, 30000, 16)])
def test_mul_mid_precomp_windows(ctx, bits, bn, depth):
    rng = np.random.default_rng(bits * bn)
    n = _modulus(rng, bits)
    b = _poly(bn + 1, bn, n)
    M = 1 << max(depth, 5)
    with FB.MulPrecomp(ctx, b, depth, n) as P:
        assert P.depth == max(depth, 5)
        for k in range(6):
            an = int(rng.integers(1, 2 * M))
            a = _poly(1000 * k + bn, an, n)
            zn = an + bn - 1
            lo = max(0, zn - M)
            zl = int(rng.integers(lo, max(lo + 1, min(zn, M))))
            zh = zl + 1 + int(rng.integers(0, max(1, min(M, zn + 3) - zl + 1)))
            z = P.mul_mid(zl, zh, a)
            fits = min(zh, zn) <= M and zn - zl <= M
            if not fits:
                assert z is None
                continue
            want = ctx.nmod_poly_mul_mid(zl, zh, a, b, n)
            assert z is not None and (z == want).all(), (an, zl, zh)


def test_mul_mid_precomp_refuses_wrapping_window(ctx):
    n = 101
    with FB.MulPrecomp(ctx, _poly(1, 40, n), 6, n) as P:     # 64-point transform
        a = _poly(2, 40, n)                                    # product of 79 coefficients
        assert P.mul_mid(0, 79, a) is None
        assert P.mul_mid(15, 64, a) is not None
        assert (P.mul_mid(15, 64, a) == ctx.nmod_poly_mul_mid(15, 64, a, _poly(1, 40, n), n)).all()
        a20 = _poly(3, 20, n)                                  # product of 59 coefficients
        z = P.mul_mid(50, 70, a20)                             # beyond the product: zero-filled
        assert z is not None and (z[9:] == 0).all()
        assert (z == ctx.nmod_poly_mul_mid(50, 70, a20, _poly(1, 40, n), n)).all()
