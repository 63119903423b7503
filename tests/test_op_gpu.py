"""Plans and transformed operands (the reference's op API, src/fft_small/op.c).

Forward transforms kept on the device combine pointwise and come back
exactly: a single product against GMP, a dot product sum a_k b_k and
differences against Python integers, squaring, negation, nmod windows
against the Python restatement and the compiled reference, and one
transformed operand reused against many others.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("an,bn", [(1, 1), (100, 37), (5000, 5000), (70000, 3000)])
def test_mul_matches_gmp(ctx, an, bn):
    torch = pytest.importorskip("torch")
    a, b = O.rand_limbs(an + 1, an), O.rand_limbs(bn + 2, bn)
    P = FB.FftPlan.mpn(ctx, an, bn)
    A, B, Z = P.op(), P.op(), P.op()
    da, db = _dev(torch, a), _dev(torch, b)
    dz = torch.empty(an + bn, dtype=torch.int64, device="cuda")
    A.fft(da.data_ptr(), an)
    B.fft(db.data_ptr(), bn)
    P.pointwise(FB.OP_MUL, Z, A, B)
    Z.ifft()
    Z.export_mpn(dz.data_ptr(), an + bn)
    P.check()
    assert (_host(dz) == O.gmp_mpn_mul(a, b)).all()


def test_dot_product_difference_square_negation(ctx):
    torch = pytest.importorskip("torch")
    n = 3000
    xs = [O.rand_limbs(10 + k, n) for k in range(6)]
    P = FB.FftPlan.mpn(ctx, n, n, len_bound=4 * n)
    ops = []
    for x in xs:
        o = P.op()
        o.fft(_dev(torch, x).data_ptr(), n)
        ops.append(o)
    torch.cuda.synchronize()
    Z = P.op()
    P.pointwise(FB.OP_MUL, Z, ops[0], ops[1])
    P.pointwise(FB.OP_ADDMUL, Z, ops[2], ops[3])
    P.pointwise(FB.OP_ADDMUL, Z, ops[4], ops[5])
    Z.ifft()
    dz = torch.empty(2 * n + 1, dtype=torch.int64, device="cuda")
    Z.export_mpn(dz.data_ptr(), 2 * n + 1)
    P.check()
    v = [O.to_int(x) for x in xs]
    assert O.to_int(_host(dz)) == v[0] * v[1] + v[2] * v[3] + v[4] * v[5]
    # the unsigned export needs nonnegative coefficients (as the reference's
    # fft_small_export_mpn does): (x0 + x1)^2 through ADD and SQR
    D, S = P.op(), P.op()
    P.pointwise(FB.OP_ADD, D, ops[0], ops[1])
    P.pointwise(FB.OP_SQR, S, D)
    S.ifft()
    dz2 = torch.empty(2 * n + 1, dtype=torch.int64, device="cuda")
    S.export_mpn(dz2.data_ptr(), 2 * n + 1)
    P.check()
    assert O.to_int(_host(dz2)) == (v[0] + v[1]) ** 2
    # SUBMUL undoes ADDMUL, SUB undoes ADD, NEG twice is the identity
    W, E = P.op(), P.op()
    P.pointwise(FB.OP_MUL, W, ops[0], ops[1])
    P.pointwise(FB.OP_ADDMUL, W, ops[2], ops[3])
    P.pointwise(FB.OP_SUBMUL, W, ops[2], ops[3])
    P.pointwise(FB.OP_NEG, W, W)
    P.pointwise(FB.OP_NEG, W, W)
    P.pointwise(FB.OP_ADD, E, ops[4], ops[5])
    P.pointwise(FB.OP_SUB, E, E, ops[5])
    P.pointwise(FB.OP_ADDMUL, W, E, ops[3])
    W.ifft()
    dz3 = torch.empty(2 * n + 1, dtype=torch.int64, device="cuda")
    W.export_mpn(dz3.data_ptr(), 2 * n + 1)
    P.check()
    assert O.to_int(_host(dz3)) == v[0] * v[1] + v[4] * v[3]


def test_one_transformed_operand_against_many(ctx):
    torch = pytest.importorskip("torch")
    n, m = 40000, 20000
    b = O.rand_limbs(99, m)
    P = FB.FftPlan.mpn(ctx, n, m)
    B = P.op()
    B.fft(_dev(torch, b).data_ptr(), m)
    A, Z = P.op(), P.op()
    for k in range(4):
        a = O.rand_limbs(200 + k, n - 7 * k)
        A.fft(_dev(torch, a).data_ptr(), len(a))
        P.pointwise(FB.OP_MUL, Z, A, B)
        Z.ifft()
        dz = torch.empty(len(a) + m, dtype=torch.int64, device="cuda")
        Z.export_mpn(dz.data_ptr(), len(a) + m)
        P.check()
        assert (_host(dz) == O.gmp_mpn_mul(a, b)).all()


@pytest.mark.parametrize("an,bn,zl,zh,bits", [(200, 150, 100, 300, 62), (1000, 1000, 0, 1999, 3),
                                              (1 << 16, 1 << 16, 1 << 15, 3 << 15, 62)])
def test_nmod_window(ctx, an, bn, zl, zh, bits):
    torch = pytest.importorskip("torch")
    from tests.golden.make_golden import nmod_modulus
    n = nmod_modulus(an + bits, bits)
    a, b = O.rand_below(an + 3, an, n), O.rand_below(bn + 4, bn, n)
    zn = an + bn - 1
    P = FB.FftPlan.nmod(ctx, zl, zh, zn, n, len_bound=min(an, bn))
    A, B, Z = P.op(), P.op(), P.op()
    A.fft(_dev(torch, a).data_ptr(), an)
    B.fft(_dev(torch, b).data_ptr(), bn)
    P.pointwise(FB.OP_MUL, Z, A, B)
    Z.ifft()
    dz = torch.empty(zh - zl, dtype=torch.int64, device="cuda")
    Z.export_nmod(dz.data_ptr(), zl, zh)
    P.check()
    if an * bn <= 10 ** 6:
        want = O.nmod_mul_mid_python(zl, zh, a, b, n)
    else:
        want = O.port_nmod_mul_mid(zl, zh, a, b, n)
    assert (_host(dz) == np.array(want, dtype=np.uint64)).all()


def test_domain_and_plan_checks(ctx):
    torch = pytest.importorskip("torch")
    P = FB.FftPlan.mpn(ctx, 100, 100)
    Q = FB.FftPlan.mpn(ctx, 5000, 5000)
    A, B, Z = P.op(), P.op(), P.op()
    x = _dev(torch, O.rand_limbs(5, 100))
    A.fft(x.data_ptr(), 100)
    B.fft(x.data_ptr(), 100)
    P.pointwise(FB.OP_MUL, Z, A, B)
    with pytest.raises(FB.GpuFftSmallError):
        P.pointwise(FB.OP_MUL, Z, Z, A)          # product of a product
    with pytest.raises(FB.GpuFftSmallError):
        P.pointwise(FB.OP_ADD, Z, A, Z)          # mixed domains
    with pytest.raises(FB.GpuFftSmallError):
        P.pointwise(FB.OP_ADDMUL, A, A, B)       # accumulate into a forward transform
    with pytest.raises(FB.GpuFftSmallError):
        Q.pointwise(FB.OP_MUL, Z, A, B)          # operands of another plan
