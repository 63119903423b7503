"""The rest of the plan/op API (src/fft_small.h:587-601, 636-686): signed
exports (whole and windowed), cyclic integer and nmod plans, forced prime
counts and operands in caller-provided storage.

Signed exports follow the reference's uses: the real part a c - b d of a
complex product (src/gr/transformed_mpn.c), which can be negative, and the
signed export of an unsigned product, which must agree with the unsigned one
with sign 0 (src/fft_small/test/t-op_mpn.c:216-233).  Everything is compared
with Python integers.
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


def _ops(torch, P, xs):
    out = []
    for x in xs:
        o = P.op()
        o.fft(_dev(torch, x).data_ptr(), len(x))
        out.append(o)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("an,bn,seed", [(1, 1, 0), (40, 17, 1), (3000, 3000, 2), (100000, 777, 3),
                                        (600, 600, 4)])
def test_signed_export_of_a_difference(ctx, an, bn, seed):
    torch = pytest.importorskip("torch")
    a, b = O.rand_limbs(100 + seed, an), O.rand_limbs(200 + seed, an)
    c, d = O.rand_limbs(300 + seed, bn), O.rand_limbs(400 + seed, bn)
    P = FB.FftPlan.mpn(ctx, an, bn, len_bound=2, is_signed=True)
    A, B, C, D = _ops(torch, P, [a, b, c, d])
    Z = P.op()
    P.pointwise(FB.OP_MUL, Z, A, C)
    P.pointwise(FB.OP_SUBMUL, Z, B, D)
    Z.ifft()
    nslots = an + bn - 1
    zn = an + bn + 3
    dz = torch.full((zn,), -1, dtype=torch.int64, device="cuda")
    sign = Z.export_mpn_signed(dz.data_ptr(), zn, nslots)
    v = O.to_int(a) * O.to_int(c) - O.to_int(b) * O.to_int(d)
    assert sign == (1 if v < 0 else 0)
    assert O.to_int(_host(dz)) == abs(v)
    # windows of |v|: exact limbs [lo, lo + w)
    for lo in (1, an // 2 + 1, an + bn - 2):
        w = zn - lo + 2
        dw = torch.empty(w, dtype=torch.int64, device="cuda")
        Z2 = P.op()
        P.pointwise(FB.OP_MUL, Z2, A, C)
        P.pointwise(FB.OP_SUBMUL, Z2, B, D)
        Z2.ifft()
        s2 = Z2.export_mpn_signed(dw.data_ptr(), w, nslots, lo_limbs=lo)
        want = (abs(v) >> (64 * lo)) % (1 << (64 * w))
        assert O.to_int(_host(dw)) == want, lo
        assert s2 == (1 if (v < 0 and want != 0) else 0)


def test_signed_export_zero_and_unsigned_product(ctx):
    torch = pytest.importorskip("torch")
    n = 2500
    a, b = O.rand_limbs(7, n), O.rand_limbs(8, n)
    P = FB.FftPlan.mpn(ctx, n, n, len_bound=2, is_signed=True)
    A, B = _ops(torch, P, [a, b])
    Z = P.op()
    P.pointwise(FB.OP_MUL, Z, A, B)
    P.pointwise(FB.OP_SUBMUL, Z, A, B)        # exactly zero
    Z.ifft()
    dz = torch.full((2 * n + 3,), -1, dtype=torch.int64, device="cuda")
    assert Z.export_mpn_signed(dz.data_ptr(), 2 * n + 3, 2 * n - 1) == 0
    assert (_host(dz) == 0).all()
    Z2 = P.op()
    P.pointwise(FB.OP_MUL, Z2, A, B)
    Z2.ifft()
    assert Z2.export_mpn_signed(dz.data_ptr(), 2 * n + 3, 2 * n - 1) == 0
    z = _host(dz)
    assert (z[:2 * n] == O.gmp_mpn_mul(a, b)).all() and (z[2 * n:] == 0).all()
    with pytest.raises(FB.GpuFftSmallError):      # window too short for the sign
        Z2.export_mpn_signed(dz.data_ptr(), 2 * n, 2 * n - 1)


def test_mpn_cyclic_plan(ctx):
    torch = pytest.importorskip("torch")
    P, nn = FB.FftPlan.mpn_cyclic(ctx, 1000)
    assert nn == 1024
    a, b = O.rand_limbs(11, nn), O.rand_limbs(12, 700)
    A, B = _ops(torch, P, [a, b])
    Z = P.op()
    P.pointwise(FB.OP_MUL, Z, A, B)
    Z.ifft()
    dz = torch.empty(nn + 3, dtype=torch.int64, device="cuda")
    Z.export_mpn(dz.data_ptr(), nn + 3)
    P.check()
    z = O.to_int(_host(dz))
    mod = (1 << (64 * nn)) - 1
    assert z % mod == (O.to_int(a) * O.to_int(b)) % mod
    assert z < 2 ** (64 * nn + 128 + 10)


def test_nmod_cyclic_plan_folds_long_operands(ctx):
    torch = pytest.importorskip("torch")
    n = (1 << 61) - 1
    depth, N = 10, 1 << 10
    a, b = O.rand_below(21, 2500, n), O.rand_below(22, 700, n)
    P = FB.FftPlan.nmod_cyclic(ctx, depth, N, n)
    A, B = P.op(), P.op()
    A.fft(_dev(torch, a).data_ptr(), len(a))
    B.fft(_dev(torch, b).data_ptr(), len(b))
    Z = P.op()
    P.pointwise(FB.OP_MUL, Z, A, B)
    Z.ifft()
    dz = torch.empty(N, dtype=torch.int64, device="cuda")
    Z.export_nmod(dz.data_ptr(), 0, N)
    P.check()
    want = [0] * N
    for i, x in enumerate(int(v) for v in a):
        if x:
            for j, y in enumerate(int(v) for v in b):
                want[(i + j) % N] = (want[(i + j) % N] + x * y) % n
    assert [int(v) for v in _host(dz)] == want


def test_forced_prime_count_and_borrowed_storage(ctx):
    torch = pytest.importorskip("torch")
    n = 4000
    a, b = O.rand_limbs(31, n), O.rand_limbs(32, n)
    P6 = FB.FftPlan.mpn_np(ctx, n, n, 1, False, 6)
    assert P6.np == 6
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.FftPlan.mpn_np(ctx, n, n, 1, False, 4)
    assert e.value.code == FB.ENOPRIMES
    words = P6.sizeof_data() // 4
    assert words >= P6.np << P6.logM
    store = torch.zeros(2 * words, dtype=torch.int32, device="cuda")
    A = P6.op(store.data_ptr())
    B = P6.op(store.data_ptr() + 4 * words)
    A.fft(_dev(torch, a).data_ptr(), n)
    B.fft(_dev(torch, b).data_ptr(), n)
    P6.pointwise(FB.OP_MUL, A, A, B)
    A.ifft()
    dz = torch.empty(2 * n, dtype=torch.int64, device="cuda")
    A.export_mpn(dz.data_ptr(), 2 * n)
    P6.check()
    assert (_host(dz) == O.gmp_mpn_mul(a, b)).all()
    A.close()
    B.close()
    assert int(store.abs().sum().item()) != 0       # caller storage survives the operands
