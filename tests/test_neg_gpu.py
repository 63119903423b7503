"""GPU parity of products modulo 2^N + 1 (sd_fft_mpn_mulmod_2expp1, the
pointwise stage of Schoenhage-Strassen) through the C ABI.

Outputs are compared limb for limb with the golden fixtures made by the
reference's own engine, and on fresh seeded inputs with the Python product
folded mod 2^N + 1 (the check of src/fft_small/test/
t-sd_fft_mpn_mulmod_2expp1.c:21-48).  Operand shapes follow that test:
random, 2^N, unreduced top limb, sparse, all-ones, squaring; plus batches,
strides, the staged (cached transform) form and batches longer than one
chunk of the residue buffer.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O
from tests.golden.make_golden import NEG_CASES, neg_inputs

pytestmark = pytest.mark.gpu

KINDS = ["rand", "two_n", "unreduced", "sparse", "ones", "zero"]


def _check_record(rec, z):
    if "full" in rec:
        assert ["%016x" % int(v) for v in z] == rec["full"]
    else:
        assert len(z) == rec["len"]
        assert O.digest(z) == rec["digest"]


@pytest.mark.parametrize("name", [c["name"] for c in NEG_CASES])
def test_golden_negacyclic(ctx, golden, name):
    case = next(c for c in golden["neg"] if c["name"] == name)
    N, x, y = neg_inputs(case)
    with FB.Mulmod2expp1(ctx, N, case["m"]) as C:
        _check_record(case, C.mul(x, x if case["ky"] == "square" else y))


def test_context_choices_and_errors(ctx):
    with FB.Mulmod2expp1(ctx, 16 * 64, 16) as C:       # 16 digits run as 32 of 32 bits
        assert (C.m, C.b) == (32, 32)
    with FB.Mulmod2expp1(ctx, 128 * 88, 128) as C:     # 88-bit digits need 7 primes: split finer
        assert C.m * C.b == 128 * 88 and C.b < 88 and C.np <= 6
    with FB.Mulmod2expp1(ctx, 47104, 0) as C:
        assert C.N == 47104 and C.m * C.b == 47104
    for N, m, code in ((1000, 0, FB.EINVAL), (64 * 48, 24, FB.EINVAL), (64 * 48, 7, FB.EINVAL),
                       (2752512, 0, FB.ENOPRIMES)):
        with pytest.raises(FB.GpuFftSmallError) as e:
            FB.Mulmod2expp1(ctx, N, m)
        assert e.value.code == code
    assert FB.mulmod_2expp1_choose_np(64, 10) == 5
    assert FB.mulmod_2expp1_choose_np(20, 5) == 2
    assert FB.mulmod_2expp1_choose_np(100, 14) == -1


@pytest.mark.parametrize("N,m", [(2048, 32), (47104, 1024), (12288, 256), (65536, 0),
                                 (1 << 20, 1 << 14), (64 * 3 * 1024, 0)])
def test_single_products_vs_python(ctx, N, m):
    n = N // 64
    with FB.Mulmod2expp1(ctx, N, m) as C:
        for s, (kx, ky) in enumerate([("rand", "rand"), ("two_n", "rand"), ("unreduced", "unreduced"),
                                      ("sparse", "ones"), ("ones", "ones"), ("two_n", "two_n"),
                                      ("zero", "rand")]):
            x = O.neg_operand(900 + s, n, kx)
            y = O.neg_operand(950 + s, n, ky)
            assert (C.mul(x, y) == O.negmul_python(x, y, N)).all(), (kx, ky)
        x = O.neg_operand(999, n, "rand")
        assert (C.mul(x, x) == O.negmul_python(x, x, N)).all()   # squaring


def _batch(n, count, seed, stride):
    X = np.zeros((count, stride), dtype=np.uint64)
    for i in range(count):
        X[i, :n + 1] = O.neg_operand(seed + i, n, KINDS[i % len(KINDS)] if i % 3 == 0 else "rand")
    return X


@pytest.mark.parametrize("N,m,count,pad", [(2048, 32, 37, 0), (47104, 1024, 9, 3),
                                           (12288, 256, 64, 1), (1 << 18, 0, 5, 0)])
def test_batch_device(ctx, N, m, count, pad):
    torch = pytest.importorskip("torch")
    n = N // 64
    stride = n + 1 + pad
    X = _batch(n, count, 5000, stride)
    Y = _batch(n, count, 7000, stride)
    dx, dy = torch.from_numpy(X.view(np.int64)).cuda(), torch.from_numpy(Y.view(np.int64)).cuda()
    dz = torch.full((count, stride), -1, dtype=torch.int64, device="cuda")
    with FB.Mulmod2expp1(ctx, N, m) as C:
        st = torch.cuda.current_stream().cuda_stream
        C.batch_device(dz.data_ptr(), dx.data_ptr(), dy.data_ptr(), count, stride, st)
        Z = dz.cpu().numpy().view(np.uint64)
        for i in range(count):
            assert (Z[i, :n + 1] == O.negmul_python(X[i, :n + 1], Y[i, :n + 1], N)).all(), i
            assert (Z[i, n + 1:] == np.uint64((1 << 64) - 1)).all()      # padding untouched
        # squaring: x == y
        C.batch_device(dz.data_ptr(), dx.data_ptr(), dx.data_ptr(), count, stride, st)
        Z = dz.cpu().numpy().view(np.uint64)
        for i in range(0, count, max(1, count // 5)):
            assert (Z[i, :n + 1] == O.negmul_python(X[i, :n + 1], X[i, :n + 1], N)).all(), i


def test_staged_matches_one_shot(ctx):
    torch = pytest.importorskip("torch")
    N, m, count = 47104, 1024, 11
    n = N // 64
    X, Y = _batch(n, count, 100, n + 1), _batch(n, count, 200, n + 1)
    dx, dy = torch.from_numpy(X.view(np.int64)).cuda(), torch.from_numpy(Y.view(np.int64)).cuda()
    with FB.Mulmod2expp1(ctx, N, m) as C:
        st = torch.cuda.current_stream().cuda_stream
        F = torch.empty(C.transformed_size(count), dtype=torch.int32, device="cuda")
        C.transform_device(F.data_ptr(), dy.data_ptr(), count, None, st)
        z1 = torch.empty_like(dx)
        z2 = torch.empty_like(dx)
        C.mul_cached_device(z1.data_ptr(), dx.data_ptr(), F.data_ptr(), count, None, st)
        C.batch_device(z2.data_ptr(), dx.data_ptr(), dy.data_ptr(), count, None, st)
        assert torch.equal(z1, z2)
        Z = z1.cpu().numpy().view(np.uint64)
        for i in range(count):
            assert (Z[i] == O.negmul_python(X[i], Y[i], N)).all(), i
        # one-operand host forms
        F1 = torch.empty(C.transformed_size(1), dtype=torch.int32, device="cuda")
        L = FB.lib()
        FB._check(L.gpu_mulmod_2expp1_transform(C.ptr, F1.data_ptr(), Y[3].ctypes.data))
        z = np.zeros(n + 1, dtype=np.uint64)
        FB._check(L.gpu_mulmod_2expp1_mul_cached(C.ptr, z.ctypes.data, X[3].ctypes.data, F1.data_ptr()))
        assert (z == Z[3]).all()


def test_batch_longer_than_one_chunk(ctx):
    """2^14 digits of 80 bits (six primes): the residue buffer holds 512
    products, so 513 run as two chunks; every 16th product and those on either
    side of the chunk boundary are compared with Python."""
    torch = pytest.importorskip("torch")
    N, m, count = 80 << 14, 1 << 14, 513
    n = N // 64
    rng = np.random.default_rng(3)
    X = rng.integers(0, 1 << 63, size=(count, n + 1), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(count, n + 1), dtype=np.uint64)
    Y = rng.integers(0, 1 << 63, size=(count, n + 1), dtype=np.uint64) * np.uint64(2)
    X[:, n] = 0
    Y[:, n] = 0
    X[7, n] = 1
    dx, dy = torch.from_numpy(X.view(np.int64)).cuda(), torch.from_numpy(Y.view(np.int64)).cuda()
    dz = torch.empty_like(dx)
    with FB.Mulmod2expp1(ctx, N, m) as C:
        assert C.np == 6
        C.batch_device(dz.data_ptr(), dx.data_ptr(), dy.data_ptr(), count, None,
                       torch.cuda.current_stream().cuda_stream)
        Z = dz.cpu().numpy().view(np.uint64)
    for i in sorted(set(range(0, count, 16)) | {7, 511, 512}):
        assert (Z[i] == O.negmul_python(X[i], Y[i], N)).all(), i


@pytest.mark.parametrize("seed", range(10))
def test_random_rings_and_batches(ctx, seed):
    """Random ring sizes N (multiples of 64), requested digit counts (0, 16 ..
    2^16) and batch counts; splits the primes cannot hold must be refused with
    ENOPRIMES, every other product exact against Python."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4000 + seed)
    n = int(rng.integers(1, 6000))
    N = 64 * n
    m = int(rng.choice([0, 16, 32, 64, 256, 1024, 1 << 14, 1 << 16]))
    if m and N % m:
        m = 0
    try:
        C = FB.Mulmod2expp1(ctx, N, m)
    except FB.GpuFftSmallError as e:
        assert e.code in (FB.ENOPRIMES, FB.EINVAL)
        return
    with C:
        assert C.m * C.b == N and 32 <= C.m <= (1 << 14) and C.np <= 6
        count = int(rng.integers(1, 40))
        X = _batch(n, count, 9000 + seed, n + 1)
        Y = _batch(n, count, 9500 + seed, n + 1)
        dx, dy = torch.from_numpy(X.view(np.int64)).cuda(), torch.from_numpy(Y.view(np.int64)).cuda()
        dz = torch.empty_like(dx)
        C.batch_device(dz.data_ptr(), dx.data_ptr(), dy.data_ptr(), count, None,
                       torch.cuda.current_stream().cuda_stream)
        Z = dz.cpu().numpy().view(np.uint64)
    for i in range(0, count, max(1, count // 6)):
        assert (Z[i] == O.negmul_python(X[i], Y[i], N)).all(), (N, m, count, i)
