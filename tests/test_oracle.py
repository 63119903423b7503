"""Pin the oracle before trusting it (CPU only).

The plain-C restatement (oracle/fft_small_oracle.c) is checked against the
golden fixtures produced by the reference itself, against GMP's mpn_mul,
against Python integers, and -- where the compiled reference is present --
against the reference directly on fresh seeded inputs.  These mirror the
reference's own randomized property tests (src/fft_small/test/t-mul.c:17-101
vs GMP, t-nmod_poly_mul.c:18-268 vs a classical product).
"""
import numpy as np
import pytest

import oracle as O
from tests.golden.make_golden import mpn_inputs, nmod_inputs


def _check_record(rec, z):
    if "full" in rec:
        assert ["%016x" % int(v) for v in z] == rec["full"]
    else:
        assert len(z) == rec["len"]
        assert O.digest(z) == rec["digest"]


@pytest.mark.parametrize("i", range(12))
def test_port_matches_golden_mpn(golden, i):
    case = golden["mpn"][i]
    if case.get("large") or case["an"] + case["bn"] > 40000:
        pytest.skip("large case is covered on the GPU")
    a, b = mpn_inputs(case)
    _check_record(case, O.port_mpn_mul(a, b))


@pytest.mark.parametrize("i", range(5))
def test_port_matches_golden_nmod(golden, i):
    case = golden["nmod"][i]
    n, a, b = nmod_inputs(case)
    _check_record(case, O.port_nmod_mul_mid(case["zl"], case["zh"], a, b, n))


def test_golden_fixture_covers_configs(golden):
    names = [c["name"] for c in golden["mpn"]] + [c["name"] for c in golden["nmod"]]
    for want in ("config1_2^16x2^16", "config2_2^24x2^24", "config2b_2^24x2^20",
                 "config3_2^20_mulmid"):
        assert want in names


@pytest.mark.parametrize("seed", range(6))
def test_port_vs_gmp_and_python(seed):
    rng = np.random.default_rng(seed)
    an = int(rng.integers(1, 3000))
    bn = int(rng.integers(1, 3000))
    a = O.rand_limbs(1000 + seed, an)
    b = O.rand_limbs(2000 + seed, bn)
    z = O.port_mpn_mul(a, b)
    assert (z == O.gmp_mpn_mul(a, b)).all()
    assert O.to_int(z) == O.to_int(a) * O.to_int(b)


def test_port_edge_cases():
    ones = np.full(77, (1 << 64) - 1, dtype=np.uint64)
    z = O.port_mpn_mul(ones, ones[:13])
    assert O.to_int(z) == O.to_int(ones) * O.to_int(ones[:13])
    zero = np.zeros(5, dtype=np.uint64)
    assert (O.port_mpn_mul(zero, ones[:3]) == 0).all()
    a = O.rand_limbs(5, 400)
    assert (O.port_mpn_mul(a, a) == O.gmp_mpn_mul(a, a)).all()


@pytest.mark.parametrize("seed", range(4))
def test_port_nmod_vs_python(seed):
    rng = np.random.default_rng(100 + seed)
    an, bn = int(rng.integers(1, 120)), int(rng.integers(1, 120))
    bits = int(rng.integers(2, 65))
    n = (int(O.rand_limbs(seed, 1, False)[0]) >> (64 - bits)) | (1 << (bits - 1))
    n = max(n, 2)
    a, b = O.rand_below(seed, an, n), O.rand_below(seed + 50, bn, n)
    zl = int(rng.integers(0, an + bn))
    zh = zl + int(rng.integers(1, an + bn + 5))
    z = O.port_nmod_mul_mid(zl, zh, a, b, n)
    zn = an + bn - 1
    ref = O.nmod_mul_mid_python(zl, min(zh, zn), a, b, n) if zl < zn else np.zeros(0, np.uint64)
    assert (z[:len(ref)] == ref).all()
    assert (z[len(ref):] == 0).all()


def test_port_context_matches_reference_primes():
    """The restated prime walk reproduces the primes listed in the reference
    (src/fft_small/mpn_mul.c:65-72)."""
    want = [1108307720798209, 659706976665601, 1086317488242689, 910395627798529,
            699289395265537, 1022545813831681, 1013749720809473, 868614185943041]
    assert [O.port().oracle_prime(i) for i in range(8)] == want


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("seed", range(4))
def test_port_vs_compiled_reference(seed):
    rng = np.random.default_rng(7 + seed)
    an = int(rng.integers(1, 60000))
    bn = int(rng.integers(1, 60000))
    a, b = O.rand_limbs(300 + seed, an), O.rand_limbs(400 + seed, bn)
    assert (O.port_mpn_mul(a, b) == O.ref_mpn_mul(a, b)).all()


# ---------------------------------------------------------------- integer polynomials
@pytest.mark.parametrize("name", ["fmpz_1x1", "fmpz_40x33_signed", "fmpz_300x17_wide",
                                  "fmpz_1000x999_130", "fmpz_2048x100_1000x4096",
                                  "fmpz_square_777_300", "fmpz_window_500x400"])
def test_python_fmpz_matches_golden(golden, name):
    """The Python Kronecker restatement reproduces the reference's
    _fmpz_poly_mul outputs stored in the fixtures."""
    from tests.golden.make_golden import fmpz_inputs
    case = next(c for c in golden["fmpz"] if c["name"] == name)
    a, b, zw, zl, zh = fmpz_inputs(case)
    z = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))[zl:zh]
    flat = O.ints_to_raw(z, zw).reshape(-1)
    if "full" in case:
        assert ["%016x" % int(v) for v in flat] == case["full"]
    else:
        assert O.digest(flat) == case["digest"] and len(flat) == case["len"]


def test_fmpz_raw_round_trip():
    r = O.rand_fmpz_raw(3, 50, 200)
    vals = O.raw_to_ints(r)
    assert any(v < 0 for v in vals) and any(v > 0 for v in vals)
    assert max(abs(v) for v in vals) < 1 << 200
    assert (O.ints_to_raw(vals, r.shape[1]) == r).all()


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("seed", range(3))
def test_python_fmpz_vs_compiled_reference(seed):
    an, bn = 50 + 37 * seed, 20 + 11 * seed
    ba, bb = 64 * seed + 30, 500 - 100 * seed
    a, b = O.rand_fmpz_raw(seed + 70, an, ba), O.rand_fmpz_raw(seed + 80, bn, bb)
    zw = O.fmpz_width(ba, bb, min(an, bn))
    want = O.raw_to_ints(O.ref_fmpz_poly_mul_raw(a, b, zw))
    assert O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b)) == want


# ---------------------------------------------------------------- cost model network
def test_mlp_oracle_gradient_matches_finite_differences():
    """Pins the NumPy network (the checker of the CUDA kernels) by central
    differences of its own loss in float64."""
    from oracle import mlp_ref
    rng = np.random.default_rng(3)
    n_in, n = 16, 40
    P = rng.normal(0, 0.3, mlp_ref.offsets(n_in)["total"])
    X = rng.normal(0, 1, (n, n_in))
    t = rng.normal(0, 1, n)
    g = mlp_ref.gradient(P, X, t)
    idx = rng.choice(len(P), 60, replace=False)
    h = 1e-6
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd = (mlp_ref.loss(Pp, X, t) - mlp_ref.loss(Pm, X, t)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn,lo", [(300, 200, 0), (300, 200, 250), (4000, 3999, 1),
                                      (4000, 1000, 4990), (20000, 10000, 10000)])
def test_reference_range_contract(an, bn, lo):
    """The contract the GPU window product is held to, checked on the
    reference's own _mpn_ctx_mpn_mul_range output (pins the checker)."""
    a, b = O.rand_limbs(an * 3 + lo, an), O.rand_limbs(bn * 5 + lo, bn)
    z = O.ref_mpn_mul_range(lo, an + bn, a, b)
    O.check_mul_range_contract(a, b, lo, z)


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn,bits", [(50, 20, 20), (3000, 1200, 63), (500, 499, 2)])
def test_nmod_divrem_python_satisfies_identity(an, bn, bits):
    """Schoolbook division (the small-size checker) against the identity
    a = q b + r, with q b from the reference's own multiplication; a planted
    error in r is caught."""
    n = (1 << (bits - 1)) + 1 if bits > 2 else 3
    a, b = O.rand_below(an, an, n), O.rand_below(bn, bn, n)
    b[-1] = max(int(b[-1]), 1)
    q, r = O.nmod_divrem_python(a, b, n)
    assert O.check_nmod_divrem(a, b, n, q, r)
    if r:
        r[0] = (r[0] + 1) % n
        assert not O.check_nmod_divrem(a, b, n, q, r)


# ------------------------------------------------ products mod 2^N + 1
def test_golden_covers_negacyclic(golden):
    assert len(golden["neg"]) >= 12


@pytest.mark.parametrize("i", range(16))
def test_negmul_oracles_match_golden(golden, i):
    """Both restatements (a folded Python product, and the reference's
    digit/bias/fold algorithm) reproduce the reference's outputs."""
    from tests.golden.make_golden import neg_inputs
    case = golden["neg"][i]
    N, x, y = neg_inputs(case)
    _check_record(case, O.negmul_python(x, y, N))
    if case["m"] <= 64:
        _check_record(case, O.negacyclic_digits_python(x, y, N, case["m"]))


@pytest.mark.parametrize("seed", range(4))
def test_negmul_oracle_vs_reference(seed):
    if not O.have_ref():
        pytest.skip("compiled reference absent")
    rng = np.random.default_rng(seed)
    b = int(rng.choice([34, 40, 46, 50, 64, 84, 88, 128]))
    m = 16 << int(rng.integers(0, 4))
    N = b * m
    if N % 64:
        pytest.skip("N not a multiple of 64")
    n = N // 64
    for kx, ky in (("rand", "rand"), ("unreduced", "two_n"), ("ones", "sparse")):
        x = O.neg_operand(300 + seed, n, kx)
        y = O.neg_operand(400 + seed, n, ky)
        assert (O.negmul_python(x, y, N) == O.ref_mulmod_2expp1(x, y, N, m)).all()


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("an,bn,n", [(30, 7, 1000003), (500, 40, (1 << 61) + 15), (200, 199, 7),
                                     (3000, 2000, 7340033), (9000, 4000, (1 << 63) + 29)])
def test_reference_divrem_pinned(an, bn, n):
    """The reference's own _nmod_poly_divrem_mpn_ctx (compiled with the
    generic-ring modules its series inverse needs) against schoolbook
    division in Python at small sizes and the identity a = q b + r above."""
    import math
    a = O.rand_below(an + 1, an, n)
    b = O.rand_below(bn + 2, bn, n)
    while math.gcd(int(b[-1]), n) != 1:
        b[-1] = (int(b[-1]) + 1) % n
    q, r = O.ref_nmod_divrem(a, b, n)
    assert O.check_nmod_divrem(a, b, n, q, r)
    if an <= 500:
        qp, rp = O.nmod_divrem_python(a, b, n)
        assert [int(x) for x in q] == qp and [int(x) for x in r] == rp
