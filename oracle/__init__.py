"""Oracle for the small-prime NTT multiplication path.  TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs use this package, and only as the checker or as the timed CPU baseline;
the product (flint_b200) never imports it.

Three independent exact references are available:

* ``port()``  -- the plain-C restatement of the reference algorithm
  (oracle/fft_small_oracle.c), compiled into oracle/liboracle.so;
* ``ref()``   -- the reference's own fft_small code compiled from the
  reference tree by oracle/build_ref.py into oracle/_ref/libflint_ref.so
  (absent when that build has not been run);
* ``gmp()``   -- GMP's mpn_mul from the system libgmp.so.10.

Inputs come from ``rand_limbs`` (splitmix64, seed -> limbs), so every test,
fixture and benchmark regenerates the same operands bit for bit.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libflint_ref.so")

_port = _ref = _gmp = None


class NmodT(ctypes.Structure):
    """nmod_t of the reference (src/flint.h.in:440-447), passed by value."""
    _fields_ = [("n", ctypes.c_ulong), ("ninv", ctypes.c_ulong), ("norm", ctypes.c_ulong)]


def build_port(force=False):
    src = os.path.join(HERE, "fft_small_oracle.c")
    if (not force and os.path.exists(PORT_SO)
            and os.path.getmtime(PORT_SO) >= os.path.getmtime(src)):
        return PORT_SO
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-o", PORT_SO, src, "-lm"], check=True)
    return PORT_SO


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            build_port()
        L = ctypes.CDLL(PORT_SO)
        U, P = ctypes.c_ulong, ctypes.c_void_p
        L.oracle_mpn_mul.argtypes = [P, P, U, P, U]
        L.oracle_mpn_mul.restype = ctypes.c_int
        L.oracle_nmod_mul_mid.argtypes = [P, U, U, P, U, P, U, U]
        L.oracle_nmod_mul_mid.restype = ctypes.c_int
        L.oracle_prime.argtypes = [ctypes.c_int]
        L.oracle_prime.restype = U
        _port = L
    return _port


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_SO)
        U, S, P = ctypes.c_ulong, ctypes.c_long, ctypes.c_void_p
        L.mpn_mul_default_mpn_ctx.argtypes = [P, P, S, P, S]
        L.mpn_mul_default_mpn_ctx.restype = None
        L.get_default_mpn_ctx.restype = P
        L.mpn_ctx_mpn_mul.argtypes = [P, P, P, U, P, U]
        L.mpn_ctx_mpn_mul.restype = None
        L._nmod_poly_mul_mid_mpn_ctx.argtypes = [P, U, U, P, U, P, U, NmodT, P]
        L._nmod_poly_mul_mid_mpn_ctx.restype = None
        L.flint_set_num_threads.argtypes = [ctypes.c_int]
        L.flint_get_num_threads.restype = ctypes.c_int
        L.n_preinvert_limb.argtypes = [U]
        L.n_preinvert_limb.restype = U
        L._nmod_poly_divrem_mpn_ctx.argtypes = [P, P, P, U, P, U, NmodT, P]
        L._nmod_poly_divrem_mpn_ctx.restype = None
        _ref = L
    return _ref


def gmp():
    global _gmp
    if _gmp is None:
        for cand in ("/usr/lib/x86_64-linux-gnu/libgmp.so.10", "libgmp.so.10"):
            try:
                L = ctypes.CDLL(cand)
                break
            except OSError:
                L = None
        if L is None:
            raise OSError("libgmp.so.10 not found")
        P, S = ctypes.c_void_p, ctypes.c_long
        L.__gmpn_mul.argtypes = [P, P, S, P, S]
        L.__gmpn_mul.restype = ctypes.c_ulong
        _gmp = L
    return _gmp


# ---------------------------------------------------------------- inputs
_MASK = (1 << 64) - 1


def rand_limbs(seed, n, top_nonzero=True):
    """n uniform 64-bit limbs from splitmix64(seed); vectorised."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & _MASK) + i * np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    if top_nonzero and n and x[-1] == 0:
        x[-1] = 1
    return x


def rand_below(seed, n, m):
    """n values uniform in [0, m) (m < 2^64) by rejection-free 128-bit scaling."""
    x = rand_limbs(seed, n, top_nonzero=False)
    # floor(x * m / 2^64) -- exact via splitting into 32-bit halves
    m = int(m)
    lo = x & np.uint64(0xFFFFFFFF)
    hi = x >> np.uint64(32)
    mlo, mhi = np.uint64(m & 0xFFFFFFFF), np.uint64(m >> 32)
    with np.errstate(over="ignore"):
        t1 = lo * mlo
        t2 = hi * mlo + (t1 >> np.uint64(32))
        t3 = lo * mhi + (t2 & np.uint64(0xFFFFFFFF))
        return hi * mhi + (t2 >> np.uint64(32)) + (t3 >> np.uint64(32))


# ---------------------------------------------------------------- products
def to_int(x):
    return int.from_bytes(np.ascontiguousarray(x, dtype=np.uint64).tobytes(), "little")


def from_int(v, n):
    return np.frombuffer(v.to_bytes(8 * n, "little"), dtype=np.uint64).copy()


def port_mpn_mul(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    z = np.zeros(len(a) + len(b), dtype=np.uint64)
    rc = port().oracle_mpn_mul(z.ctypes.data, a.ctypes.data, len(a), b.ctypes.data, len(b))
    if rc:
        raise RuntimeError("oracle_mpn_mul failed")
    return z


def port_nmod_mul_mid(zl, zh, a, b, n):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    z = np.zeros(max(zh - zl, 0), dtype=np.uint64)
    rc = port().oracle_nmod_mul_mid(z.ctypes.data, zl, zh, a.ctypes.data, len(a),
                                    b.ctypes.data, len(b), n)
    if rc:
        raise RuntimeError("oracle_nmod_mul_mid failed")
    return z


def ref_mpn_mul(a, b):
    """The reference's own mpn_ctx_mpn_mul on its default context."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    if len(a) < len(b):
        a, b = b, a
    z = np.zeros(len(a) + len(b), dtype=np.uint64)
    ref().mpn_mul_default_mpn_ctx(z.ctypes.data, a.ctypes.data, len(a), b.ctypes.data, len(b))
    return z


def ref_nmod_mul_mid(zl, zh, a, b, n):
    """The reference's _nmod_poly_mul_mid_mpn_ctx on its default context."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    L = ref()
    norm = 64 - int(n).bit_length()
    ninv = L.n_preinvert_limb(n << norm)
    z = np.zeros(max(zh - zl, 0), dtype=np.uint64)
    L._nmod_poly_mul_mid_mpn_ctx(z.ctypes.data, zl, zh, a.ctypes.data, len(a), b.ctypes.data,
                                 len(b), NmodT(n, ninv, norm), L.get_default_mpn_ctx())
    return z


def gmp_mpn_mul(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    if len(a) < len(b):
        a, b = b, a
    z = np.zeros(len(a) + len(b), dtype=np.uint64)
    gmp().__gmpn_mul(z.ctypes.data, a.ctypes.data, len(a), b.ctypes.data, len(b))
    return z


def nmod_mul_mid_python(zl, zh, a, b, n):
    """Schoolbook window product mod n in Python integers (small sizes)."""
    a = [int(x) for x in a]
    b = [int(x) for x in b]
    out = []
    for k in range(zl, zh):
        s = 0
        for i in range(max(0, k - len(b) + 1), min(k, len(a) - 1) + 1):
            s += a[i] * b[k - i]
        out.append(s % n)
    return np.array(out, dtype=np.uint64)


def digest(z):
    """Short content hash of a limb vector, for fixtures of large outputs."""
    import hashlib
    return hashlib.blake2b(np.ascontiguousarray(z, dtype=np.uint64).tobytes(),
                           digest_size=16).hexdigest()


# ---------------------------------------------------------------- integer polynomials
# Coefficients travel as fixed-width two's complement limb rows (w limbs per
# coefficient), the raw form of the GPU library; fmpz vectors of the
# reference are built and read with its own fmpz_set_signed_ui_array /
# fmpz_get_signed_ui_array (src/fmpz.h:238-239).

def rand_fmpz_raw(seed, n, bits, w=None):
    """n signed coefficients uniform in (-2^bits, 2^bits) as an (n, w) uint64
    two's complement array, w = ceil((bits + 1) / 64) unless given."""
    wm = (bits + 63) // 64
    w = w or (bits + 1 + 63) // 64
    mag = rand_limbs(seed, n * wm, top_nonzero=False).reshape(n, wm)
    if bits % 64:
        mag[:, -1] &= np.uint64((1 << (bits % 64)) - 1)
    out = np.zeros((n, w), dtype=np.uint64)
    out[:, :wm] = mag
    neg = (rand_limbs(seed ^ 0x5DEECE66D, n, top_nonzero=False) & np.uint64(1)).astype(bool)
    rows = out[neg]
    rows = ~rows
    carry = np.ones(len(rows), dtype=np.uint64)
    with np.errstate(over="ignore"):
        for k in range(w):
            v = rows[:, k] + carry
            carry = ((v == 0) & (carry == 1)).astype(np.uint64)
            rows[:, k] = v
    out[neg] = rows
    return out


def fmpz_width(bits_a, bits_b, mn):
    """Limbs per product coefficient for factors below 2^bits_a, 2^bits_b in
    magnitude, at most mn terms per coefficient, plus a sign bit."""
    return (bits_a + bits_b + (mn - 1).bit_length() + 1 + 63) // 64


def raw_to_ints(raw):
    """Signed integers of an (n, w) two's complement limb array."""
    raw = np.ascontiguousarray(raw, dtype=np.uint64)
    w = raw.shape[1]
    top = 1 << (64 * w)
    res = []
    for row in raw:
        v = int.from_bytes(row.tobytes(), "little")
        res.append(v - top if v >> (64 * w - 1) else v)
    return res


def ints_to_raw(vals, w):
    out = np.zeros((len(vals), w), dtype=np.uint64)
    mod = 1 << (64 * w)
    for i, v in enumerate(vals):
        out[i] = np.frombuffer((v % mod).to_bytes(8 * w, "little"), dtype=np.uint64)
    return out


def fmpz_poly_mul_python(a, b):
    """Exact product of integer polynomials (lists of ints) by Kronecker
    substitution in Python integers; for test sizes."""
    if not a or not b:
        return []
    ma = max(abs(x) for x in a)
    mb = max(abs(x) for x in b)
    k = ma.bit_length() + mb.bit_length() + min(len(a), len(b)).bit_length() + 2

    def pack(p):
        v = 0
        for x in reversed(p):
            v = (v << k) + x
        return v

    c = pack(a) * pack(b)
    out = []
    half, full = 1 << (k - 1), 1 << k
    for _ in range(len(a) + len(b) - 1):
        d = c & (full - 1)
        if d >= half:
            d -= full
        out.append(d)
        c = (c - d) >> k
    assert c == 0
    return out


def _ref_fmpz():
    L = ref()
    if not getattr(L, "_fmpz_ready", False):
        P, S = ctypes.c_void_p, ctypes.c_long
        L._fmpz_vec_init.argtypes = [S]
        L._fmpz_vec_init.restype = P
        L._fmpz_vec_clear.argtypes = [P, S]
        L._fmpz_vec_clear.restype = None
        L.fmpz_set_signed_ui_array.argtypes = [P, P, S]
        L.fmpz_set_signed_ui_array.restype = None
        L.fmpz_get_signed_ui_array.argtypes = [P, S, P]
        L.fmpz_get_signed_ui_array.restype = None
        L._fmpz_poly_mul.argtypes = [P, P, S, P, S]
        L._fmpz_poly_mul.restype = None
        L._fmpz_poly_mul_mid_mpn_ctx.argtypes = [P, ctypes.c_ulong, ctypes.c_ulong, P,
                                                 ctypes.c_ulong, P, ctypes.c_ulong, P]
        L._fmpz_poly_mul_mid_mpn_ctx.restype = ctypes.c_int
        L._fmpz_vec_equal.argtypes = [P, P, S]
        L._fmpz_vec_equal.restype = ctypes.c_int
        L._fmpz_ready = True
    return L


class RefFmpzVec:
    """An fmpz vector allocated by the reference library."""

    def __init__(self, n):
        self.L = _ref_fmpz()
        self.n = n
        self.ptr = self.L._fmpz_vec_init(max(n, 1))

    def set_raw(self, raw):
        raw = np.ascontiguousarray(raw, dtype=np.uint64)
        w = raw.shape[1]
        for i in range(self.n):
            self.L.fmpz_set_signed_ui_array(self.ptr + 8 * i, raw[i].ctypes.data, w)
        return self

    def get_raw(self, w):
        out = np.zeros((self.n, w), dtype=np.uint64)
        for i in range(self.n):
            self.L.fmpz_get_signed_ui_array(out[i].ctypes.data, w, self.ptr + 8 * i)
        return out

    def close(self):
        if self.ptr:
            self.L._fmpz_vec_clear(self.ptr, max(self.n, 1))
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ref_fmpz_poly_mul_raw(a_raw, b_raw, zw):
    """The reference's _fmpz_poly_mul (src/fmpz_poly/mul.c:100-186) on raw
    coefficient rows; returns the (an + bn - 1, zw) raw product."""
    an, bn = len(a_raw), len(b_raw)
    if an < bn:
        a_raw, b_raw, an, bn = b_raw, a_raw, bn, an
    L = _ref_fmpz()
    with RefFmpzVec(an) as A, RefFmpzVec(bn) as B, RefFmpzVec(an + bn - 1) as Z:
        A.set_raw(a_raw)
        B.set_raw(b_raw)
        L._fmpz_poly_mul(Z.ptr, A.ptr, an, B.ptr, bn)
        return Z.get_raw(zw)


def ref_mpn_mul_range(lo, hi, a, b):
    """The reference's _mpn_ctx_mpn_mul_range (src/fft_small/mpn_mul.c:1617-1978)
    on its default context: limbs [lo, hi) of a * b, a lower approximation
    for lo > 0."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
    if len(a) < len(b):
        a, b = b, a
    L = ref()
    if not getattr(L, "_range_ready", False):
        P, U = ctypes.c_void_p, ctypes.c_ulong
        L._mpn_ctx_mpn_mul_range.argtypes = [P, P, U, U, P, U, P, U]
        L._mpn_ctx_mpn_mul_range.restype = None
        L._range_ready = True
    z = np.zeros(max(hi - lo, 0), dtype=np.uint64)
    if hi > lo:
        L._mpn_ctx_mpn_mul_range(L.get_default_mpn_ctx(), z.ctypes.data, lo, hi, a.ctypes.data,
                                 len(a), b.ctypes.data, len(b))
    return z


def check_mul_range_contract(a, b, lo, z):
    """The contract of _mpn_ctx_mpn_mul_range (src/fft_small/test/t-mpn_mulmid.c:
    96-117) for z = limbs [lo, an + bn): a lower approximation of
    floor(a b / 2^(64 lo)) with deficit <= min(an, bn, lo) 2^64, exact for
    lo = 0.  Returns the deficit."""
    an, bn = len(a), len(b)
    exact = (to_int(a) * to_int(b)) >> (64 * lo)
    d = exact - to_int(z)
    assert d >= 0, "not a lower approximation"
    assert d <= min(an, bn, lo) << 64, "deficit exceeds min(an, bn, lo) 2^64"
    if lo == 0:
        assert d == 0, "lo = 0 must be exact"
    return d


def ref_nmod_divrem(a, b, n):
    """The reference's own _nmod_poly_divrem_mpn_ctx (src/fft_small/
    nmod_poly_mul.c:1248-1277) on its default context: (q, r) with
    a = q b + r mod n, r of bn - 1 coefficients (b's leading coefficient a
    unit mod n, bn >= 2)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    L = ref()
    norm = 64 - int(n).bit_length()
    ninv = L.n_preinvert_limb(n << norm)
    an, bn = len(a), len(b)
    q = np.zeros(an - bn + 1, dtype=np.uint64)
    r = np.zeros(bn - 1, dtype=np.uint64)
    L._nmod_poly_divrem_mpn_ctx(q.ctypes.data, r.ctypes.data, a.ctypes.data, an, b.ctypes.data, bn,
                                NmodT(n, ninv, norm), L.get_default_mpn_ctx())
    return q, r


def check_nmod_divrem(a, b, n, q, r):
    """a = q b + r mod n with r of bn - 1 coefficients, checked with the
    reference's own _nmod_poly_mul_mid_mpn_ctx for the product q b.
    Quotient and remainder are unique when b's leading coefficient is a
    unit, so the identity pins them (ref_nmod_divrem gives the reference's
    own division for a direct comparison)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    an, bn = len(a), len(b)
    assert len(q) == an - bn + 1 and len(r) == bn - 1
    qb = ref_nmod_mul_mid(0, an, np.ascontiguousarray(q, dtype=np.uint64), np.ascontiguousarray(b, dtype=np.uint64), n)
    rr = np.zeros(an, dtype=object)
    rr[:bn - 1] = [int(x) for x in r]
    lhs = [(int(x) - int(y)) % n for x, y in zip(a, rr)]
    return lhs == [int(x) for x in qb]


def nmod_divrem_python(a, b, n):
    """Schoolbook division with remainder mod n in Python integers (small sizes)."""
    a = [int(x) % n for x in a]
    b = [int(x) % n for x in b]
    inv = pow(b[-1], -1, n)
    qn = len(a) - len(b) + 1
    q = [0] * qn
    for k in range(qn - 1, -1, -1):
        c = a[k + len(b) - 1] * inv % n
        q[k] = c
        if c:
            for j in range(len(b)):
                a[k + j] = (a[k + j] - c * b[j]) % n
    return q, a[:len(b) - 1]


# ---------------------------------------------------------------- mod 2^N + 1
def negmul_python(x, y, N):
    """z = x y mod 2^N + 1 by Python integers.  x, y have n + 1 limbs
    (N = 64 n; the top limb 0 or 1, possibly unreduced); z is the unique
    representative in [0, 2^N] in n + 1 limbs.  The same check the reference
    uses, a full product folded once (src/fft_small/test/
    t-sd_fft_mpn_mulmod_2expp1.c:21-48)."""
    n = N // 64
    v = to_int(x) * to_int(y)
    # one fold (2^N = -1) leaves |v| < 2^(N+2): the final % has a tiny quotient
    v = ((v & ((1 << N) - 1)) - (v >> N)) % ((1 << N) + 1)
    return from_int(v, n + 1)


def negacyclic_digits_python(x, y, N, m):
    """The reference's negacyclic algorithm restated on Python integers, small
    m only (src/fft_small/negacyclic.c): b-bit digits with digit 0 lowered by
    the top limb (negacyclic.c:243-289, 322-323), the negacyclic convolution
    of the digit vectors (there: twist by w^i, cyclic transforms, untwist by
    w^-i m^-1, negacyclic.c:327-438; here: schoolbook), biased coefficients
    c_i + B with B = 2^(2b + log2 m) (negacyclic.c:137-161, 429-438), their sum
    at bit offsets b i minus the bias polynomial and the fold of the part
    above 2^N (negacyclic.c:440-488)."""
    n = N // 64
    b = N // m
    depth = m.bit_length() - 1
    mask = (1 << b) - 1

    def digits(v):
        lo = to_int(np.asarray(v, dtype=np.uint64)[:n])
        d = [(lo >> (b * i)) & mask for i in range(m)]
        d[0] -= int(int(v[n]) != 0)
        return d

    dx, dy = digits(x), digits(y)
    B = 1 << (2 * b + depth)
    c = [0] * m
    for i in range(m):
        xi = dx[i]
        if xi == 0:
            continue
        for j in range(m):
            k = i + j
            if k < m:
                c[k] += xi * dy[j]
            else:
                c[k - m] -= xi * dy[j]
    W = 0
    bias = 0
    for i in range(m):
        assert 0 <= c[i] + B < 2 * B
        W += (c[i] + B) << (b * i)
        bias += B << (b * i)
    w = W - bias
    lo, hi = w & ((1 << N) - 1), w >> N      # hi signed (arithmetic shift)
    return from_int((lo - hi) % ((1 << N) + 1), n + 1)


class _RefNegCtx:
    """sd_fft_mpn_mulmod_2expp1 of the compiled reference, for small
    configurations its own test covers (src/fft_small/test/
    t-sd_fft_mpn_mulmod_2expp1.c:53-80): the context struct is held in an
    opaque buffer, its leading fields N, b, m, depth, np read back."""

    def __init__(self, N, m):
        L = ref()
        P, S = ctypes.c_void_p, ctypes.c_long
        for name, args in (("sd_fft_mpn_mulmod_2expp1_ctx_init", [P, P, S, S]),
                           ("sd_fft_mpn_mulmod_2expp1_ctx_clear", [P]),
                           ("sd_fft_mpn_mulmod_2expp1_scratch_init", [P, P]),
                           ("sd_fft_mpn_mulmod_2expp1_scratch_clear", [P]),
                           ("sd_fft_mpn_mulmod_2expp1", [P, P, P, P, P])):
            getattr(L, name).argtypes = args
            getattr(L, name).restype = None
        self.L = L
        self.C = ctypes.create_string_buffer(16384)
        self.S = ctypes.create_string_buffer(256)
        L.sd_fft_mpn_mulmod_2expp1_ctx_init(self.C, L.get_default_mpn_ctx(), N, m)
        L.sd_fft_mpn_mulmod_2expp1_scratch_init(self.S, self.C)
        f = np.frombuffer(self.C.raw[:40], dtype=np.int64)
        self.N, self.b, self.m, self.depth, self.np = (int(v) for v in f)

    def mul(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        y = x if y is x else np.ascontiguousarray(y, dtype=np.uint64)
        z = np.zeros(self.N // 64 + 1, dtype=np.uint64)
        self.L.sd_fft_mpn_mulmod_2expp1(self.C, z.ctypes.data, x.ctypes.data, y.ctypes.data,
                                        self.S)
        return z

    def close(self):
        if self.C is not None:
            self.L.sd_fft_mpn_mulmod_2expp1_scratch_clear(self.S)
            self.L.sd_fft_mpn_mulmod_2expp1_ctx_clear(self.C)
            self.C = None


def ref_mulmod_2expp1(x, y, N, m):
    """The reference's sd_fft_mpn_mulmod_2expp1 on its default context."""
    R = _RefNegCtx(N, m)
    try:
        return R.mul(x, y)
    finally:
        R.close()


def neg_operand(seed, n, kind="rand"):
    """An (n + 1)-limb operand of the shapes the reference's test draws
    (t-sd_fft_mpn_mulmod_2expp1.c:109-137): random low limbs with top limb 0,
    "two_n" (2^N), "unreduced" (top limb 1 over random low limbs), "sparse"
    (one random limb), "ones" (all low limbs 2^64 - 1), "zero"."""
    x = np.zeros(n + 1, dtype=np.uint64)
    if kind == "rand":
        x[:n] = rand_limbs(seed, n, top_nonzero=False)
    elif kind == "two_n":
        x[n] = 1
    elif kind == "unreduced":
        x[:n] = rand_limbs(seed, n, top_nonzero=False)
        x[n] = 1
    elif kind == "sparse":
        r = rand_limbs(seed, 2, top_nonzero=False)
        x[int(r[0]) % n] = r[1]
    elif kind == "ones":
        x[:n] = np.uint64((1 << 64) - 1)
    elif kind != "zero":
        raise ValueError(kind)
    return x
