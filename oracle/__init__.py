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
