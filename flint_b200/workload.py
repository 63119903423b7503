"""Seeded synthetic workloads of the multiplication path.

There is no public dataset for this path: the workloads are the shapes the
reference's own benchmarks and tests exercise, generated from fixed seeds.

  splitmix_limbs(seed, n)   uniform 64-bit limbs (splitmix64), top limb != 0
  uneven_batch(seed, n)     sizes of n products: an = round(2^U), U ~ U[10, 18];
                            ratio 2^V, V ~ U[0, 4]; bn = max(1, round(an / 2^V))
"""
import numpy as np


def splitmix_limbs(seed, n):
    """n limbs from splitmix64 seeded with `seed`; the top limb is nonzero."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    if n and x[-1] == 0:
        x[-1] = 1
    return x


def uneven_batch(seed, n, log_lo=10.0, log_hi=18.0, log_ratio_hi=4.0):
    """[(an, bn)] for n products with log-uniform sizes and ratios."""
    rng = np.random.default_rng(seed)
    U = rng.uniform(log_lo, log_hi, n)
    V = rng.uniform(0.0, log_ratio_hi, n)
    an = np.rint(np.exp2(U)).astype(np.int64)
    bn = np.maximum(1, np.rint(an / np.exp2(V))).astype(np.int64)
    return [(int(a), int(b)) for a, b in zip(an, bn)]


def batch_operands(seed, sizes):
    """Concatenated operands of a batch: (limbs, [(a offset, an, b offset, bn)])."""
    total = sum(a + b for a, b in sizes)
    buf = np.empty(total, dtype=np.uint64)
    spans = []
    off = 0
    for k, (an, bn) in enumerate(sizes):
        buf[off:off + an] = splitmix_limbs(seed * 1000003 + 2 * k, an)
        buf[off + an:off + an + bn] = splitmix_limbs(seed * 1000003 + 2 * k + 1, bn)
        spans.append((off, an, off + an, bn))
        off += an + bn
    return buf, spans


def request_stream(seed, n, mpn_log=(6.0, 22.0), mpn_ratio_log=(0.0, 6.0), fmpz_len_log=(8.0, 16.0),
                   fmpz_bits=(64, 4096)):
    """n requests (kind, an, bn, aw, bw), half mpn products (an log-uniform
    in 2^mpn_log, ratio an/bn log-uniform in 2^mpn_ratio_log) and half integer
    polynomial products (lengths log-uniform in 2^fmpz_len_log, one coefficient
    bit size per request uniform in fmpz_bits, aw = bw = ceil((bits + 1) / 64))."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        if rng.random() < 0.5:
            an = int(round(2.0 ** rng.uniform(*mpn_log)))
            bn = max(1, int(round(an / 2.0 ** rng.uniform(*mpn_ratio_log))))
            out.append((0, an, bn, 1, 1))
        else:
            an = int(round(2.0 ** rng.uniform(*fmpz_len_log)))
            bn = int(round(2.0 ** rng.uniform(*fmpz_len_log)))
            bits = int(rng.integers(fmpz_bits[0], fmpz_bits[1] + 1))
            w = (bits + 1 + 63) // 64
            out.append((1, an, bn, w, w))
    return out
