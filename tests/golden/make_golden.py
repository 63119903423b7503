#!/usr/bin/env python3
"""Generate tests/golden/golden.json from the compiled reference.

Runs in the development container only (it needs oracle/_ref/libflint_ref.so,
built from the reference tree by oracle/build_ref.py).  Every case names its
inputs by generator and seed (oracle.rand_limbs / oracle.rand_below /
oracle.rand_fmpz_raw), so the
fixture stores no input data; outputs are stored in full when short and as a
blake2b-128 digest otherwise.  The GPU tests recompute the inputs and compare.

    python tests/golden/make_golden.py
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

FULL_MAX = 64   # outputs up to this many words are stored in full


def nmod_modulus(seed, bits=62):
    x = int(O.rand_limbs(seed, 1, top_nonzero=False)[0])
    return (x >> (64 - bits)) | (1 << (bits - 1)) | 1


def mpn_inputs(case):
    if case.get("fill") == "ones":
        import numpy as np
        a = np.full(case["an"], (1 << 64) - 1, dtype=np.uint64)
        b = np.full(case["bn"], (1 << 64) - 1, dtype=np.uint64)
        return a, b
    a = O.rand_limbs(case["seed_a"], case["an"])
    b = a if case.get("square") else O.rand_limbs(case["seed_b"], case["bn"])
    return a, b


def nmod_inputs(case):
    n = nmod_modulus(case["seed_n"], case["modbits"])
    a = O.rand_below(case["seed_a"], case["an"], n)
    b = a if case.get("square") else O.rand_below(case["seed_b"], case["bn"], n)
    return n, a, b


def record(z):
    z = [int(v) for v in z]
    if len(z) <= FULL_MAX:
        return {"full": ["%016x" % v for v in z]}
    return {"digest": O.digest(z), "len": len(z)}


MPN_CASES = [
    dict(name="1x1", an=1, bn=1, seed_a=11, seed_b=12),
    dict(name="2x1", an=2, bn=1, seed_a=13, seed_b=14),
    dict(name="7x5", an=7, bn=5, seed_a=15, seed_b=16),
    dict(name="32x32", an=32, bn=32, seed_a=17, seed_b=18),
    dict(name="300x3", an=300, bn=3, seed_a=19, seed_b=20),
    dict(name="1000x999", an=1000, bn=999, seed_a=21, seed_b=22),
    dict(name="ones_100x57", an=100, bn=57, fill="ones"),
    dict(name="ones_4096x4096", an=4096, bn=4096, fill="ones"),
    dict(name="square_5000", an=5000, bn=5000, seed_a=23, square=True),
    dict(name="40000x40001_np2_edge", an=40001, bn=40000, seed_a=24, seed_b=25),
    dict(name="config1_2^16x2^16", an=1 << 16, bn=1 << 16, seed_a=1, seed_b=2),
    dict(name="2^20x2^12", an=1 << 20, bn=1 << 12, seed_a=26, seed_b=27),
    dict(name="config2_2^24x2^24", an=1 << 24, bn=1 << 24, seed_a=3, seed_b=4, large=True),
    dict(name="config2b_2^24x2^20", an=1 << 24, bn=1 << 20, seed_a=5, seed_b=6, large=True),
]

NMOD_CASES = [
    dict(name="nmod_small_62", an=10, bn=7, zl=0, zh=16, seed_n=31, modbits=62, seed_a=32, seed_b=33),
    dict(name="nmod_window_64bit", an=200, bn=150, zl=100, zh=300, seed_n=34, modbits=64,
         seed_a=35, seed_b=36),
    dict(name="nmod_tiny_mod", an=1000, bn=1000, zl=0, zh=1999, seed_n=37, modbits=3,
         seed_a=38, seed_b=39),
    dict(name="nmod_square", an=777, bn=777, zl=5, zh=1600, seed_n=40, modbits=50, seed_a=41,
         square=True),
    dict(name="nmod_beyond_zn", an=50, bn=40, zl=60, zh=120, seed_n=42, modbits=62, seed_a=43,
         seed_b=44),
    dict(name="config3_2^20_mulmid", an=1 << 20, bn=1 << 20, zl=1 << 19, zh=(1 << 20) + (1 << 19),
         seed_n=7, modbits=62, seed_a=8, seed_b=9),
]


FMPZ_CASES = [
    dict(name="fmpz_1x1", an=1, bn=1, bits_a=64, bits_b=64, seed_a=51, seed_b=52),
    dict(name="fmpz_40x33_signed", an=40, bn=33, bits_a=100, bits_b=20, seed_a=53, seed_b=54),
    dict(name="fmpz_300x17_wide", an=300, bn=17, bits_a=500, bits_b=9, seed_a=55, seed_b=56),
    dict(name="fmpz_1000x999_130", an=1000, bn=999, bits_a=130, bits_b=130, seed_a=57, seed_b=58),
    dict(name="fmpz_2048x100_1000x4096", an=2048, bn=100, bits_a=1000, bits_b=4096, seed_a=59,
         seed_b=60),
    dict(name="fmpz_square_777_300", an=777, bn=777, bits_a=300, bits_b=300, seed_a=61,
         square=True),
    dict(name="fmpz_window_500x400", an=500, bn=400, bits_a=64, bits_b=64, seed_a=62, seed_b=63,
         zl=200, zh=700),
    dict(name="fmpz_2^16x2^16_4096", an=1 << 16, bn=1 << 16, bits_a=4096, bits_b=4096, seed_a=64,
         seed_b=65, large=True),
]


def fmpz_inputs(case):
    a = O.rand_fmpz_raw(case["seed_a"], case["an"], case["bits_a"])
    b = a if case.get("square") else O.rand_fmpz_raw(case["seed_b"], case["bn"], case["bits_b"])
    zw = O.fmpz_width(case["bits_a"], case["bits_b"], min(case["an"], case["bn"]))
    zn = case["an"] + case["bn"] - 1
    return a, b, zw, case.get("zl", 0), case.get("zh", zn)


# z = x y mod 2^N + 1 by the reference's sd_fft_mpn_mulmod_2expp1: digit
# sizes and counts drawn from its own test (t-sd_fft_mpn_mulmod_2expp1.c:
# 56-60), operand shapes as its switch (:109-137)
NEG_CASES = [
    dict(name="neg_b64_m16", b=64, m=16, kx="rand", ky="rand", seed=71),
    dict(name="neg_b64_m128", b=64, m=128, kx="rand", ky="rand", seed=72),
    dict(name="neg_b84_m32", b=84, m=32, kx="rand", ky="rand", seed=73),
    dict(name="neg_b88_m128", b=88, m=128, kx="rand", ky="rand", seed=74),
    dict(name="neg_b112_m64", b=112, m=64, kx="unreduced", ky="rand", seed=75),
    dict(name="neg_b126_m32", b=126, m=32, kx="rand", ky="rand", seed=76),
    dict(name="neg_b128_m16", b=128, m=16, kx="rand", ky="two_n", seed=77),
    dict(name="neg_b136_m64", b=136, m=64, kx="sparse", ky="rand", seed=78),
    dict(name="neg_b144_m128", b=144, m=128, kx="rand", ky="rand", seed=79),
    dict(name="neg_b168_m32", b=168, m=32, kx="ones", ky="ones", seed=80),
    dict(name="neg_b192_m128", b=192, m=128, kx="rand", ky="rand", seed=81),
    dict(name="neg_b34_m64", b=34, m=64, kx="rand", ky="rand", seed=82),
    dict(name="neg_b40_m128", b=40, m=128, kx="two_n", ky="two_n", seed=83),
    dict(name="neg_b46_m32", b=46, m=32, kx="rand", ky="square", seed=84),
    dict(name="neg_b50_m64", b=50, m=64, kx="unreduced", ky="unreduced", seed=85),
    dict(name="neg_b50_m128_zero", b=50, m=128, kx="zero", ky="rand", seed=86),
]


def neg_inputs(case):
    N = case["b"] * case["m"]
    n = N // 64
    x = O.neg_operand(case["seed"], n, case["kx"])
    y = x if case["ky"] == "square" else O.neg_operand(case["seed"] + 1000, n, case["ky"])
    return N, x, y


def main():
    if not O.have_ref():
        raise SystemExit("oracle/_ref/libflint_ref.so missing: run python oracle/build_ref.py")
    O.ref().flint_set_num_threads(os.cpu_count() or 1)
    out = {"generator": "oracle.rand_limbs / oracle.rand_below (splitmix64)",
           "source": "reference fft_small (oracle/_ref/libflint_ref.so)",
           "mpn": [], "nmod": [], "fmpz": [], "neg": []}
    for case in MPN_CASES:
        t = time.time()
        a, b = mpn_inputs(case)
        z = O.ref_mpn_mul(a, b)
        out["mpn"].append(dict(case, **record(z)))
        print("%-28s %.2fs" % (case["name"], time.time() - t))
    for case in NMOD_CASES:
        t = time.time()
        n, a, b = nmod_inputs(case)
        z = O.ref_nmod_mul_mid(case["zl"], case["zh"], a, b, n)
        out["nmod"].append(dict(case, modulus="%x" % n, **record(z)))
        print("%-28s %.2fs" % (case["name"], time.time() - t))
    for case in NEG_CASES:
        t = time.time()
        N, x, y = neg_inputs(case)
        z = O.ref_mulmod_2expp1(x, y, N, case["m"])
        out["neg"].append(dict(case, N=N, **record(z)))
        print("%-28s %.2fs" % (case["name"], time.time() - t))
    for case in FMPZ_CASES:
        t = time.time()
        a, b, zw, zl, zh = fmpz_inputs(case)
        z = O.ref_fmpz_poly_mul_raw(a, b, zw)[zl:zh]
        out["fmpz"].append(dict(case, zw=zw, **record(z.reshape(-1))))
        print("%-28s %.2fs" % (case["name"], time.time() - t))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
