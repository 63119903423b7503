#!/usr/bin/env python3
"""Build recipe: the reference's own fft_small tests run against the GPU path
from C (test infrastructure only).

The reference's test programs ``src/fft_small/test/t-mul.c``,
``t-nmod_poly_mul.c``, ``t-fmpz_poly_mul.c`` and ``t-nmod_poly_divrem.c`` are
compiled unchanged from the reference tree, with the entry points under test renamed by the preprocessor
to the C shim of this repository (``flint_b200/shim/fft_small_gpu_shim.c``):

    mpn_ctx_mpn_mul              -> gpu_shim_mpn_ctx_mpn_mul
    _mpn_ctx_mpn_mul_range       -> gpu_shim__mpn_ctx_mpn_mul_range
    _nmod_poly_mul_mid_mpn_ctx   -> gpu_shim__nmod_poly_mul_mid_mpn_ctx
    _fmpz_poly_mul_mid_mpn_ctx   -> gpu_shim__fmpz_poly_mul_mid_mpn_ctx
    _nmod_poly_divrem_mpn_ctx    -> gpu_shim__nmod_poly_divrem_mpn_ctx

so every product they check comes from libflint_b200.so through its C ABI,
while their yardsticks (GMP's mpn_mul / mpn_sqr, _nmod_poly_mul_KS,
_fmpz_poly_mul_KS, the generic _nmod_poly_divrem) and their harness (random states, TEST_MAIN) come from
the compiled reference (oracle/_ref/libflint_ref.so, build_ref.py).  A small
generated main file lists the four test functions.  The binary,
``oracle/_ref/t-gpu-fft_small``, finds both libraries through its run path;
tests/test_c_caller_gpu.py runs it on a GPU.  Nothing is written outside
oracle/_ref.  Usage::

    python oracle/build_ref_tests.py [--ref DIR]
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
import build_ref  # noqa: E402

OUT = build_ref.OUT
BINARY = os.path.join(OUT, "t-gpu-fft_small")
RENAMES = {
    "mpn_ctx_mpn_mul": "gpu_shim_mpn_ctx_mpn_mul",
    "_mpn_ctx_mpn_mul_range": "gpu_shim__mpn_ctx_mpn_mul_range",
    "_nmod_poly_mul_mid_mpn_ctx": "gpu_shim__nmod_poly_mul_mid_mpn_ctx",
    "_fmpz_poly_mul_mid_mpn_ctx": "gpu_shim__fmpz_poly_mul_mid_mpn_ctx",
    "_nmod_poly_divrem_mpn_ctx": "gpu_shim__nmod_poly_divrem_mpn_ctx",
}
TESTS = ["t-mul.c", "t-nmod_poly_mul.c", "t-fmpz_poly_mul.c", "t-nmod_poly_divrem.c"]
# the test functions those files define (TEST_FUNCTION_START labels)
LABELS = ["mpn_ctx_mpn_mul", "_nmod_poly_mul_mid_mpn_ctx", "_fmpz_poly_mul_mid_mpn_ctx",
          "_nmod_poly_divrem_mpn_ctx"]

MAIN = """\
/* generated by oracle/build_ref_tests.py: the reference's fft_small tests
   for the products the GPU shim replaces (GMP's and mpn_extras'
   declarations first: the test files use them without including them) */
#include <gmp.h>
#include "mpn_extras.h"
%(includes)s

test_struct tests[] =
{
%(entries)s
};

TEST_MAIN(tests)
"""


def build(ref=build_ref.DEFAULT_REF, quiet=False):
    lib_ref = os.path.join(OUT, "libflint_ref.so")
    if not os.path.exists(lib_ref):
        build_ref.build(ref, quiet=quiet)
    lib_gpu = os.path.join(ROOT, "flint_b200", "libflint_b200.so")
    if not os.path.exists(lib_gpu):
        raise SystemExit("libflint_b200.so is not built (python -m flint_b200.build)")
    src = os.path.join(ref, "src")
    inc = os.path.join(OUT, "include")
    obj_dir = os.path.join(OUT, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    common = (["gcc"] + build_ref.CFLAGS
              + ["-I", inc, "-I", os.path.join(HERE, "gmp_min"), "-I", src,
                 "-I", os.path.join(ROOT, "include")])
    # the shim: FLINT-side binding, compiled against the reference's headers
    shim_o = os.path.join(obj_dir, "gpu_shim.o")
    subprocess.run(common + ["-c", os.path.join(ROOT, "flint_b200", "shim", "fft_small_gpu_shim.c"),
                             "-o", shim_o], check=True)
    # the reference's test files, entry points renamed to the shim
    main_c = os.path.join(obj_dir, "t-gpu-main.c")
    with open(main_c, "w") as f:
        f.write(MAIN % {"includes": "\n".join('#include "%s"' % t for t in TESTS),
                        "entries": ",\n".join("    TEST_FUNCTION(%s)" % l for l in LABELS)})
    main_o = os.path.join(obj_dir, "t-gpu-main.o")
    defs = ["-D%s=%s" % kv for kv in RENAMES.items()]
    subprocess.run(common + defs + ["-I", os.path.join(src, "fft_small", "test"), "-c", main_c,
                                    "-o", main_o], check=True)
    gmp = build_ref.find_gmp()
    rpath = "-Wl,-rpath,$ORIGIN:$ORIGIN/../../flint_b200"
    cmd = (["gcc", "-pthread", "-o", BINARY, main_o, shim_o, "-L", OUT, "-lflint_ref",
            "-L", os.path.dirname(lib_gpu), "-lflint_b200", gmp, "-lm", rpath])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-5000:])
        raise SystemExit("link of the test program failed")
    if not quiet:
        print("built", BINARY)
    return BINARY


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=build_ref.DEFAULT_REF)
    a = ap.parse_args()
    build(a.ref)
