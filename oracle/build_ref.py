#!/usr/bin/env python3
"""Build recipe for the compiled reference (test infrastructure only).

Compiles the reference FLINT ``fft_small`` closure -- the small-prime NTT
multiplication path and the helper modules it links against -- straight from
the reference source tree into ``oracle/_ref/libflint_ref.so``.  The result is
the parity checker and the timed CPU baseline; the product never loads it.

The reference's own build systems cannot run here (no ``configure`` script,
no autoconf, ``CMakeLists.txt:31-33`` rejects non-Windows hosts, and there is
no ``gmp.h``), so this recipe

  1. writes ``flint.h`` from ``src/flint.h.in`` with the four version tokens
     (``flint.h.in:78-81``) filled in, a hand-set ``flint-config.h``, and
     ``gmpcompat.h`` / ``flint-mparam.h`` taken unchanged from the tree
     (``src/gmpcompat.h.in``, ``src/mpn_extras/x86_64/flint-mparam.h``) --
     all generated into ``oracle/_ref/include`` only;
  2. compiles with the project-written ``oracle/gmp_min/gmp.h`` (types and
     prototypes from the GMP manual) and links the system ``libgmp.so.10``;
  3. targets x86-64-v3 (AVX2 + FMA + BMI2), which ``machine_vectors.h:41``
     requires, so the library also runs on a GPU host with another CPU model.

Nothing is written outside ``oracle/_ref``.  Usage::

    python oracle/build_ref.py [--ref DIR] [-j 8]   (DIR defaults to $FLINT_REFERENCE or /root/reference)
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# Directories compiled whole: fft_small itself plus the modules its link
# closure reaches (thread pool, exceptions/memory, word-size number theory,
# nmod and fmpz layers for the nmod_poly and fmpz_poly entry points, and the
# KS / Schoenhage-Strassen routes of _fmpz_poly_mul).
DIRS = [
    "fft_small", "ulong_extras", "long_extras", "nmod", "nmod_vec", "nmod_poly",
    "fmpz", "fmpz_vec", "fmpz_poly", "mpn_extras", "thread_pool",
    "thread_support", "generic_files", "fft",
    # generic rings: _nmod_poly_inv_series (behind _nmod_poly_divrem_mpn_ctx,
    # src/fft_small/nmod_poly_mul.c:1248-1277) hands series longer than 10
    # terms to _gr_poly_inv_series over the nmod ring (src/nmod_poly/inv_series.c:63-77)
    "gr", "gr_generic", "gr_poly", "gr_vec",
]

# Single files outside the whole directories: the non-reentrant fmpz memory
# link (the variant the reference's default configuration selects).
TOP_FILES = ["fmpz/link/fmpz_single.c"]

CFLAGS = ["-O2", "-march=x86-64-v3", "-fPIC", "-pthread", "-w",
          "-std=gnu11", "-DFLINT_NOSTDIO_TEST=0"]

FLINT_CONFIG = """\
/* hand-set configuration for the oracle build of the reference */
#define FLINT_BITS 64
#define FLINT_HAVE_FFT_SMALL 1
#define FLINT_USES_PTHREAD 1
#define FLINT_USES_TLS 1
#define FLINT_KNOW_STRONG_ORDER 1
#define FLINT_HAVE_NATIVE_mpn_add_n_sub_n 0
#define FLINT_HAVE_NATIVE_mpn_add_nc 0
#define FLINT_HAVE_NATIVE_mpn_addlsh1_n 0
#define FLINT_HAVE_NATIVE_mpn_addlsh1_n_ip1 0
#define FLINT_HAVE_NATIVE_mpn_addmul_2 0
#define FLINT_HAVE_NATIVE_mpn_modexact_1_odd 0
#define FLINT_HAVE_NATIVE_mpn_mulmid_n 0
#define FLINT_HAVE_NATIVE_mpn_rsh1add_n 0
#define FLINT_HAVE_NATIVE_mpn_rsh1sub_n 0
#define FLINT_HAVE_NATIVE_mpn_sub_nc 0
#define FLINT_HAVE_ASSEMBLY_x86_64_adx 0
#define FLINT_HAVE_ASSEMBLY_armv8 0
#define FLINT_WANT_ASSEMBLY 0
#define FLINT_WANT_ASSERT 0
#define FLINT_USES_GC 0
#define FLINT_USES_BLAS 0
#define FLINT_USES_CPUSET 0
#define FLINT_REENTRANT 0
#define FLINT_UNROLL_LOOPS 0
#define FLINT_WANT_GMP_INTERNALS 0
#define FLINT_WANT_PRETTY_TESTS 0
#define HAVE_ALIGNED_ALLOC 1
/* compiler-pragma helpers the reference's generated config.h provides;
   empty here, as in CMake/cmake_config.h.in */
#define DIAGNOSTIC_PUSH
#define DIAGNOSTIC_POP
#define DIAGNOSTIC_IGNORE_INCOMPATIBLE_FUNCTION_POINTER_TYPES
#define DIAGNOSTIC_IGNORE_DISCARDED_QUALIFIERS
#define DIAGNOSTIC_IGNORE_FORMAT
#define DIAGNOSTIC_IGNORE_DANGLING_POINTER
#define DIAGNOSTIC_IGNORE_CAST_FUNCTION_TYPE
#define DIAGNOSTIC_IGNORE_OVERLENGTH_STRINGS
#define DIAGNOSTIC_IGNORE_UNUSED_VARIABLE
#define DIAGNOSTIC_IGNORE_MAYBE_UNINITIALIZED
#define PUSH_OPTIONS
#define POP_OPTIONS
#define OPTIMIZE_O2
#define OPTIMIZE_OSIZE
#define OPTIMIZE_UNROLL_LOOPS
"""

# Files that need MPFR beyond mpfr_free_cache (conversions to mpfr_t and the
# mpfr-based ceil-log); nothing on the multiplication path calls them.
SKIP = {"ulong_extras/clog.c"}


def read_version(ref):
    with open(os.path.join(ref, "VERSION")) as f:
        v = f.read().strip()
    m = re.match(r"(\d+)\.(\d+)\.(\d+)", v)
    if m:
        return v, m.group(1), m.group(2), m.group(3)
    m = re.match(r"(\d+)\.(\d+)", v)
    return v, m.group(1), m.group(2), "0"


def gen_headers(ref, inc):
    src = os.path.join(ref, "src")
    os.makedirs(inc, exist_ok=True)
    full, major, minor, patch = read_version(ref)
    with open(os.path.join(src, "flint.h.in")) as f:
        text = f.read()
    text = (text.replace("@FLINT_MAJOR@", major)
                .replace("@FLINT_MINOR@", minor)
                .replace("@FLINT_PATCH@", patch)
                .replace("@FLINT_VERSION_FULL@", full))
    with open(os.path.join(inc, "flint.h"), "w") as f:
        f.write(text)
    with open(os.path.join(inc, "flint-config.h"), "w") as f:
        f.write(FLINT_CONFIG)
    shutil.copyfile(os.path.join(src, "gmpcompat.h.in"),
                    os.path.join(inc, "gmpcompat.h"))
    shutil.copyfile(os.path.join(src, "mpn_extras", "x86_64", "flint-mparam.h"),
                    os.path.join(inc, "flint-mparam.h"))


def sources(ref):
    src = os.path.join(ref, "src")
    out = []
    for d in DIRS:
        dd = os.path.join(src, d)
        for name in sorted(os.listdir(dd)):
            if name.endswith(".c") and d + "/" + name not in SKIP:
                out.append(os.path.join(dd, name))
    for name in TOP_FILES:
        out.append(os.path.join(src, name))
    return out


def compile_one(args):
    ref, inc, obj_dir, path = args
    src = os.path.join(ref, "src")
    rel = os.path.relpath(path, src).replace(os.sep, "__")
    obj = os.path.join(obj_dir, rel[:-2] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path):
        return obj, None
    cmd = (["gcc"] + CFLAGS + ["-I", inc, "-I", os.path.join(HERE, "gmp_min"),
                               "-I", src, "-c", path, "-o", obj])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return None, (path, r.stderr[-3000:])
    return obj, None


def find_gmp():
    for cand in ("/usr/lib/x86_64-linux-gnu/libgmp.so.10", "/usr/lib64/libgmp.so.10",
                 "/usr/lib/libgmp.so.10"):
        if os.path.exists(cand):
            return cand
    raise SystemExit("libgmp.so.10 not found")


def find_lib(name):
    for d in ("/usr/lib/x86_64-linux-gnu", "/lib/x86_64-linux-gnu", "/usr/lib64"):
        if os.path.exists(os.path.join(d, name)):
            return os.path.join(d, name)
    raise SystemExit(name + " not found")


def _nm(path, dynamic=False):
    args = ["nm", "-D" if dynamic else "-g"] + ([] if not dynamic else ["--defined-only"])
    r = subprocess.run(args + [path], capture_output=True, text=True, check=True)
    defined, undefined = set(), set()
    for line in r.stdout.splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0] in ("U", "w", "v"):
            if parts[0] == "U":
                undefined.add(parts[1].split("@")[0])
        elif len(parts) >= 3:
            defined.add(parts[2].split("@")[0])
    return defined, undefined


def link_closure(objs, shared_libs, obj_dir):
    """Close the link with aborting stubs for symbols outside the closure.

    The whole directories compiled above reference modules outside the
    multiplication path (factoring, matrices, ball arithmetic, generic
    rings, printing of those types).  The library must load with every
    symbol bound, so each such function gets a generated stub that prints
    its name and aborts; the oracle never reaches them, and if it ever did
    the process would stop loudly instead of computing something else."""
    system = {"_GLOBAL_OFFSET_TABLE_", "__tls_get_addr"}  # provided at link/load
    for lib in shared_libs:
        system |= _nm(lib, dynamic=True)[0]
    defined, undefined = set(system), set()
    for o in objs:
        d, u = _nm(o)
        defined |= d
        undefined |= u
    missing = sorted(undefined - defined)
    stub_c = os.path.join(obj_dir, "closure_stubs.c")
    with open(stub_c, "w") as f:
        f.write("#include <stdio.h>\n#include <stdlib.h>\n")
        f.write("static void outside(const char *s)\n{\n"
                "    fprintf(stderr, \"reference oracle: %s is outside the "
                "compiled closure\\n\", s);\n    abort();\n}\n")
        for name in missing:
            f.write("void %s(void) { outside(\"%s\"); }\n" % (name, name))
    stub_o = stub_c[:-2] + ".o"
    subprocess.run(["gcc", "-O1", "-fPIC", "-c", stub_c, "-o", stub_o], check=True)
    return objs + [stub_o]


REQUIRED = ["mpn_ctx_init", "mpn_ctx_clear", "mpn_ctx_mpn_mul",
            "_mpn_ctx_mpn_mul_range", "_nmod_poly_mul_mid_mpn_ctx",
            "_fmpz_poly_mul_mid_mpn_ctx", "get_default_mpn_ctx",
            "mpn_mul_default_mpn_ctx", "_fmpz_poly_mul", "flint_set_num_threads",
            "flint_mpn_mul", "_nmod_poly_mul_KS", "_fmpz_poly_mul_KS",
            "sd_fft_trunc", "sd_ifft_trunc", "sd_fft_ctx_init_prime",
            "_nmod_poly_divrem_mpn_ctx", "_nmod_poly_divrem", "_gr_poly_inv_series"]


DEFAULT_REF = os.environ.get("FLINT_REFERENCE", "/root/reference")


def build(ref=DEFAULT_REF, jobs=None, quiet=False):
    lib = os.path.join(OUT, "libflint_ref.so")
    if not os.path.isdir(os.path.join(ref, "src", "fft_small")):
        raise SystemExit("reference tree not found at %s" % ref)
    inc = os.path.join(OUT, "include")
    obj_dir = os.path.join(OUT, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    gen_headers(ref, inc)
    srcs = sources(ref)
    jobs = jobs or os.cpu_count() or 4
    objs, errs = [], []
    with ThreadPoolExecutor(jobs) as ex:
        for obj, err in ex.map(compile_one, [(ref, inc, obj_dir, s) for s in srcs]):
            if err:
                errs.append(err)
            else:
                objs.append(obj)
    if errs:
        for path, msg in errs[:10]:
            sys.stderr.write("== %s\n%s\n" % (path, msg))
        raise SystemExit("%d reference files failed to compile" % len(errs))
    gmp = find_gmp()
    mpfr = gmp.replace("libgmp.so.10", "libmpfr.so.6")
    objs = link_closure(objs, [gmp, mpfr, find_lib("libc.so.6"), find_lib("libm.so.6")],
                        obj_dir)
    cmd = (["gcc", "-shared", "-pthread", "-Wl,--no-undefined", "-o", lib]
           + sorted(objs) + [mpfr, gmp, "-lm"])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-5000:])
        raise SystemExit("link failed")
    exported = _nm(lib, dynamic=True)[0]
    missing = [s for s in REQUIRED if s not in exported]
    if missing:
        raise SystemExit("reference closure lacks " + ", ".join(missing))
    if not quiet:
        print("built", lib, "from", len(objs), "reference files")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    build(a.ref, a.j)
