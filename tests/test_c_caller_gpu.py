"""The reference's own fft_small tests, compiled as C against the GPU path.

oracle/build_ref_tests.py compiles the reference's test programs
(src/fft_small/test/t-mul.c, t-nmod_poly_mul.c, t-fmpz_poly_mul.c,
t-nmod_poly_divrem.c) with the
entry points under test renamed to the C shim flint_b200/shim/
fft_small_gpu_shim.c, which forwards to libflint_b200.so through its C ABI;
their yardsticks (GMP, _nmod_poly_mul_KS, _fmpz_poly_mul_KS, the generic
_nmod_poly_divrem) and harness
come from the compiled reference.  A passing run means a C caller with the
reference's signatures gets exactly the reference's answers from the GPU --
products, squarings, low windows, nmod windows, integer-polynomial
products whose coefficients FLINT allocates through the registered setter,
and divisions with remainder.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "t-gpu-fft_small")
needs_binary = pytest.mark.skipif(not os.path.exists(BINARY),
                                  reason="C caller not built (oracle/build_ref_tests.py)")


@needs_binary
@pytest.mark.gpu
@pytest.mark.parametrize("label", ["mpn_ctx_mpn_mul", "_nmod_poly_mul_mid_mpn_ctx",
                                   "_fmpz_poly_mul_mid_mpn_ctx", "_nmod_poly_divrem_mpn_ctx"])
def test_reference_tests_pass_through_the_c_shim(label):
    r = subprocess.run([BINARY, label], capture_output=True, text=True, timeout=1200)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-3000:]
    assert "PASS" in out, out[-3000:]


@needs_binary
def test_c_caller_fails_loudly_without_gpu():
    """Without a usable GPU the shim's first call raises a FLINT exception
    naming the library's error (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    r = subprocess.run([BINARY, "mpn_ctx_mpn_mul"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "gpu_fft_small" in r.stdout + r.stderr
