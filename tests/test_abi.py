"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol include/gpu_fft_small.h declares, plans like the host code says, and
fails loudly (no CPU fallback) when no GPU is present."""
import os
import re
import subprocess

import pytest

import flint_b200 as FB

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpu_fft_small.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "sizeof", "defined", "handler", "void", "int", "return", "__attribute__",
            "visibility"}
    return sorted({n for n in names if n not in skip and not n.isupper()})


def test_header_declares_entry_points():
    fns = declared_functions()
    for want in ("gpu_mpn_ctx_init", "gpu_mpn_ctx_clear", "gpu_mpn_ctx_mpn_mul",
                 "_gpu_mpn_ctx_mpn_mul_range", "_gpu_nmod_poly_mul_mid_mpn_ctx",
                 "gpu_mpn_mul_default_mpn_ctx", "gpu_mpn_mul_device"):
        assert want in fns


def test_library_exports_every_declared_symbol():
    lib = FB.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", FB.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)
        assert name in FB.SIGNATURES, name


def test_library_has_no_oracle_or_cpu_path():
    out = subprocess.run(["nm", "-D", FB.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out
    deps = subprocess.run(["ldd", FB.LIB_PATH], capture_output=True, text=True).stdout
    assert "liboracle" not in deps and "flint_ref" not in deps and "libgmp" not in deps


def test_plan_matches_design():
    assert FB.mpn_mul_plan(1 << 24, 1 << 24) == (5, 25)
    assert FB.mpn_mul_plan(1 << 24, 1 << 20) == (5, 25)
    assert FB.mpn_mul_plan(1 << 16, 1 << 16) == (5, 17)
    assert FB.mpn_mul_plan(1, 1) == (5, 5)   # smallest transform: 32 points
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.mpn_mul_plan(1 << 25, 1 << 25)
    assert e.value.code == FB.ETOOBIG
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.mpn_mul_plan(0, 5)
    assert e.value.code == FB.EINVAL


def test_prime_set():
    prod = 1
    for i in range(7):
        p = FB.prime(i)
        assert p < (1 << 31) and (p - 1) % (1 << 25) == 0
        assert all(pow(a, p - 1, p) == 1 for a in (2, 3, 5, 7, 11, 13))
        if i < 5:
            prod *= p
    # five primes hold a 2^24 x 2^24 coefficient with the CRT rounding margin
    assert prod > 2 * (1 << 24) * ((1 << 64) - 1) ** 2
    assert FB.prime(7) == 0


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_fails_loudly_without_gpu():
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.MpnCtx()
    assert e.value.code == FB.ECUDA
    # a pipeline of host-pointer products builds its slots from contexts
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.MpnPipe(2)
    assert e.value.code == FB.ECUDA


def test_pipe_depth_is_checked():
    for depth in (0, 5):
        with pytest.raises(FB.GpuFftSmallError) as e:
            FB.MpnPipe(depth)
        assert e.value.code == FB.EINVAL


def test_missing_library_is_an_error(monkeypatch):
    monkeypatch.setattr(FB, "_lib", None)
    monkeypatch.setattr(FB, "LIB_PATH", "/nonexistent/libflint_b200.so")
    with pytest.raises(ImportError):
        FB.lib()
