"""The module-wide constant tables survive every order of set-up.

Every kernel reads the radix-32 twiddles of all seven primes from one
constant-memory table per device.  Contexts and the allocation-free entry
point (gpu_mpn_mul_device_noalloc) both need it on the device; whichever comes
first writes it, the other must leave it alone.  A set-up that rewrote it with
only five primes filled in would silently break every six- or seven-prime
product of a context opened before it.  These tests run six-prime products on
a context (an mpn product under an explicit configuration and an integer
polynomial product) after the allocation-free call has done its set-up, in
both orders, and compare them with GMP and the Python restatement.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _six_prime_products(ctx):
    """A six-prime mpn product and a six-prime integer-polynomial product on
    ctx, each checked exactly; returns nothing, raises on a mismatch."""
    import torch
    s = torch.cuda.current_stream()
    an, bn = 30000, 20001
    a = O.rand_limbs(71, an)
    b = O.rand_limbs(72, bn)
    cfg = FB.resolve_config(0, an, bn)
    cfg = FB.resolve_config(0, an, bn, FB.MulConfig(cfg.route, 6, cfg.logM, cfg.logC))
    assert cfg.np == 6
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
    ctx.mpn_mul_device_config(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, cfg,
                              s.cuda_stream)
    s.synchronize()
    assert (dz.cpu().numpy().view(np.uint64) == O.gmp_mpn_mul(a, b)).all(), \
        "six-prime mpn product differs from GMP"

    fa = O.rand_fmpz_raw(81, 700, 300)
    fb = O.rand_fmpz_raw(82, 500, 200)
    (n1, aw), (n2, bw) = fa.shape, fb.shape
    zw = FB.fmpz_result_width(fa, fb)
    zn = n1 + n2 - 1
    fcfg = FB.resolve_config(1, n1, n2, aw=aw, bw=bw)
    fcfg = FB.resolve_config(1, n1, n2, FB.MulConfig(fcfg.route, 6, fcfg.logM, fcfg.logC),
                             aw=aw, bw=bw)
    assert fcfg.np == 6
    dfa = torch.from_numpy(fa.view(np.int64)).cuda()
    dfb = torch.from_numpy(fb.view(np.int64)).cuda()
    dfz = torch.full((zn, zw), -1, dtype=torch.int64, device="cuda")
    ctx.fmpz_poly_mul_device_config(dfz.data_ptr(), zw, 0, zn, dfa.data_ptr(), aw, n1,
                                    dfb.data_ptr(), bw, n2, fcfg, s.cuda_stream)
    s.synchronize()
    got = O.raw_to_ints(dfz.cpu().numpy().view(np.uint64))
    want = O.fmpz_poly_mul_python(O.raw_to_ints(fa), O.raw_to_ints(fb))
    assert got == want, "six-prime integer polynomial product differs"


def _noalloc_call():
    import torch
    lib = FB.lib()
    a = O.rand_limbs(91, 3000)
    b = O.rand_limbs(92, 2000)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.full((5000,), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    rc = lib.gpu_mpn_mul_device_noalloc(dz.data_ptr(), da.data_ptr(), 3000, db.data_ptr(), 2000,
                                        s.cuda_stream)
    s.synchronize()
    assert rc == FB.OK
    assert (dz.cpu().numpy().view(np.uint64) == O.gmp_mpn_mul(a, b)).all()


def test_context_first_then_noalloc_then_six_primes():
    """A context opened before the allocation-free call's set-up keeps
    correct six-prime tables afterwards."""
    pytest.importorskip("torch")
    with FB.MpnCtx() as ctx:
        _six_prime_products(ctx)          # tables as the context wrote them
        _noalloc_call()                   # set-up on this device (first call in this process)
        _six_prime_products(ctx)          # same context, after the set-up


_CHILD = r"""
import sys
sys.path.insert(0, %r)
from tests import test_shared_tables_gpu as T
import flint_b200 as FB
T._noalloc_call()                         # set-up before any context exists
with FB.MpnCtx() as ctx:
    T._six_prime_products(ctx)
print("ok")
"""


def test_noalloc_first_then_context_six_primes():
    """In a fresh process, the allocation-free call sets the device up before
    any context; a context opened afterwards still multiplies exactly with
    six primes."""
    pytest.importorskip("torch")
    r = subprocess.run([sys.executable, "-c", _CHILD % ROOT], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
