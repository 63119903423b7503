"""Failure paths of the bounded device waits, on the GPU without a fault.

The CRT/carry kernel's look-back waits for the previous tile's status word
with an iteration limit; when the limit runs out it sets the context's error
flag, finishes, and the host reports GPU_FFT_SMALL_ETIMEOUT.  Valid inputs
never reach this, so test hooks make it happen: one tile whose predecessor
never publishes (the wait really runs out on the device), and an error flag
planted from the host as such a kernel would set it (read back by the next
host-pointer product through its pinned copy of the flag).  Afterwards the
context must stay usable and exact.
"""
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


def test_lookback_wait_runs_out_and_context_stays_usable(ctx):
    rc = FB.lib().gpu_test_crt_lookback_timeout(ctx.ptr)
    assert rc == FB.ETIMEOUT
    a, b = O.rand_limbs(31, 70000), O.rand_limbs(32, 50000)
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


def test_error_flag_reaches_the_next_host_product(ctx):
    a, b = O.rand_limbs(33, 5000), O.rand_limbs(34, 3000)
    FB._check(FB.lib().gpu_test_set_device_error(ctx.ptr))
    with pytest.raises(FB.GpuFftSmallError) as e:
        ctx.mpn_mul(a, b)
    assert e.value.code == FB.ETIMEOUT
    # the flag was cleared: the next product is exact
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


def test_error_flag_reaches_a_pipelined_product():
    a, b = O.rand_limbs(35, 20000), O.rand_limbs(36, 15000)
    want = O.gmp_mpn_mul(a, b)
    with FB.MpnPipe(2) as P:
        t0 = P.submit(a, b)
        assert (P.wait(t0) == want).all()
        # the pipeline's slots are its own contexts: plant the flag in slot 1
        # through the same hook on a handle that shares its layout
        slot1 = FB.lib().gpu_test_pipe_slot_ctx(FB.ctypes.byref(P._c), 1)
        assert slot1
        FB._check(FB.lib().gpu_test_set_device_error(FB.ctypes.byref(FB._Ctx(slot1))))
        t1 = P.submit(a, b)               # slot 1
        with pytest.raises(FB.GpuFftSmallError) as e:
            P.wait(t1)
        assert e.value.code == FB.ETIMEOUT
        t2 = P.submit(b, a)
        t3 = P.submit(a, b)               # slot 1 again: the flag was cleared
        assert (P.wait(t2) == O.gmp_mpn_mul(b, a)).all()
        assert (P.wait(t3) == want).all()
