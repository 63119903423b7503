"""The allocation-free entry point, gpu_mpn_mul_device_noalloc.

It serves callers that may not call cudaMalloc -- a framework whose pool owns
all device memory, or a latency-critical pipeline that cannot afford the
implicit synchronisation of a fresh allocation.  Such a caller hands over only
device buffers for the operands and the product; the library works in scratch
that is part of its own device image.

The test calls it through the C ABI twice in a row (the second call must not
be disturbed by what the first left in the shared scratch) and compares each
product limb for limb with the context-based device entry point; further
cases (small, mid-size, unbalanced, squaring, the largest accepted size)
are checked against the oracle, and sizes above the documented limit, or
whose sum wraps around, are refused.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it passes alone in a fresh process as well.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu

MAX_LIMBS = (1 << 18) + 1   # an + bn limit of the allocation-free path


def test_noalloc_matches_context_entry_point_twice():
    torch = pytest.importorskip("torch")
    lib = FB.lib()
    stream = torch.cuda.current_stream()
    with FB.MpnCtx() as ctx:
        for k, (an, bn) in enumerate([(100000, 70001), (131072, 131073)]):
            a = O.rand_limbs(500 + k, an)
            b = O.rand_limbs(600 + k, bn)
            da = torch.from_numpy(a.view(np.int64)).cuda()
            db = torch.from_numpy(b.view(np.int64)).cuda()
            want = torch.empty(an + bn, dtype=torch.int64, device="cuda")
            got = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
            ctx.mpn_mul_device(want.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn,
                               stream.cuda_stream)
            rc = lib.gpu_mpn_mul_device_noalloc(got.data_ptr(), da.data_ptr(), an,
                                                db.data_ptr(), bn, stream.cuda_stream)
            stream.synchronize()
            assert rc == FB.OK
            assert torch.equal(got, want), "call %d differs from the context entry point" % k


@pytest.mark.parametrize("an,bn,square", [
    (60, 40, False), (1, 1, False), (3000, 2000, False), (2500, 2500, True),
    (40000, 7, False), (131072, 131073, False), (131072, 131072, True),
])
def test_noalloc_against_oracle(an, bn, square):
    """Small, mid-size, very unbalanced, largest and squaring products (each
    transform length runs its own launch shape) against the oracle, twice in a
    row on the shared scratch."""
    torch = pytest.importorskip("torch")
    lib = FB.lib()
    stream = torch.cuda.current_stream()
    for rep in range(2):
        a = O.rand_limbs(700 + an + rep, an)
        b = a if square else O.rand_limbs(800 + bn + rep, bn)
        want = O.port_mpn_mul(a, b)
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = da if square else torch.from_numpy(b.view(np.int64)).cuda()
        got = torch.full((an + bn,), -1, dtype=torch.int64, device="cuda")
        rc = lib.gpu_mpn_mul_device_noalloc(got.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn,
                                            stream.cuda_stream)
        stream.synchronize()
        assert rc == FB.OK
        assert (got.cpu().numpy().view(np.uint64) == want).all(), (an, bn, square, rep)


def test_noalloc_rejects_sizes_beyond_limit():
    torch = pytest.importorskip("torch")
    lib = FB.lib()
    an, bn = MAX_LIMBS - 100, 101
    da = torch.zeros(an, dtype=torch.int64, device="cuda")
    db = torch.zeros(bn, dtype=torch.int64, device="cuda")
    dz = torch.zeros(an + bn, dtype=torch.int64, device="cuda")
    rc = lib.gpu_mpn_mul_device_noalloc(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, None)
    assert rc == FB.ETOOBIG
    rc = lib.gpu_mpn_mul_device_noalloc(dz.data_ptr(), da.data_ptr(), 0, db.data_ptr(), bn, None)
    assert rc == FB.EINVAL
    # sizes whose sum wraps around 64 bits are refused, not read past
    rc = lib.gpu_mpn_mul_device_noalloc(dz.data_ptr(), da.data_ptr(), (1 << 64) - 1,
                                        db.data_ptr(), 2, None)
    assert rc == FB.ETOOBIG
