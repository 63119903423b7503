"""The request-stream executor under a schedule: every product identical to
the product under the fixed rule, and a subsample identical to the
reference's own products."""
import numpy as np
import pytest

import oracle as O
from flint_b200 import tuner
from flint_b200.stream import run_stream
from flint_b200.workload import request_stream

pytestmark = pytest.mark.gpu


def test_stream_schedules_agree_and_match_reference(ctx):
    torch = pytest.importorskip("torch")
    reqs = request_stream(31, 40, mpn_log=(0.0, 17.0), fmpz_len_log=(4.0, 10.0),
                          fmpz_bits=(64, 700))
    # a deliberately varied schedule: cycle through each request's candidates
    cfgs = [tuner.candidates(r)[k % len(tuner.candidates(r))] for k, r in enumerate(reqs)]
    default = [tuner.default_config(r) for r in reqs]
    stream = torch.cuda.current_stream()
    keep = set(range(0, 40, 3))
    res = run_stream(ctx, torch, reqs, cfgs, 5, stream, torch.device("cuda"), chunk_limbs=1 << 18,
                     keep=keep)
    ref = run_stream(ctx, torch, reqs, default, 5, stream, torch.device("cuda"), chunk_limbs=1 << 18)
    # every product's digest equals the fixed rule's (same operands, other configurations)
    assert (res["digests"] == ref["digests"]).all()
    assert res["mpn_requests"] + res["fmpz_requests"] == len(reqs)
    for k in keep:
        r = reqs[k]
        if r[0] == 0:
            ops, z = res["kept"][k]
            an, bn = r[1], r[2]
            assert (z == O.gmp_mpn_mul(ops[:an], ops[an:an + bn])).all()
        else:
            a, b, z = res["kept"][k]
            _, an, bn, aw, bw = r
            want = O.fmpz_poly_mul_python(O.raw_to_ints(a.reshape(an, aw)),
                                          O.raw_to_ints(b.reshape(bn, bw)))
            assert O.raw_to_ints(z.reshape(an + bn - 1, aw + bw + 1)) == want


def test_fmpz_list_entry_point_matches_single_calls(ctx):
    """gpu_fmpz_poly_mul_mid_device_list queues several products (different
    widths, a squaring, a window) with one call; each equals the single-call
    device entry point.  An invalid request fails the call, naming its index,
    before anything is queued."""
    torch = pytest.importorskip("torch")
    import flint_b200 as FB
    shapes = [(300, 200, 2, 3, 0, None), (1000, 17, 1, 1, 0, None), (64, 64, 5, 5, 0, "sq"),
              (777, 500, 2, 2, 100, 900)]
    stream = torch.cuda.current_stream()
    lst, outs, want = [], [], []
    keepalive = []
    for k, (an, bn, aw, bw, zl, zh) in enumerate(shapes):
        a = torch.from_numpy(O.rand_fmpz_raw(900 + k, an, 64 * aw - 1).view(np.int64)).cuda()
        b = a if zh == "sq" else torch.from_numpy(O.rand_fmpz_raw(950 + k, bn, 64 * bw - 1).view(np.int64)).cuda()
        zh = an + bn - 1 if zh in (None, "sq") else zh
        zw = aw + bw + 1
        z = torch.full(((zh - zl) * zw,), -1, dtype=torch.int64, device="cuda")
        w = torch.full_like(z, -2)
        ctx.fmpz_poly_mul_device(w.data_ptr(), zw, zl, zh, a.data_ptr(), aw, an, b.data_ptr(), bw, bn,
                                 stream.cuda_stream)
        lst.append(FB.FmpzMulReq(z.data_ptr(), zw, zl, zh, a.data_ptr(), aw, an, b.data_ptr(), bw, bn))
        outs.append(z)
        want.append(w)
        keepalive += [a, b]
    ctx.fmpz_poly_mul_device_list(lst, None, stream.cuda_stream)
    stream.synchronize()
    for z, w in zip(outs, want):
        assert torch.equal(z, w)
    bad = list(lst)
    bad[2] = FB.FmpzMulReq(lst[2].z, lst[2].zw, 0, 10 ** 9, lst[2].a, lst[2].aw, lst[2].an, lst[2].b,
                           lst[2].bw, lst[2].bn)
    with pytest.raises(FB.GpuFftSmallError, match="request 2"):
        ctx.fmpz_poly_mul_device_list(bad, None, stream.cuda_stream)
