"""GPU parity of batches of uneven products (gpu_mpn_batch_*).

A batch runs many products of different sizes in a few launches per
(primes, transform length) class.  Every product of every batch is compared
limb for limb with GMP's mpn_mul (small batches) or with the single-product
device entry point (the full uneven workload: 2^10..2^18 limbs, ratios up
to 16).  Schedules (graph capture or direct launches, class promotion,
stream counts) must not change a single limb, and a replayed graph must pick
up new operand values written in place.
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O
from flint_b200.workload import batch_operands, uneven_batch

pytestmark = pytest.mark.gpu

EDGE_SIZES = [(1, 1), (2, 1), (1, 7), (31, 1), (32, 32), (33, 31), (1000, 1), (1024, 1024),
              (4095, 4097), (8192, 8192), (16383, 2), (16384, 16385), (65537, 65535),
              (100000, 3), (131072, 131072)]


def _device_batch(torch, sizes, seed):
    host, spans = batch_operands(seed, sizes)
    d_in = torch.from_numpy(host.view(np.int64)).cuda()
    zlen = sum(an + bn for an, bn in sizes)
    d_out = torch.full((zlen,), -1, dtype=torch.int64, device="cuda")
    reqs, zoff = [], []
    base_in, base_out, esz = d_in.data_ptr(), d_out.data_ptr(), 8
    off = 0
    for (ao, an, bo, bn) in spans:
        reqs.append((base_out + off * esz, base_in + ao * esz, an, base_in + bo * esz, bn))
        zoff.append(off)
        off += an + bn
    return host, spans, d_in, d_out, reqs, zoff


def _check_vs_gmp(host, spans, out, zoff):
    for (ao, an, bo, bn), zo in zip(spans, zoff):
        want = O.gmp_mpn_mul(host[ao:ao + an], host[bo:bo + bn])
        assert (out[zo:zo + an + bn] == want).all(), "product %dx%d differs" % (an, bn)


@pytest.mark.parametrize("opts", [
    dict(promote_small=0, max_streams=4, use_graph=True),
    dict(promote_small=0, max_streams=1, use_graph=False),
    dict(promote_small=6, max_streams=2, use_graph=True),
])
def test_small_batch_vs_gmp(ctx, opts):
    torch = pytest.importorskip("torch")
    sizes = uneven_batch(11, 120, log_lo=0.0, log_hi=13.0) + EDGE_SIZES
    host, spans, d_in, d_out, reqs, zoff = _device_batch(torch, sizes, 3)
    stream = torch.cuda.current_stream()
    with FB.MpnBatch(ctx, reqs, **opts) as B:
        assert B.classes >= 1
        B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
        assert B.launches >= 3 * B.classes
    out = d_out.cpu().numpy().view(np.uint64)
    _check_vs_gmp(host, spans, out, zoff)


def test_graph_replay_sees_new_operands(ctx):
    torch = pytest.importorskip("torch")
    sizes = uneven_batch(5, 60, log_lo=4.0, log_hi=15.0)
    host, spans, d_in, d_out, reqs, zoff = _device_batch(torch, sizes, 8)
    stream = torch.cuda.current_stream()
    with FB.MpnBatch(ctx, reqs, use_graph=True) as B:
        B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
        _check_vs_gmp(host, spans, d_out.cpu().numpy().view(np.uint64), zoff)
        # new operand values, same pointers: the replayed graph must use them
        host2, _ = batch_operands(9, sizes)
        host2[0] = np.uint64(0xFFFFFFFFFFFFFFFF)
        d_in.copy_(torch.from_numpy(host2.view(np.int64)))
        d_out.fill_(-1)
        for _ in range(2):
            B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
        _check_vs_gmp(host2, spans, d_out.cpu().numpy().view(np.uint64), zoff)


def test_all_ones_batch(ctx):
    """Longest carry chains inside every product of a batch."""
    torch = pytest.importorskip("torch")
    sizes = [(n, m) for n in (1, 5, 300, 5000, 40000) for m in (1, 7, 299)]
    host = np.full(sum(a + b for a, b in sizes), (1 << 64) - 1, dtype=np.uint64)
    d_in = torch.from_numpy(host.view(np.int64)).cuda()
    d_out = torch.empty(host.size, dtype=torch.int64, device="cuda")
    reqs, spans, zoff, off = [], [], [], 0
    for an, bn in sizes:
        reqs.append((d_out.data_ptr() + 8 * off, d_in.data_ptr() + 8 * off, an,
                     d_in.data_ptr() + 8 * (off + an), bn))
        spans.append((off, an, off + an, bn))
        zoff.append(off)
        off += an + bn
    stream = torch.cuda.current_stream()
    with FB.MpnBatch(ctx, reqs) as B:
        B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
    _check_vs_gmp(host, spans, d_out.cpu().numpy().view(np.uint64), zoff)


def test_uneven_workload_matches_single_products(ctx):
    """The full-range uneven workload (512 products, 2^10..2^18 limbs) against
    the single-product device entry point, and a GMP check of a subsample."""
    torch = pytest.importorskip("torch")
    sizes = uneven_batch(2024, 512)
    host, spans, d_in, d_out, reqs, zoff = _device_batch(torch, sizes, 21)
    stream = torch.cuda.current_stream()
    d_want = torch.empty_like(d_out)
    for (z, a, an, b, bn), zo in zip(reqs, zoff):
        ctx.mpn_mul_device(d_want.data_ptr() + 8 * zo, a, an, b, bn, stream.cuda_stream)
    with FB.MpnBatch(ctx, reqs, promote_small=4) as B:
        B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
    assert torch.equal(d_out, d_want)
    out = d_out.cpu().numpy().view(np.uint64)
    pick = list(range(0, len(sizes), 37))
    _check_vs_gmp(host, [spans[k] for k in pick], out, [zoff[k] for k in pick])


def test_batch_rejects_bad_requests(ctx):
    torch = pytest.importorskip("torch")
    d = torch.zeros(16, dtype=torch.int64, device="cuda")
    p = d.data_ptr()
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.MpnBatch(ctx, [(p, p + 64, 4, p + 96, 0)])
    assert e.value.code == FB.EINVAL
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.MpnBatch(ctx, [])
    assert e.value.code == FB.EINVAL


def test_configured_batch_with_basecase_classes(ctx):
    """Per-request configurations: basecase, shorter rows, a longer transform
    and an extra prime, mixed in one batch; every product exact."""
    torch = pytest.importorskip("torch")
    from flint_b200 import tuner
    sizes = uneven_batch(77, 90, log_lo=0.0, log_hi=14.0) + [(5000, 1024), (1024, 1024), (1, 1),
                                                             (70000, 3), (3, 70000)]
    host, spans, d_in, d_out, reqs, zoff = _device_batch(torch, sizes, 5)
    configs = []
    for k, (an, bn) in enumerate(sizes):
        cs = tuner.candidates((0, an, bn), flags=False)   # what a planned batch accepts
        configs.append(cs[k % len(cs)])
    assert any(c.route == FB.ROUTE_BASECASE for c in configs)
    stream = torch.cuda.current_stream()
    with FB.MpnBatch(ctx, reqs, configs=configs, promote_small=3) as B:
        B.run(stream.cuda_stream)
        B.check(stream.cuda_stream)
        out = d_out.cpu().numpy().view(np.uint64)
        _check_vs_gmp(host, spans, out, zoff)
        d_out.fill_(-1)
        B.run(stream.cuda_stream)   # graph replay
        B.check(stream.cuda_stream)
    _check_vs_gmp(host, spans, d_out.cpu().numpy().view(np.uint64), zoff)


def test_time_batched_is_positive(ctx):
    from flint_b200 import tuner
    for an, bn in [(100, 100), (3000, 700), (1 << 16, 1 << 12)]:
        for c in tuner.candidates((0, an, bn), flags=False)[:4]:   # what a planned batch takes
            ms = ctx.time_batched(an, bn, c, copies=tuner.batch_copies(an, bn), reps=2)
            assert 0.0 < ms < 100.0
