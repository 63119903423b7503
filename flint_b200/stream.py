"""Execution of a stream of multiplication requests under a schedule.

A request is (kind, an, bn, aw, bw) as in flint_b200.tuner: kind 0 an
an x bn-limb mpn product, kind 1 an integer-polynomial product of an x bn
coefficients of aw and bw limbs.  ``run_stream`` executes every request with
the configuration a chooser gives it:

* mpn requests go in chunks (at most ``chunk_limbs`` operand limbs each) into
  planned batches (gpu_mpn_batch_init_config), so products that share a
  configuration share launches; requests whose configuration carries flags
  (a 3 2^k-point transform, a split product, a forced row-pass width) or
  takes the basecase route beyond a planned batch's limit (a short operand
  above 1024 limbs) go in chunks through the per-instance list call
  (gpu_mpn_mul_device_list) instead;
* integer-polynomial requests go in chunks through one list call each
  (gpu_fmpz_poly_mul_mid_device_list): every product of a chunk is queued by
  native code on one stream, with the scratch sized before the timing.

Operands come from one pool of pseudo-random limbs generated on the device
from the seed (torch's CUDA generator): request k reads the pool at an offset
hashed from k, so its operands do not depend on how a schedule groups the
requests.  They are gathered outside the timed region; the device time of the products is measured with
CUDA events on the launching stream.  Every product also gets a 64-bit
digest (a weighted sum of its limbs with fixed pseudo-random weights,
computed on the device), so two runs under different schedules can be
compared product by product without copying them to the host; ``keep`` lets
a caller copy selected products (with their operands) to the host.
"""
import numpy as np

from . import ROUTE_BASECASE, FmpzMulReq, MpnBatch, MulReq
from .tuner import BASECASE_BATCH_MAX


def _per_instance(r, cfg):
    """True for an mpn request whose configuration a planned batch does not
    take (flags, or the basecase route with a short operand above the
    batch's limit)."""
    return bool(cfg.flags) or (cfg.route == ROUTE_BASECASE and min(r[1], r[2]) > BASECASE_BATCH_MAX)


def _weights(torch, n, dev):
    """Fixed pseudo-random int64 weights for product digests."""
    g = torch.Generator(device=dev)
    g.manual_seed(0x5EED)
    return torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64, device=dev, generator=g)


def _digests(torch, out, starts, lens, weights):
    """Per-product digests sum_i out[s + i] * weights[i] (mod 2^64) for the
    products at out[starts[k] : starts[k] + lens[k]] (consecutive, in
    order).  A scan, not atomics: each limb's position inside its product
    comes from a running count of product starts, and a product's digest is
    the difference of the wrapping prefix sums at its two ends."""
    dev = out.device
    n = int(starts[-1] + lens[-1])
    st = torch.tensor(starts, dtype=torch.int64, device=dev)
    ends = st + torch.tensor(lens, dtype=torch.int64, device=dev)
    marks = torch.zeros(n, dtype=torch.int32, device=dev)
    marks[st[1:]] = 1
    owner = torch.cumsum(marks, 0)
    local = torch.arange(n, device=dev) - st[owner]
    cs = torch.cumsum(out[:n] * weights[local], 0)
    lo = torch.where(st > 0, cs[(st - 1).clamp(min=0)], torch.zeros_like(st))
    return cs[ends - 1] - lo


POOL_LIMBS = 1 << 27


def _pool_offset(k, n):
    """Pool offset of request k's n operand limbs (a fixed hash of k)."""
    return ((k + 1) * 0x9E3779B97F4A7C15 >> 17) % (POOL_LIMBS - n)


def _gather(torch, pool, starts, lens):
    """The pool slices [starts[k], starts[k] + lens[k]) concatenated."""
    dev = pool.device
    st = torch.tensor(starts, dtype=torch.int64, device=dev)
    ln = torch.tensor(lens, dtype=torch.int64, device=dev)
    base = torch.repeat_interleave(torch.cumsum(ln, 0) - ln, ln)
    idx = torch.arange(int(sum(lens)), device=dev) - base + torch.repeat_interleave(st, ln)
    return pool[idx]


def _chunks(idx, size_of, limit):
    out, cur, size = [], [], 0
    for k in idx:
        n = size_of(k)
        if cur and size + n > limit:
            out.append(cur)
            cur, size = [], 0
        cur.append(k)
        size += n
    if cur:
        out.append(cur)
    return out


def run_stream(ctx, torch, reqs, configs, seed, stream, dev, chunk_limbs=1 << 27, keep=None):
    """Execute reqs under configs (one per request).  Returns a dict of device
    milliseconds (mpn, fmpz, total), limbs processed, a per-request digest
    array ('digests', int64, in request order) and, for the request indices
    in `keep`, host copies of operands and products in 'kept'."""
    gen = torch.Generator(device=dev)
    s = stream.cuda_stream
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    res = {"mpn_ms": 0.0, "fmpz_ms": 0.0, "mpn_limbs": 0, "fmpz_coeff_limbs": 0,
           "mpn_requests": 0, "fmpz_requests": 0, "kept": {}}
    digests = np.zeros(len(reqs), dtype=np.int64)
    mpn_list = [k for k, r in enumerate(reqs) if r[0] == 0 and _per_instance(r, configs[k])]
    mpn = [k for k, r in enumerate(reqs) if r[0] == 0 and not _per_instance(r, configs[k])]
    fz = [k for k, r in enumerate(reqs) if r[0] == 1]
    wmax = 1
    for r in reqs:
        wmax = max(wmax, r[1] + r[2] if r[0] == 0 else (r[1] + r[2] - 1) * (r[3] + r[4] + 1))
    weights = _weights(torch, wmax, dev)
    gen.manual_seed(seed)
    pool = torch.randint(-(1 << 63), (1 << 63) - 1, (POOL_LIMBS,), dtype=torch.int64, device=dev,
                         generator=gen)

    def operands(idx, size_of):
        return _gather(torch, pool, [_pool_offset(k, size_of(k)) for k in idx], [size_of(k) for k in idx])

    for ci, idx in enumerate(_chunks(mpn, lambda k: reqs[k][1] + reqs[k][2], chunk_limbs)):
        tot = sum(reqs[k][1] + reqs[k][2] for k in idx)
        d_in = operands(idx, lambda k: reqs[k][1] + reqs[k][2])
        d_out = torch.empty(tot, dtype=torch.int64, device=dev)
        rq, off, offs = [], 0, []
        for k in idx:
            an, bn = reqs[k][1], reqs[k][2]
            p = d_in.data_ptr() + 8 * off
            rq.append((d_out.data_ptr() + 8 * off, p, an, p + 8 * an, bn))
            offs.append(off)
            off += an + bn
        with MpnBatch(ctx, rq, configs=[configs[k] for k in idx]) as B:
            B.run(s)                      # plan + graph capture outside the timing
            stream.synchronize()
            ev0.record(stream)
            B.run(s)
            ev1.record(stream)
            B.check(s)
            res["mpn_ms"] += ev0.elapsed_time(ev1)
        dg = _digests(torch, d_out, offs, [reqs[k][1] + reqs[k][2] for k in idx], weights)
        digests[idx] = dg.cpu().numpy()
        if keep:
            for k, o in zip(idx, offs):
                if k in keep:
                    an, bn = reqs[k][1], reqs[k][2]
                    res["kept"][k] = (d_in[o:o + an + bn].cpu().numpy().view(np.uint64).copy(),
                                      d_out[o:o + an + bn].cpu().numpy().view(np.uint64).copy())
        res["mpn_limbs"] += tot
        res["mpn_requests"] += len(idx)

    # flagged mpn requests: one list call per chunk, queued by native code;
    # the context's scratch is sized outside the timing by untimed products of
    # the largest request and of the request whose configuration needs the
    # most residue words (a list call grows the scratch to its products' need)
    if mpn_list:
        for big in {max(mpn_list, key=lambda k: reqs[k][1] + reqs[k][2]),
                    max(mpn_list, key=lambda k: (configs[k].np << configs[k].logM, reqs[k][1] + reqs[k][2]))}:
            an, bn = reqs[big][1], reqs[big][2]
            ta = torch.zeros(an + bn, dtype=torch.int64, device=dev)
            tz = torch.empty(an + bn, dtype=torch.int64, device=dev)
            ctx.mpn_mul_device_list([MulReq(tz.data_ptr(), ta.data_ptr(), an, ta.data_ptr() + 8 * an, bn)],
                                    [configs[big]], s)
            stream.synchronize()
            del ta, tz
    for ci, idx in enumerate(_chunks(mpn_list, lambda k: reqs[k][1] + reqs[k][2], chunk_limbs)):
        tot = sum(reqs[k][1] + reqs[k][2] for k in idx)
        d_in = operands(idx, lambda k: reqs[k][1] + reqs[k][2])
        d_out = torch.empty(tot, dtype=torch.int64, device=dev)
        lst, offs, off = [], [], 0
        for k in idx:
            an, bn = reqs[k][1], reqs[k][2]
            p = d_in.data_ptr() + 8 * off
            lst.append(MulReq(d_out.data_ptr() + 8 * off, p, an, p + 8 * an, bn))
            offs.append(off)
            off += an + bn
        ev0.record(stream)
        ctx.mpn_mul_device_list(lst, [configs[k] for k in idx], s)
        ev1.record(stream)
        ev1.synchronize()
        res["mpn_ms"] += ev0.elapsed_time(ev1)
        dg = _digests(torch, d_out, offs, [reqs[k][1] + reqs[k][2] for k in idx], weights)
        digests[idx] = dg.cpu().numpy()
        if keep:
            for k, o in zip(idx, offs):
                if k in keep:
                    an, bn = reqs[k][1], reqs[k][2]
                    res["kept"][k] = (d_in[o:o + an + bn].cpu().numpy().view(np.uint64).copy(),
                                      d_out[o:o + an + bn].cpu().numpy().view(np.uint64).copy())
        res["mpn_limbs"] += tot
        res["mpn_requests"] += len(idx)
        res["mpn_listed_requests"] = res.get("mpn_listed_requests", 0) + len(idx)

    if fz:
        # size the context's scratch outside the timing: untimed products of
        # the largest integer-polynomial request and of the one whose
        # configuration needs the most residue words
        for big in {max(fz, key=lambda k: (reqs[k][1] + reqs[k][2] - 1) * (reqs[k][3] + reqs[k][4] - 1)),
                    max(fz, key=lambda k: (configs[k].np << configs[k].logM,
                                           (reqs[k][1] + reqs[k][2] - 1) * (reqs[k][3] + reqs[k][4] - 1)))}:
            _, an, bn, aw, bw = reqs[big]
            ta = torch.zeros(an * aw + bn * bw, dtype=torch.int64, device=dev)
            tz = torch.empty((an + bn - 1) * (aw + bw + 1), dtype=torch.int64, device=dev)
            ctx.fmpz_poly_mul_device_list(
                [FmpzMulReq(tz.data_ptr(), aw + bw + 1, 0, an + bn - 1, ta.data_ptr(), aw, an,
                            ta.data_ptr() + 8 * an * aw, bw, bn)], [configs[big]], s)
            stream.synchronize()
            del ta, tz

    def fz_size(k):
        _, an, bn, aw, bw = reqs[k]
        return an * aw + bn * bw + (an + bn - 1) * (aw + bw + 1)

    for ci, idx in enumerate(_chunks(fz, fz_size, chunk_limbs)):
        tin = sum(reqs[k][1] * reqs[k][3] + reqs[k][2] * reqs[k][4] for k in idx)
        tout = sum((reqs[k][1] + reqs[k][2] - 1) * (reqs[k][3] + reqs[k][4] + 1) for k in idx)
        # coefficients of w limbs uniform in (-2^(64w-1), 2^(64w-1)): bits = 64w - 1
        d_in = operands(idx, lambda k: reqs[k][1] * reqs[k][3] + reqs[k][2] * reqs[k][4])
        d_out = torch.empty(tout, dtype=torch.int64, device=dev)
        lst, ins, outs, zlens = [], [], [], []
        oi = oo = 0
        for k in idx:
            _, an, bn, aw, bw = reqs[k]
            zw, zn = aw + bw + 1, an + bn - 1
            pa = d_in.data_ptr() + 8 * oi
            lst.append(FmpzMulReq(d_out.data_ptr() + 8 * oo, zw, 0, zn, pa, aw, an,
                                  pa + 8 * an * aw, bw, bn))
            ins.append(oi)
            outs.append(oo)
            zlens.append(zn * zw)
            oi += an * aw + bn * bw
            oo += zn * zw
        ev0.record(stream)
        ctx.fmpz_poly_mul_device_list(lst, [configs[k] for k in idx], s)
        ev1.record(stream)
        ev1.synchronize()
        res["fmpz_ms"] += ev0.elapsed_time(ev1)
        dg = _digests(torch, d_out, outs, zlens, weights)
        digests[idx] = dg.cpu().numpy()
        if keep:
            for k, i0, o0 in zip(idx, ins, outs):
                if k in keep:
                    _, an, bn, aw, bw = reqs[k]
                    zw, zn = aw + bw + 1, an + bn - 1
                    res["kept"][k] = (
                        d_in[i0:i0 + an * aw].cpu().numpy().view(np.uint64).copy(),
                        d_in[i0 + an * aw:i0 + an * aw + bn * bw].cpu().numpy().view(np.uint64).copy(),
                        d_out[o0:o0 + zn * zw].cpu().numpy().view(np.uint64).copy())
        res["fmpz_coeff_limbs"] += tin
        res["fmpz_requests"] += len(idx)
    res["total_ms"] = res["mpn_ms"] + res["fmpz_ms"]
    res["digests"] = digests
    return res
