"""Execution of a stream of multiplication requests under a schedule.

A request is (kind, an, bn, aw, bw) as in flint_b200.tuner: kind 0 an
an x bn-limb mpn product, kind 1 an integer-polynomial product of an x bn
coefficients of aw and bw limbs.  ``run_stream`` executes every request with
the configuration a chooser gives it:

* mpn requests go in chunks (at most ``chunk_limbs`` operand limbs each) into
  planned batches (gpu_mpn_batch_init_config), so products that share a
  configuration share launches;
* integer-polynomial requests run one device call each
  (gpu_fmpz_poly_mul_mid_device_config).

Operands are generated on the device from a seed (torch's CUDA generator),
outside the timed region; the device time of the products is measured with
CUDA events on the launching stream.  ``outputs`` lets a caller keep or
compare the products (e.g. a learned schedule against the fixed rule: the
products must be identical).
"""
import numpy as np

from . import MpnBatch


def _fill_fmpz(torch, n, w, bits, gen, dev):
    """n coefficients of w limbs, uniform in (-2^bits, 2^bits), two's complement."""
    x = torch.randint(-(1 << 63), (1 << 63) - 1, (n, w), dtype=torch.int64, device=dev, generator=gen)
    t = bits - 64 * (w - 1) + 1            # significant bits of the top limb, sign included
    x[:, -1] = x[:, -1] >> (64 - t) if t < 64 else x[:, -1]
    return x


def run_stream(ctx, torch, reqs, configs, seed, stream, dev, chunk_limbs=1 << 26, keep=None,
               check_against=None):
    """Execute reqs under configs (one per request).  Returns a dict of device
    milliseconds (mpn, fmpz, total), limbs/bits processed, and, when
    check_against is another config list, whether every product equals the
    product under those configurations.  keep: optional set of request
    indices whose products are returned (host arrays) in 'kept'."""
    gen = torch.Generator(device=dev)
    s = stream.cuda_stream
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    res = {"mpn_ms": 0.0, "fmpz_ms": 0.0, "mpn_limbs": 0, "fmpz_coeff_limbs": 0,
           "mpn_requests": 0, "fmpz_requests": 0, "identical": True, "kept": {}}
    mpn = [k for k, r in enumerate(reqs) if r[0] == 0]
    fz = [k for k, r in enumerate(reqs) if r[0] == 1]
    # mpn requests: chunks of bounded operand size
    chunks, cur, size = [], [], 0
    for k in mpn:
        n = reqs[k][1] + reqs[k][2]
        if cur and size + n > chunk_limbs:
            chunks.append(cur)
            cur, size = [], 0
        cur.append(k)
        size += n
    if cur:
        chunks.append(cur)
    for ci, idx in enumerate(chunks):
        tot = sum(reqs[k][1] + reqs[k][2] for k in idx)
        gen.manual_seed(seed * 1000003 + ci)
        d_in = torch.randint(-(1 << 63), (1 << 63) - 1, (tot,), dtype=torch.int64, device=dev,
                             generator=gen)
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
        if check_against is not None:
            d_ref = torch.empty_like(d_out)
            rq2 = [(d_ref.data_ptr() + 8 * o, a, an, b, bn) for o, (_, a, an, b, bn) in zip(offs, rq)]
            with MpnBatch(ctx, rq2, configs=[check_against[k] for k in idx]) as B2:
                B2.run(s)
                B2.check(s)
            res["identical"] &= bool(torch.equal(d_out, d_ref))
        if keep:
            for k, o in zip(idx, offs):
                if k in keep:
                    an, bn = reqs[k][1], reqs[k][2]
                    res["kept"][k] = (d_in[o:o + an + bn].cpu().numpy().view(np.uint64).copy(),
                                      d_out[o:o + an + bn].cpu().numpy().view(np.uint64).copy())
        res["mpn_limbs"] += tot
        res["mpn_requests"] += len(idx)
    # integer-polynomial requests, one call each
    for k in fz:
        _, an, bn, aw, bw = reqs[k]
        bits = 64 * aw - 1
        gen.manual_seed(seed * 1000003 + 7919 * (k + 1))
        a = _fill_fmpz(torch, an, aw, bits, gen, dev)
        b = _fill_fmpz(torch, bn, bw, bits, gen, dev)
        zw = aw + bw + 1
        zn = an + bn - 1
        z = torch.empty((zn, zw), dtype=torch.int64, device=dev)
        ctx.fmpz_poly_mul_device_config(z.data_ptr(), zw, 0, zn, a.data_ptr(), aw, an, b.data_ptr(),
                                        bw, bn, configs[k], s)    # warm-up (scratch growth)
        stream.synchronize()
        ev0.record(stream)
        ctx.fmpz_poly_mul_device_config(z.data_ptr(), zw, 0, zn, a.data_ptr(), aw, an, b.data_ptr(),
                                        bw, bn, configs[k], s)
        ev1.record(stream)
        ev1.synchronize()
        res["fmpz_ms"] += ev0.elapsed_time(ev1)
        if check_against is not None:
            z2 = torch.empty_like(z)
            ctx.fmpz_poly_mul_device_config(z2.data_ptr(), zw, 0, zn, a.data_ptr(), aw, an,
                                            b.data_ptr(), bw, bn, check_against[k], s)
            stream.synchronize()
            res["identical"] &= bool(torch.equal(z, z2))
        if keep and k in keep:
            res["kept"][k] = (a.cpu().numpy().view(np.uint64).copy(),
                              b.cpu().numpy().view(np.uint64).copy(),
                              z.cpu().numpy().view(np.uint64).copy())
        res["fmpz_coeff_limbs"] += an * aw + bn * bw
        res["fmpz_requests"] += 1
    res["total_ms"] = res["mpn_ms"] + res["fmpz_ms"]
    return res
