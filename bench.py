#!/usr/bin/env python3
"""Headline benchmark: bit-exact product throughput of a 2^24 x 2^24-limb
mpn_mul on one B200 (Gbit/s of product = 64 (an + bn) / t).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mpn24|mpn24x20]

Prints one JSON line (rank 0).  Our arm:
  value       device-resident throughput: operands already in HBM, K products
              timed with CUDA events on the launching stream;
  e2e         the same metric through the host-pointer C-ABI call
              (gpu_mpn_ctx_mpn_mul) from pinned host buffers, host<->device
              copies inside the timed region;
  roofline    the dominant kernel's algorithmic bytes / its mean launch time
              (CUDA events recorded by the library between launches);
  cpu_baseline the reference's own fft_small (oracle/_ref, compiled from the
              reference tree) timed on this host's cores.
The reference arm (--impl reference) times that CPU implementation alone.
Under torchrun each rank runs an independent replica (no collective on the
data path); the device time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bit-exact product Gbit/s, mpn_mul 2^24 limbs + uneven batch: learned vs plain"
WORKLOADS = {
    "mpn24": (1 << 24, 1 << 24, "mpn_mul 2^24 x 2^24 limbs, uniform random limbs"),
    "mpn24x20": (1 << 24, 1 << 20, "mpn_mul 2^24 x 2^20 limbs (unbalanced), uniform random limbs"),
    # profiling-sized case: operands 64 MB, residues 320 MB (larger than L2)
    "mpn22": (1 << 22, 1 << 22, "mpn_mul 2^22 x 2^22 limbs, uniform random limbs"),
    # the small-product (latency-bound) case, 2^17-point transforms
    "mpn16": (1 << 16, 1 << 16, "mpn_mul 2^16 x 2^16 limbs, uniform random limbs"),
    # a 3 2^23-point (truncated-length) transform
    "mpn3x22": (3 << 22, 3 << 22, "mpn_mul 3 2^22 x 3 2^22 limbs, uniform random limbs"),
}
NS_LIMB_BITS = 64

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch measured
# with ncu on the headline 2^24 x 2^24-limb product itself (M = 2^25, 5 primes;
# profiles/*_mpn24.md); for another size the figure is scaled by M / 2^25
# (traffic grows in proportion to the residue points).
NCU_TRAFFIC_2P25 = {
    "k_fwd_cols": 0.269502e9 + 1.291129e9,
    "k_rows": 1.343848e9 + 0.625707e9,
    "k_inv_cols": 0.671660e9 + 0.617331e9,
    "k_crt_carry": 0.671662e9 + 0.244607e9,
}


def splitmix_limbs(seed, n):
    """Same generator as the test fixtures (splitmix64), vectorised."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    if n and x[-1] == 0:
        x[-1] = 1
    return x


def to_int(x):
    return int.from_bytes(np.ascontiguousarray(x, dtype=np.uint64).tobytes(), "little")


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def ref_library():
    import oracle
    if oracle.have_ref():
        L = oracle.ref()
        n = os.cpu_count() or 1
        L.flint_set_num_threads(n)
        return L, "reference", n
    return None, "port", 1


def host_info():
    """CPU model, host threads and GMP version of this host (the CPU
    baseline's context)."""
    import ctypes
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    gmp_version = "unknown"
    try:
        import oracle
        gmp_version = ctypes.c_char_p.in_dll(oracle.gmp(), "__gmp_version").value.decode()
    except (OSError, ValueError, AttributeError):
        pass
    return {"cpu_model": model, "host_threads": os.cpu_count() or 1, "gmp_version": gmp_version}


def cpu_baseline_run(an, bn, steps, warmup, max_seconds=60.0):
    """Time the reference's fft_small mpn_mul (or, when it is not built, the
    oracle's C restatement on a smaller sample) on this host."""
    import oracle
    L, kind, nthreads = ref_library()
    if L is not None:
        a, b = splitmix_limbs(3, an), splitmix_limbs(4, bn)
        fn = lambda: oracle.ref_mpn_mul(a, b)  # noqa: E731
        sample = "full %dx%d-limb product per step" % (an, bn)
        bits = NS_LIMB_BITS * (an + bn)
        # fft_small caps its pool at 8 threads (mpn_mul.c:1257)
        cores = min(nthreads, 8)
    else:
        n = 1 << 16
        a, b = splitmix_limbs(3, n), splitmix_limbs(4, n)
        fn = lambda: oracle.port_mpn_mul(a, b)  # noqa: E731
        sample = "2^16 x 2^16-limb product per step (C restatement, 1 thread)"
        bits = NS_LIMB_BITS * 2 * n
        cores = 1
    for _ in range(max(warmup, 1)):
        fn()
    times = []
    t_all = time.perf_counter()
    for _ in range(steps):
        t = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t_all > max_seconds:
            break
    med = statistics.median(times)
    return {"value": bits / med / 1e9, "unit": "Gbit/s", "cores": cores, "kind": kind,
            "sample": sample + ", median of %d, host threads available %d" %
            (len(times), os.cpu_count() or 1),
            "ms_per_step": med * 1e3, "steps_timed": len(times), **host_info()}


BATCH_N, BATCH_SEED = 4096, 4096


def replica_seeds(rank):
    """Operand seeds of rank `rank`: every replica multiplies its own operands."""
    return 3 + 1000 * rank, 4 + 1000 * rank


def max_over_ranks(x, dist, device):
    """Max of a per-rank time over all ranks (replicas finish when the
    slowest does); identity without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_on_stream(torch, stream, fn, steps, warmup):
    """Mean milliseconds of fn() over `steps` calls, CUDA events on `stream`."""
    for _ in range(max(warmup, 3)):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def train_cost_model(ctx):
    """The learned schedule used by the batch and stream legs: exhaustive
    autotuner timings of a training sample (mpn products timed as the marginal
    cost inside a batch, integer-polynomial products alone), then the MLP cost
    model trained on them by the library's CUDA kernels."""
    from flint_b200 import tuner
    from flint_b200.workload import request_stream, uneven_batch
    t0 = time.perf_counter()
    train = [(0, a, b) for a, b in uneven_batch(BATCH_SEED + 1, 160)]
    train += request_stream(STREAM_SEED + 1, 192)
    tun = tuner.Autotuner(ctx, reps=3, batched=True)
    X, t = tuner.dataset(tun, train)
    t_tune = time.perf_counter() - t0
    t0 = time.perf_counter()
    # the model's argmin replaces the fixed rule's configuration only where it
    # predicts at least 10% saving (measured: batch 446 -> 463 Gbit/s, stream
    # 0.98 -> 1.00 of the rule, held-out regret 2.3% -> 0.2%, against no margin)
    model = tuner.CostModel(seed=11, margin=0.10)
    loss = model.fit(X, t, epochs=800)
    info = {"train_requests": len(train), "train_rows": int(len(X)), "tuning_s": t_tune,
            "fit_s": time.perf_counter() - t0, "fit_mse_log_ms": loss,
            "decision_margin": model.margin, "class_margin": CLASS_MARGIN,
            "decisions": "per class of the fixed rule (requests of one kind and one rule configuration), by "
                         "the model's summed prediction over the class (class_margin for mpn classes, "
                         "decision_margin for integer-polynomial ones); in the request stream "
                         "an mpn request moves to a flagged configuration (run alone) only where the model "
                         "predicts decision_margin below its class's choice",
            "network": "%d -> 64 -> 64 -> 64 -> 1 ReLU fp32, Adam, library CUDA kernels" % tuner.N_FEATURES,
            "candidates": "route (transform / basecase: short operand up to 4096 limbs alone, 1024 in "
                          "a planned batch), primes (min, +1), length (min, x2), rows (the rule's, the longest .. "
                          "8x shorter), and for mpn requests run alone the THREE (3 2^k length), SPLIT and "
                          "row-pass width (16 / 32 points per thread) flags"}
    return model, tun, info


STREAM_SEED = 5005
# a planned batch's classes move to the learned configuration where the model
# predicts at least this saving over the class's requests
# (tuner.CostModel.choose_classes)
CLASS_MARGIN = 0.05


def bench_stream(torch, FB, ctx, dev, stream, model, tun, n_req, cpu_seconds, n_held=1000):
    """The mixed request stream (half mpn products, an log-uniform in
    [2^6, 2^22], ratio log-uniform in [1, 64]; half integer-polynomial
    products, lengths log-uniform in [2^8, 2^16], coefficient bits uniform in
    [64, 4096]) under the learned schedule and under the fixed rule.  Every
    product of the two runs is compared by a 64-bit device digest; a
    stratified subsample is compared limb for limb with the reference's own
    products (and timed on the host)."""
    from flint_b200 import tuner
    from flint_b200.stream import run_stream
    from flint_b200.workload import request_stream
    reqs = request_stream(STREAM_SEED, n_req)
    t0 = time.perf_counter()
    learned = model.choose_stream(reqs, class_margin=CLASS_MARGIN)
    t_choose = time.perf_counter() - t0
    default = [tuner.default_config(r) for r in reqs]
    refrule = [tuner.reference_rule(r) for r in reqs]
    keep = stream_subsample(reqs)
    w0 = time.perf_counter()
    rl = run_stream(ctx, torch, reqs, learned, 17, stream, dev, keep=keep)
    w1 = time.perf_counter()
    rd = run_stream(ctx, torch, reqs, default, 17, stream, dev)
    w2 = time.perf_counter()
    rr = run_stream(ctx, torch, reqs, refrule, 17, stream, dev)
    w3 = time.perf_counter()
    same = (rl["digests"] == rd["digests"]) & (rl["digests"] == rr["digests"])
    held = request_stream(STREAM_SEED + 2, n_held)
    t0 = time.perf_counter()
    reg = tuner.regret(tun, held, model.choose_stream(held, class_margin=CLASS_MARGIN))
    reg["seconds"] = time.perf_counter() - t0
    bits_mpn = NS_LIMB_BITS * rl["mpn_limbs"]
    res = {
        "workload": "%d requests: half mpn_mul (an log-uniform [2^6, 2^22], an/bn log-uniform "
                    "[1, 64]), half fmpz_poly_mul (lengths log-uniform [2^8, 2^16], coefficient "
                    "bits uniform [64, 4096]), seed %d; mpn products in planned batches, "
                    "integer polynomials in list calls (gpu_fmpz_poly_mul_mid_device_list)"
                    % (n_req, STREAM_SEED),
        "requests": n_req, "mpn_requests": rl["mpn_requests"], "fmpz_requests": rl["fmpz_requests"],
        "mpn_limbs": rl["mpn_limbs"], "fmpz_coeff_limbs": rl["fmpz_coeff_limbs"],
        "learned": {"total_ms": rl["total_ms"], "mpn_ms": rl["mpn_ms"], "fmpz_ms": rl["fmpz_ms"],
                    "mpn_Gbit_s": bits_mpn / rl["mpn_ms"] / 1e6},
        "default_rule": {"total_ms": rd["total_ms"], "mpn_ms": rd["mpn_ms"], "fmpz_ms": rd["fmpz_ms"],
                         "mpn_Gbit_s": bits_mpn / rd["mpn_ms"] / 1e6,
                         "rule": "fewest primes, shortest power-of-two transform, longest rows, "
                                 "every mpn product in a planned batch"},
        "reference_rule": {"total_ms": rr["total_ms"], "mpn_ms": rr["mpn_ms"], "fmpz_ms": rr["fmpz_ms"],
                           "mpn_Gbit_s": bits_mpn / rr["mpn_ms"] / 1e6,
                           "rule": "the reference's mpn_ctx_best_profile score over this library's "
                                   "configurations (gpu_mul_reference_rule, host C): 3 2^k lengths where "
                                   "they fit, run per instance"},
        "gain_over_default_rule": rd["total_ms"] / rl["total_ms"],
        "gain_over_reference_rule": rr["total_ms"] / rl["total_ms"],
        "flags_chosen": {"three": sum(bool(c.flags & FB.FLAG_THREE) for c in learned),
                         "split": sum(bool(c.flags & FB.FLAG_SPLIT) for c in learned),
                         "rows16": sum(bool(c.flags & FB.FLAG_ROWS16) for c in learned),
                         "rows32": sum(bool(c.flags & FB.FLAG_ROWS32) for c in learned)},
        "choose_s": t_choose, "wall_s": {"learned_run": w1 - w0, "default_run": w2 - w1, "reference_rule_run": w3 - w2},
        "routes": {"transform": sum(c.route == 0 for c in learned),
                   "basecase": sum(c.route == 1 for c in learned)},
        "identical_to_default_rule": bool(same.all()),
        "identical_note": "learned, fixed-rule and reference-rule runs: every product's digest equal",
        "digests_compared": int(len(same)), "digests_equal": int(same.sum()),
        "digest_note": "per product: sum of its limbs times fixed pseudo-random 64-bit weights, "
                       "mod 2^64, computed on the device, learned run against default-rule run",
        "held_out_regret_vs_exhaustive": reg,
    }
    if cpu_seconds > 0:
        res["cpu_baseline"] = stream_cpu_check(reqs, rl["kept"], cpu_seconds)
    return res


def stream_subsample(reqs, per_kind=24, mpn_cap=1 << 20, fmpz_cap=1 << 22):
    """Indices of a stratified subsample of the stream: for each kind, requests
    spread evenly over the kind's size order, up to a size cap so the
    reference's host products stay within seconds."""
    out = set()
    for kind, cap in ((0, mpn_cap), (1, fmpz_cap)):
        idx = [k for k, r in enumerate(reqs) if r[0] == kind]
        size = (lambda r: r[1] + r[2]) if kind == 0 else (lambda r: (r[1] + r[2]) * (r[3] + r[4]))
        idx = sorted((k for k in idx if size(reqs[k]) <= cap), key=lambda k: size(reqs[k]))
        if idx:
            step = max(1, len(idx) // per_kind)
            out.update(idx[::step][:per_kind])
    return out


def stream_cpu_check(reqs, kept, seconds):
    """The reference's own products for the stream's subsample, timed on the
    host, each compared limb for limb with the GPU's product."""
    import oracle
    L, kind, nthreads = ref_library()
    if L is None:
        return None
    t0 = time.perf_counter()
    done, same, t_ref, bits = 0, 0, 0.0, 0
    for k in sorted(kept):
        if time.perf_counter() - t0 > seconds:
            break
        r = reqs[k]
        if r[0] == 0:
            ops, z = kept[k]
            an, bn = r[1], r[2]
            t = time.perf_counter()
            want = oracle.ref_mpn_mul(ops[:an], ops[an:an + bn])
            t_ref += time.perf_counter() - t
            bits += NS_LIMB_BITS * (an + bn)
        else:
            a, b, z = kept[k]
            _, an, bn, aw, bw = r
            zw = aw + bw + 1
            t = time.perf_counter()
            want = oracle.ref_fmpz_poly_mul_raw(a.reshape(an, aw), b.reshape(bn, bw), zw)
            t_ref += time.perf_counter() - t
            want = want.reshape(-1)
        done += 1
        same += int(np.array_equal(np.asarray(want).reshape(-1), np.asarray(z).reshape(-1)))
    return {"checked": done, "identical": same, "ref_seconds": t_ref, "cores": min(nthreads, 8),
            "kind": kind, **host_info(),
            "sample": "stratified subsample: up to 24 mpn products (an + bn <= 2^20 limbs) and 24 "
                      "integer-polynomial products (<= 2^22 coefficient limbs), spread over each "
                      "kind's size order; reference product vs GPU product, limb for limb"}


def bench_batch(torch, FB, ctx, dev, stream, steps, warmup, cpu_seconds, model, tun, train_info):
    """4096 uneven products (an = round(2^U), U ~ U[10,18]; bn = an / 2^V,
    V ~ U[0,4]): the per-instance device entry point in a loop against one
    planned batch.  Returns the `batch` object of the JSON line."""
    from flint_b200 import tuner
    from flint_b200.workload import batch_operands, uneven_batch
    sizes = uneven_batch(BATCH_SEED, BATCH_N)
    host, spans = batch_operands(7, sizes)
    total = int(sum(a + b for a, b in sizes))
    d_in = torch.from_numpy(host.view(np.int64)).to(dev)
    d_out = torch.empty(total, dtype=torch.int64, device=dev)
    d_ref = torch.empty(total, dtype=torch.int64, device=dev)
    reqs, zoffs, off = [], [], 0
    for (ao, an, bo, bn) in spans:
        reqs.append((d_out.data_ptr() + 8 * off, d_in.data_ptr() + 8 * ao, an,
                     d_in.data_ptr() + 8 * bo, bn))
        zoffs.append(off)
        off += an + bn
    delta = d_ref.data_ptr() - d_out.data_ptr()
    s = stream.cuda_stream

    def per_instance_python():
        for (z, a, an, b, bn) in reqs:
            ctx.mpn_mul_device(z + delta, a, an, b, bn, s)

    # the per-instance path without the interpreter: one native call queues
    # every product as gpu_mpn_mul_device would (gpu_mpn_mul_device_list)
    list_reqs = [FB.MulReq(z + delta, a, an, b, bn) for (z, a, an, b, bn) in reqs]

    def per_instance():
        ctx.mpn_mul_device_list(list_reqs, None, s)

    bits = NS_LIMB_BITS * total
    k_plain = max(2, steps // 3)
    ms_plain = time_on_stream(torch, stream, per_instance, k_plain, 3)
    stream.synchronize()
    t0 = time.perf_counter()
    per_instance()
    host_issue_ms = (time.perf_counter() - t0) * 1e3
    stream.synchronize()
    # GPU-busy time of the per-instance path: the sum of its kernels' own
    # durations (CUDA events around each launch) over one step
    ctx.set_timing(True)
    per_instance()
    stream.synchronize()
    busy_ms = sum(v[0] for v in ctx.kernel_times().values())
    ctx.set_timing(False)
    ms_plain_py = time_on_stream(torch, stream, per_instance_python, max(2, k_plain // 2), 1)
    B0 = FB.MpnBatch(ctx, reqs)
    ms_default = time_on_stream(torch, stream, lambda: B0.run(s), steps, warmup)
    B0.check(s)
    exact_default = bool(torch.equal(d_out, d_ref))
    B0.close()
    # learned schedule: one configuration per request of the batch from the
    # cost model; its regret on held-out requests of this distribution
    # planned batches run plain transforms: the model chooses among those
    held = [(0, a, b) for a, b in uneven_batch(BATCH_SEED + 2, 48)]
    reg = tuner.regret(tun, held, model.choose_classes(held, margin=CLASS_MARGIN), flags=False)
    t0 = time.perf_counter()
    configs = model.choose_classes([(0, a, b) for a, b in sizes], margin=CLASS_MARGIN)
    t_choose = time.perf_counter() - t0
    B = FB.MpnBatch(ctx, reqs, configs=configs)
    d_out.fill_(0)
    ms_batch = time_on_stream(torch, stream, lambda: B.run(s), steps, warmup)
    B.check(s)
    exact = bool(torch.equal(d_out, d_ref)) and exact_default
    # residue fingerprints of a subsample (Python integers)
    out = d_out.cpu().numpy().view(np.uint64)
    q = 2305843009213693951
    fp_ok = True
    for k in range(0, BATCH_N, 97):
        ao, an, bo, bn = spans[k]
        zo = zoffs[k]
        fp_ok &= (to_int(host[ao:ao + an]) % q) * (to_int(host[bo:bo + bn]) % q) % q == \
            to_int(out[zo:zo + an + bn]) % q

    # end to end: pinned host operands in, products out, copies inside the timed region
    h_in = torch.from_numpy(host.view(np.int64)).pin_memory()
    h_out = torch.empty(total, dtype=torch.int64).pin_memory()

    def e2e():
        d_in.copy_(h_in, non_blocking=True)
        B.run(s)
        h_out.copy_(d_out, non_blocking=True)

    ms_e2e_whole = time_on_stream(torch, stream, e2e, max(3, steps // 2), 2)
    B.check(s)
    e2e_ok = bool(np.array_equal(h_out.numpy().view(np.uint64), out))

    # end to end, overlapped: the requests in E2E_CHUNKS runs of consecutive
    # requests (contiguous operand and product ranges), one planned batch
    # each; chunk c's upload, batch and download go on an upload, the compute
    # and a download stream, so one chunk's download, the next one's batch and
    # a later one's upload overlap.  A step starts after the previous one has
    # finished (its first upload waits for the step's start on `stream`).
    E2E_CHUNKS = 8
    cuts = [len(reqs) * c // E2E_CHUNKS for c in range(E2E_CHUNKS + 1)]
    parts = []
    for c in range(E2E_CHUNKS):
        r0, r1 = cuts[c], cuts[c + 1]
        lo, hi = spans[r0][0], spans[r1 - 1][2] + spans[r1 - 1][3]   # operands and products share offsets
        parts.append((lo, hi, FB.MpnBatch(ctx, reqs[r0:r1], configs=configs[r0:r1])))
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def e2e_overlapped():
        start = torch.cuda.Event()
        start.record(stream)
        up.wait_event(start)
        for lo, hi, Bc in parts:
            with torch.cuda.stream(up):
                d_in[lo:hi].copy_(h_in[lo:hi], non_blocking=True)
            e_in = torch.cuda.Event()
            e_in.record(up)
            stream.wait_event(e_in)
            Bc.run(s)
            e_run = torch.cuda.Event()
            e_run.record(stream)
            down.wait_event(e_run)
            with torch.cuda.stream(down):
                h_out[lo:hi].copy_(d_out[lo:hi], non_blocking=True)
        done = torch.cuda.Event()
        done.record(down)
        stream.wait_event(done)

    h_out.zero_()
    ms_e2e = time_on_stream(torch, stream, e2e_overlapped, max(3, steps // 2), 2)
    for _, _, Bc in parts:
        Bc.check(s)
        Bc.close()
    e2e_ok = e2e_ok and bool(np.array_equal(h_out.numpy().view(np.uint64), out))
    res = {
        "workload": "%d uneven products, an = round(2^U), U~U[10,18], bn = max(1, round(an/2^V)), "
                    "V~U[0,4], seed %d" % (BATCH_N, BATCH_SEED),
        "limbs": total, "classes": B.classes, "launches_per_step": B.launches,
        "schedule": "learned (cost model per request, batched by configuration)",
        "value": bits / ms_batch / 1e6, "unit": "Gbit/s", "ms_per_step": ms_batch,
        "per_instance": {"value": bits / ms_plain / 1e6, "ms_per_step": ms_plain,
                         "launches_per_step": 4 * BATCH_N,
                         "api": "gpu_mpn_mul_device_list: one native call queues the products one by "
                                "one, as gpu_mpn_mul_device runs them",
                         "host_issue_ms_per_step": host_issue_ms, "gpu_busy_ms_per_step": busy_ms,
                         "note": "launch-bound: the kernels are busy for gpu_busy_ms of each step, the host "
                                 "needs host_issue_ms to issue its 4 launches per product"},
        "per_instance_python_loop": {"value": bits / ms_plain_py / 1e6, "ms_per_step": ms_plain_py,
                                     "api": "gpu_mpn_mul_device called from a Python loop"},
        "plain_batched": {"value": bits / ms_default / 1e6, "ms_per_step": ms_default,
                          "schedule": "default configuration for every request"},
        "speedup_vs_per_instance": ms_plain / ms_batch,
        "speedup_vs_plain_batched": ms_default / ms_batch,
        "learned": {"training": train_info, "choose_s_4096": t_choose,
                    "routes": {"transform": sum(c.route == 0 for c in configs),
                               "basecase": sum(c.route == 1 for c in configs)},
                    "held_out_regret_vs_exhaustive": reg},
        "e2e": {"value": bits / ms_e2e / 1e6, "unit": "Gbit/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": 8 * total, "d2h_bytes_per_step": 8 * total,
                "schedule": "%d chunks of consecutive requests, upload / batch / download overlapped "
                            "on three streams" % E2E_CHUNKS},
        "e2e_unchunked": {"value": bits / ms_e2e_whole / 1e6, "unit": "Gbit/s", "ms_per_step": ms_e2e_whole,
                          "schedule": "whole batch: upload, batch, download in turn"},
        "exact_vs_per_instance": exact, "fingerprints_ok": bool(fp_ok), "e2e_matches": e2e_ok,
        "roofline": {"bound": "hbm", "alg_bytes": 208 * total,
                     "achieved": 208 * total / ms_batch / 1e6},
    }
    B.close()
    if cpu_seconds > 0:
        res["cpu_baseline"] = batch_cpu_baseline(sizes, host, spans, cpu_seconds)
    return res


def batch_cpu_baseline(sizes, host, spans, seconds):
    """The reference's fft_small, one product at a time over the batch in
    order (all host threads), until `seconds` have passed."""
    import oracle
    L, kind, nthreads = ref_library()
    if L is None:
        return None
    t0 = time.perf_counter()
    done_limbs, k = 0, 0
    while k < len(spans) and time.perf_counter() - t0 < seconds:
        ao, an, bo, bn = spans[k]
        oracle.ref_mpn_mul(host[ao:ao + an], host[bo:bo + bn])
        done_limbs += an + bn
        k += 1
    dt = time.perf_counter() - t0
    return {"value": NS_LIMB_BITS * done_limbs / dt / 1e9, "unit": "Gbit/s",
            "cores": min(nthreads, 8), "kind": kind,
            "sample": "first %d of the %d products, one mpn_ctx_mpn_mul each" % (k, len(spans))}


def bench_configs(torch, FB, ctx, dev, stream, steps, cpu):
    """The other measured configurations: 2^16 x 2^16, 2^24 x 2^20 and
    3 2^22 x 3 2^22 limbs (mpn_mul; the last on a 3 2^23-point transform), and
    the nmod window product (coefficients [2^19, 3 2^19) of
    two 2^20-coefficient polynomials mod an odd n in [2^61, 2^62)), each
    device-resident (CUDA events) against its algorithmic byte model, with
    the compiled reference timed on the host and its output compared."""
    import oracle
    L = ref_library()[0] if cpu else None
    peak = load_peaks()[0]
    s = stream.cuda_stream
    out = []

    def ref_time(fn, reps):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            r = fn()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), r

    for name, an, bn, seed in [("1: mpn_mul 2^16 x 2^16", 1 << 16, 1 << 16, 11),
                               ("2b: mpn_mul 2^24 x 2^20", 1 << 24, 1 << 20, 12),
                               ("2c: mpn_mul 3 2^22 x 3 2^22 (a 3 2^23-point truncated transform)",
                                3 << 22, 3 << 22, 13)]:
        a, b = splitmix_limbs(seed, an), splitmix_limbs(seed + 1, bn)
        da = torch.from_numpy(a.view(np.int64)).to(dev)
        db = torch.from_numpy(b.view(np.int64)).to(dev)
        dz = torch.empty(an + bn, dtype=torch.int64, device=dev)
        k = max(steps, 50 if an < (1 << 20) else 10)
        ms = time_on_stream(torch, stream, lambda: ctx.mpn_mul_device(dz.data_ptr(), da.data_ptr(), an,
                                                                    db.data_ptr(), bn, s), k, 3)
        z = dz.cpu().numpy().view(np.uint64)
        alg = 208 * (an + bn)
        r = {"workload": name, "ms": ms, "value": NS_LIMB_BITS * (an + bn) / ms / 1e6, "unit": "Gbit/s",
             "transform_points": FB.mpn_mul_transform_points(an, bn),
             "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved": alg / ms / 1e6, "peak": peak,
                          "frac": alg / ms / 1e6 / peak}}
        if L is not None:
            t, zr = ref_time(lambda: oracle.ref_mpn_mul(a, b), 5 if an < (1 << 20) else 2)
            r.update(cpu_ms=t * 1e3, speedup_vs_cpu=t * 1e3 / ms, identical_to_reference=bool(np.array_equal(z, zr)))
        out.append(r)
    # nmod window product
    n_ = (int(splitmix_limbs(21, 1)[0]) >> 2 | (1 << 61)) | 1
    an = bn = 1 << 20
    zl, zh = 1 << 19, 3 << 19
    a = splitmix_limbs(22, an) % np.uint64(n_)     # inputs reduced mod n, as the call requires
    b = splitmix_limbs(23, bn) % np.uint64(n_)
    da = torch.from_numpy(a.view(np.int64)).to(dev)
    db = torch.from_numpy(b.view(np.int64)).to(dev)
    dz = torch.empty(zh - zl, dtype=torch.int64, device=dev)
    ms = time_on_stream(torch, stream, lambda: ctx.nmod_poly_mul_mid_device(dz.data_ptr(), zl, zh, da.data_ptr(),
                                                                          an, db.data_ptr(), bn, n_, s),
                        max(steps, 50), 3)
    z = dz.cpu().numpy().view(np.uint64)
    alg = 200 * (an + bn) + 8 * (zh - zl)
    r = {"workload": "3: nmod window product, coefficients [2^19, 3 2^19) of two 2^20-coefficient "
                     "polynomials mod odd n in [2^61, 2^62)", "ms": ms,
         "value": (zh - zl) / ms / 1e3, "unit": "M coefficients/s",
         "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved": alg / ms / 1e6, "peak": peak,
                      "frac": alg / ms / 1e6 / peak,
                      "note": "the working set is largely L2-resident, so a fraction above 1 is possible"}}
    if L is not None:
        t, zr = ref_time(lambda: oracle.ref_nmod_mul_mid(zl, zh, a, b, n_), 3)
        r.update(cpu_ms=t * 1e3, speedup_vs_cpu=t * 1e3 / ms, identical_to_reference=bool(np.array_equal(z, zr)))
    out.append(r)
    if L is not None:
        for r in out:
            r["cpu_note"] = "compiled reference on all host threads, median of a few calls"
    return out


def bench_precomp(torch, FB, ctx, dev, stream, steps):
    """Transformed-operand reuse (the reference's op API): b of 2^22 limbs
    transformed once, then for each a of 2^22 limbs: forward transform of a,
    pointwise product, inverse, export -- against the full product."""
    n = 1 << 22
    g = torch.Generator(device=dev)
    g.manual_seed(123)
    a = torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64, device=dev, generator=g)
    b = torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64, device=dev, generator=g)
    z1 = torch.empty(2 * n, dtype=torch.int64, device=dev)
    z2 = torch.empty_like(z1)
    s = stream.cuda_stream
    P = FB.FftPlan.mpn(ctx, n, n)
    A, B, Z = P.op(), P.op(), P.op()
    B.fft(b.data_ptr(), n, s)

    def with_op():
        A.fft(a.data_ptr(), n, s)
        P.pointwise(FB.OP_MUL, Z, A, B, s)
        Z.ifft(s)
        Z.export_mpn(z1.data_ptr(), 2 * n, s)

    ms_op = time_on_stream(torch, stream, with_op, steps, 3)
    ms_full = time_on_stream(torch, stream, lambda: ctx.mpn_mul_device(z2.data_ptr(), a.data_ptr(), n,
                                                                       b.data_ptr(), n, s), steps, 3)
    P.check(s)
    same = bool(torch.equal(z1, z2))
    for o in (A, B, Z):
        o.close()
    P.close()
    return {"workload": "a x b, 2^22 x 2^22 limbs, b transformed once (plan/op API)",
            "ms_with_transformed_b": ms_op, "ms_full_product": ms_full,
            "speedup": ms_full / ms_op, "identical": same}


# products mod 2^N + 1 (Schoenhage-Strassen pointwise stage): ring size in
# bits, products per batch; operands of every batch exceed L2 (126 MB)
NEG_WORKLOADS = [(47104, 16384), (1 << 20, 512)]


def neg_cpu_baseline(N, X, Y, seconds):
    """The reference's sd_fft_mpn_mulmod_2expp1 (its own digit split, m = 0)
    over the batch in order, one product per call, on every host thread (each
    with its own context and scratch; ctypes releases the GIL)."""
    import oracle
    if not oracle.have_ref():
        return None, None
    nthreads = os.cpu_count() or 1
    count = len(X)
    nxt = [0]
    lock = threading.Lock()
    done = [0] * nthreads
    outs = {}
    t0 = time.perf_counter()

    def work(t):
        R = oracle._RefNegCtx(N, 0)
        try:
            while time.perf_counter() - t0 < seconds:
                with lock:
                    i = nxt[0]
                    nxt[0] += 1
                if i >= count:
                    break
                z = R.mul(X[i], Y[i])
                if i < 8:
                    outs[i] = z
                done[t] += 1
        finally:
            R.close()

    th = [threading.Thread(target=work, args=(t,)) for t in range(nthreads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    k = sum(done)
    return ({"value": k / dt, "unit": "products/s", "cores": nthreads, "kind": "reference",
             "sample": "%d of the %d products, one sd_fft_mpn_mulmod_2expp1 call each" % (k, count)},
            outs)


def bench_negacyclic(torch, FB, ctx, dev, stream, steps, cpu_seconds):
    """Batches of products mod 2^N + 1 (gpu_mulmod_2expp1_batch_device),
    device-resident, against the reference's engine on the host cores."""
    res = []
    s = stream.cuda_stream
    peak, peak_kind = load_peaks()
    for N, count in NEG_WORKLOADS:
        n = N // 64
        g = torch.Generator(device=dev)
        g.manual_seed(N)
        X = torch.randint(-(1 << 63), (1 << 63) - 1, (count, n + 1), dtype=torch.int64, device=dev,
                          generator=g)
        Y = torch.randint(-(1 << 63), (1 << 63) - 1, (count, n + 1), dtype=torch.int64, device=dev,
                          generator=g)
        X[:, n] = 0
        Y[:, n] = 0
        Z = torch.empty_like(X)
        C = FB.Mulmod2expp1(ctx, N, 0)
        fn = lambda: C.batch_device(Z.data_ptr(), X.data_ptr(), Y.data_ptr(), count, None, s)  # noqa: E731
        ms = time_on_stream(torch, stream, fn, steps, 3)
        # HBM bytes per product: operands and result (n + 1 limbs each), the
        # residues written by the split (2 np m words), read and written by the
        # row pass (2 np m + np m) and read by the finisher (np m)
        alg = count * (24 * (n + 1) + 24 * C.np * C.m)
        gbps = alg / (ms / 1e3) / 1e9
        item = {"workload": "%d products mod 2^%d + 1, uniform random operands" % (count, N),
                "N": N, "count": count, "m": C.m, "b": C.b, "primes": C.np,
                "ms_per_batch": ms, "products_per_s": count / (ms / 1e3),
                "operand_Gbit_s": 2 * N * count / (ms / 1e3) / 1e9,
                "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved": gbps, "peak": peak,
                             "unit": "GB/s", "frac": gbps / peak, "peak_kind": peak_kind},
                "gpu_launches_per_batch": 4}
        if cpu_seconds > 0:
            Xh = X.cpu().numpy().view(np.uint64)
            Yh = Y.cpu().numpy().view(np.uint64)
            cb, outs = neg_cpu_baseline(N, Xh, Yh, cpu_seconds)
            if cb is not None:
                item["cpu_baseline"] = cb
                item["speedup_vs_cpu"] = item["products_per_s"] / cb["value"]
                Zh = Z.cpu().numpy().view(np.uint64)
                item["identical_to_reference_sample"] = bool(outs) and all(
                    np.array_equal(Zh[i], z) for i, z in outs.items())
        C.close()
        res.append(item)
        del X, Y, Z
    return res


def kernel_bytes(name, an, bn, np_, M, L):
    """Algorithmic bytes each kernel must move in the four-pass design:
    residues are 4-byte words, np primes, M-point transforms."""
    r = 4 * np_ * M
    return {
        "k_fwd_cols": 8 * (an + bn) + 2 * r,      # limbs in, a and b residues out
        "k_rows": 3 * r,                          # a, b rows in, product rows out
        "k_inv_cols": 2 * r,                      # in place
        "k_crt_carry": 4 * np_ * L + 8 * (an + bn),   # residues in, limbs out
    }[name]


def bench_pipe(torch, FB, a, b, z, steps, dist, dev, depth=4):
    """Host-to-host throughput of a stream of products through gpu_mpn_pipe_*:
    each product has its own pinned input and output buffers (depth sets in
    rotation), the timed region runs from the first submission to the last
    completed download (host clock, fill and drain included), and every
    output is compared with the device-resident result."""
    an, bn = len(a), len(b)
    sets = [(torch.from_numpy(a.view(np.int64)).pin_memory(), torch.from_numpy(b.view(np.int64)).pin_memory(),
             torch.empty(an + bn, dtype=torch.int64).pin_memory()) for _ in range(depth)]
    nsteps = max(8 * depth, 32)                 # fill and drain amortised over the stream
    with FB.MpnPipe(depth) as P:
        for ha, hb, hz in sets:                     # warm-up: scratch growth in every slot
            P.wait(P.submit(ha, hb, out=hz))
        for _, _, hz in sets:
            hz.zero_()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        pend = []
        for k in range(nsteps):
            ha, hb, hz = sets[k % depth]
            if len(pend) == depth:                  # the set is reused: its product must be home
                P.wait(pend.pop(0))
            pend.append(P.submit(ha, hb, out=hz))
        for t in pend:
            P.wait(t)
        s = (time.perf_counter() - t0) / nsteps
    s = max_over_ranks(s, dist, dev)
    ok = all(bool(np.array_equal(hz.numpy().view(np.uint64), z)) for _, _, hz in sets)
    return {"unit": "Gbit/s", "s_per_step": s, "depth": depth, "steps": nsteps,
            "h2d_bytes_per_step": 8 * (an + bn), "d2h_bytes_per_step": 8 * (an + bn),
            "matches_device": ok,
            "api": "gpu_mpn_pipe_submit / gpu_mpn_pipe_wait (pinned host buffers, one set per slot)",
            "note": "host-clock throughput of a stream of host-resident products; one product's "
                    "download overlaps the next one's upload and kernels (full-duplex PCIe)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mpn24", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 2^16, 2^24 x 2^20 and nmod window measurements")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 4096-product uneven batch")
    ap.add_argument("--no-negacyclic", action="store_true",
                    help="skip the products mod 2^N + 1")
    ap.add_argument("--negacyclic-only", action="store_true",
                    help="run only the products mod 2^N + 1 (profiling); prints their results")
    ap.add_argument("--stream-requests", type=int, default=100000,
                    help="requests of the mixed mpn / integer-polynomial stream (0 = skip; the "
                         "configuration's stated size is 100000)")
    args = ap.parse_args()
    an, bn, desc = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": desc,
              "an": an, "bn": bn}

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_baseline_run(an, bn, args.steps, args.warmup, max_seconds=240.0)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "Gbit/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (splitmix64 limbs)",
                "config": dict(config, parallelism="host threads"),
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model",
                                                    "gmp_version")},
                "e2e": {"value": cb["value"], "unit": "Gbit/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import flint_b200 as FB
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    if args.negacyclic_only:
        ctx = FB.MpnCtx()
        res = bench_negacyclic(torch, FB, ctx, dev, torch.cuda.current_stream(dev), args.steps,
                               0.0 if args.no_cpu_baseline else 5.0)
        if rank == 0:
            print(json.dumps({"negacyclic": res}), flush=True)
        return

    sa, sb = replica_seeds(rank)
    a = splitmix_limbs(sa, an)
    b = splitmix_limbs(sb, bn)
    ctx = FB.MpnCtx()
    np_, logM = FB.mpn_mul_plan(an, bn)
    M, L = 1 << logM, an + bn - 1
    da = torch.from_numpy(a.view(np.int64)).to(dev)
    db = torch.from_numpy(b.view(np.int64)).to(dev)
    dz = torch.empty(an + bn, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        ctx.mpn_mul_device(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    # exactness spot check of the benchmarked output: residues mod 61-bit primes
    z = dz.cpu().numpy().view(np.uint64)
    ai, bi, zi = to_int(a), to_int(b), to_int(z)
    verified = all((ai % q) * (bi % q) % q == zi % q
                   for q in (2305843009213693951, 2305843009213693921))

    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # K products timed as a whole (the headline), then the same K products
    # again with the library's per-kernel events (the roofline's kernel
    # durations): the events between launches cost ~2% of a product, so the
    # headline loop runs without them
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    ctx.set_timing(True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_instrumented = e0.elapsed_time(e1) / args.steps
    ktimes = ctx.kernel_times()
    ctx.set_timing(False)
    ms = max_over_ranks(ms, dist, dev)
    ms_step = ms / args.steps
    gbits_step = NS_LIMB_BITS * (an + bn) / 1e9
    value = world * gbits_step / (ms_step / 1e3)

    # e2e: host-pointer C-ABI call from pinned host buffers
    ha = torch.from_numpy(a.view(np.int64)).pin_memory()
    hb = torch.from_numpy(b.view(np.int64)).pin_memory()
    hz = torch.empty(an + bn, dtype=torch.int64).pin_memory()
    lib = FB.lib()

    def e2e_step():
        rc = lib.gpu_mpn_ctx_mpn_mul_status(ctx.ptr, hz.data_ptr(), ha.data_ptr(), an,
                                            hb.data_ptr(), bn)
        if rc:
            raise RuntimeError(lib.gpu_fft_small_last_error().decode())

    for _ in range(2):
        e2e_step()
    e2e_steps = max(3, min(args.steps, 10))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = max_over_ranks(e2e_s, dist, dev)
    # the same products streamed through a pipeline of host-pointer products
    pipelined = bench_pipe(torch, FB, a, b, z, args.steps, dist, dev)
    pipe_s = pipelined.pop("s_per_step")
    pipelined.update(value=world * gbits_step / pipe_s, ms_per_step=pipe_s * 1e3)
    # the batch, stream and transformed-operand legs are single-GPU
    # measurements: run at N = 1 only
    batch = stream_res = precomp = negacyclic = other_configs = None
    single = world == 1
    cpu_s = 0.0 if (world > 1 or args.no_cpu_baseline) else 10.0
    if single:
        precomp = bench_precomp(torch, FB, ctx, dev, stream, max(3, args.steps // 2))
        if not args.no_configs:
            other_configs = bench_configs(torch, FB, ctx, dev, stream, args.steps, not args.no_cpu_baseline)
        if not args.no_negacyclic:
            negacyclic = bench_negacyclic(torch, FB, ctx, dev, stream, max(3, args.steps // 2),
                                          min(cpu_s, 5.0))
    if single and not (args.no_batch and args.stream_requests == 0):
        model, tun, train_info = train_cost_model(ctx)
    if single and not args.no_batch:
        batch = bench_batch(torch, FB, ctx, dev, stream, args.steps, args.warmup, cpu_s, model, tun,
                            train_info)
    if single and args.stream_requests > 0:
        stream_res = bench_stream(torch, FB, ctx, dev, stream, model, tun, args.stream_requests, cpu_s)
    clk = clocks.stop()
    e2e_ok = bool(np.array_equal(hz.numpy().view(np.uint64), z))

    peak, peak_kind = load_peaks()
    kern = {}
    for name, (tot, cnt) in ktimes.items():
        if cnt:
            per = tot / cnt
            byt = kernel_bytes(name, an, bn, np_, M, L)
            kern[name] = {"ms_per_launch": per, "share": None, "alg_bytes": byt,
                          "GBps": byt / (per / 1e3) / 1e9}
    tot_ms = sum(v["ms_per_launch"] for v in kern.values()) or 1.0
    for v in kern.values():
        v["share"] = v["ms_per_launch"] / tot_ms
    dom = max(kern, key=lambda k: kern[k]["ms_per_launch"])
    alg_pipeline = 208 * (an + bn)
    traffic = None
    scale = M / float(1 << 25)                    # residue points relative to the capture
    for name, v in kern.items():
        if name in NCU_TRAFFIC_2P25:
            v["traffic"] = NCU_TRAFFIC_2P25[name] * scale
            v["traffic_note"] = ("measured at this size" if M == 1 << 25 else
                                 "scaled from the 2^25-point capture by residue points")
    traffic = kern[dom].get("traffic")
    # integer-pipe roofline: the product's butterflies (two forward and one
    # inverse transform of M points per prime) at the butterfly rate measured
    # live by the calibration kernel
    bfly = 3 * logM * (M // 2) * np_
    rate = ctx.butterfly_rate()
    t_bound = bfly / rate * 1e3
    # the same per kernel: its share of the butterflies (forward columns: two
    # operands x logR levels; rows: three transforms x logC levels; inverse
    # columns: logR levels) at that rate, over its measured launch time
    logC_ = FB.resolve_config(0, an, bn).logC
    logR_ = logM - logC_
    kb = {"k_fwd_cols": 2 * logR_, "k_rows": 3 * logC_, "k_inv_cols": logR_}
    for name, v in kern.items():
        if name in kb:
            v["butterflies"] = kb[name] * (M // 2) * np_
            v["int_pipe_frac"] = v["butterflies"] / rate * 1e3 / v["ms_per_launch"]
    int_pipe = {"butterflies": bfly, "rate_per_s": rate, "t_bound_ms": t_bound,
                "frac": t_bound / ms_step,
                "note": "31-bit modular butterfly from registers on every SM (gpu_butterfly_rate); "
                        "frac = butterfly-only time at that rate / measured product time"}
    roofline = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["GBps"], "peak": peak,
                "unit": "GB/s", "frac": kern[dom]["GBps"] / peak, "traffic": traffic,
                "peak_kind": peak_kind, "int_pipe": int_pipe,
                "pipeline": {"alg_bytes": alg_pipeline,
                             "achieved": alg_pipeline / (ms_step / 1e3) / 1e9,
                             "frac": alg_pipeline / (ms_step / 1e3) / 1e9 / peak},
                "kernels": kern,
                "kernels_note": "per-launch CUDA events of a second run of the same %d products "
                                "(%.4f ms per product with the events)" % (args.steps, ms_instrumented)}
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_run(an, bn, steps=2, warmup=1, max_seconds=30.0)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model", "gmp_version")}
    line = {
        "metric": METRIC, "value": value, "unit": "Gbit/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (splitmix64 uniform limbs, top limb nonzero)",
        "config": dict(config, primes=np_, transform="2^%d four-step" % logM,
                       l2="inputs larger than L2 (%d MB operands)" % ((an + bn) * 8 >> 20),
                       parallelism="replicas" if world > 1 else "single GPU"),
        "verified_mod_q": bool(verified), "e2e_matches_device": e2e_ok,
        "e2e": {"value": world * gbits_step / e2e_s, "unit": "Gbit/s",
                "h2d_bytes_per_step": 8 * (an + bn), "d2h_bytes_per_step": 8 * (an + bn),
                "ms_per_step": e2e_s * 1e3},
        "e2e_pipelined": pipelined,
        "gpu_launches": 4 * args.steps,
        "gpu_launches_note": "headline product only; the batch object counts its own",
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "batch": batch,
        "stream": stream_res,
        "transformed_operand": precomp,
        "other_configs": other_configs,
        "negacyclic": negacyclic,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
