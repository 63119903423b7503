"""Autotuner and learned schedule for the multiplication path.

The reference picks its transform parameters with a fixed heuristic
(mpn_ctx_best_profile, src/fft_small/mpn_mul.c:1248-1340) and routes small
operands to GMP by size thresholds (src/mpn_extras/mul.c:52-75).  Here the
choice per request is a gpu_mul_config:

    route   transform or basecase (schoolbook, shorter operand <= 1024 limbs)
    np      prime count (the minimum, or one more)
    logM    transform length (the minimum, or twice it)
    logC    four-step row length (the longest allowed, or 2x / 4x / 8x shorter)

Every valid configuration gives the same exact product; only time differs.

* ``candidates`` enumerates the configurations of a request;
* ``Autotuner`` measures them on the device (gpu_mul_time_config, CUDA
  events, median of a few runs) -- the exhaustive tuner, which is both the
  fallback and the yardstick of the learned model (its regret);
* ``CostModel`` is the learned part: an MLP (16 inputs -> 3 x 64 -> 1, fp32,
  the library's own CUDA training and inference kernels) that predicts the
  log device time of (request, configuration); ``choose`` takes the argmin
  over a request's candidates in one batched forward pass;
* ``regret`` compares chosen configurations with the exhaustive optimum.

A request is (kind, an, bn, aw, bw): kind 0 is an mpn product of an x bn
limbs (aw = bw = 1), kind 1 an integer-polynomial product of an x bn
coefficients of aw and bw limbs.
"""
import math

import numpy as np

from . import (MulConfig, ROUTE_BASECASE, ROUTE_NTT, GpuFftSmallError, Mlp, resolve_config)

BASECASE_MAX = 1024
N_FEATURES = 16


def _req(r):
    kind, an, bn = r[0], int(r[1]), int(r[2])
    aw = int(r[3]) if len(r) > 3 else 1
    bw = int(r[4]) if len(r) > 4 else 1
    return kind, an, bn, aw, bw


def default_config(r):
    """The fixed rule (the method without the model): transform route, fewest
    primes, shortest transform, longest rows."""
    kind, an, bn, aw, bw = _req(r)
    return resolve_config(kind, an, bn, None, aw, bw)


def candidates(r):
    """All configurations the tuner considers for request r (resolved)."""
    kind, an, bn, aw, bw = _req(r)
    base = default_config(r)
    out = []
    if kind == 0 and min(an, bn) <= BASECASE_MAX:
        out.append(MulConfig(ROUTE_BASECASE, 0, 0, 0))
    for dnp in (0, 1):
        for dm in (0, 1):
            for dc in (0, 1, 2, 3):
                np_, logM = base.np + dnp, base.logM + dm
                logC = min(logM, 14) - dc
                c = MulConfig(ROUTE_NTT, np_, logM, logC)
                try:
                    out.append(resolve_config(kind, an, bn, c, aw, bw))
                except GpuFftSmallError:
                    pass
    return out


def features(r, cfg):
    """Input vector of the cost model for request r under configuration cfg."""
    kind, an, bn, aw, bw = _req(r)
    base = default_config(r)
    pts = (an + bn - 1) * (1 if kind == 0 else aw + bw - 1)
    bc = cfg.route == ROUTE_BASECASE
    f = np.zeros(N_FEATURES, dtype=np.float32)
    f[0] = kind
    f[1] = math.log2(an) / 22
    f[2] = math.log2(bn) / 22
    f[3] = math.log2(an / bn) / 6
    f[4] = math.log2(aw) / 7
    f[5] = math.log2(bw) / 7
    f[6] = math.log2(pts) / 25
    f[7] = math.log2(min(an, bn)) / 22
    f[8] = 1.0 if bc else 0.0
    if bc:
        f[9] = math.log2(an * bn) / 44
    else:
        f[10] = cfg.np - base.np
        f[11] = cfg.logM - base.logM
        f[12] = cfg.logM / 25
        f[13] = cfg.logC / 14
        f[14] = (cfg.logM - cfg.logC) / 11
        f[15] = math.log2(pts) / 25 - cfg.logM / 25
    return f


def batch_copies(an, bn):
    """Products per timing batch in batched mode: about 2^22 limbs of operands,
    between 1 and 64 products."""
    return max(1, min(64, (1 << 22) // (an + bn)))


class Autotuner:
    """Exhaustive measurement of a request's candidates on the device.

    batched=False times a product alone (gpu_mul_time_config); batched=True
    times mpn products as the marginal cost inside a batch of identical
    products (gpu_mpn_mul_time_batched), the cost that matters when requests
    are executed as planned batches."""

    def __init__(self, ctx, reps=3, batched=False):
        self.ctx = ctx
        self.reps = reps
        self.batched = batched
        self.cache = {}

    def time(self, r, cfg):
        kind, an, bn, aw, bw = _req(r)
        key = (kind, an, bn, aw, bw, cfg.key())
        if key not in self.cache:
            if self.batched and kind == 0:
                self.cache[key] = self.ctx.time_batched(an, bn, cfg, batch_copies(an, bn), self.reps)
            else:
                self.cache[key] = self.ctx.time_config(kind, an, bn, cfg, aw, bw, self.reps)
        return self.cache[key]

    def table(self, r):
        """[(cfg, ms)] for every candidate of r."""
        return [(c, self.time(r, c)) for c in candidates(r)]

    def best(self, r):
        return min(self.table(r), key=lambda x: x[1])


def dataset(tuner, reqs):
    """Training rows (features, log ms) from the tuner's measurements."""
    X, t = [], []
    for r in reqs:
        for c, ms in tuner.table(r):
            X.append(features(r, c))
            t.append(math.log(max(ms, 1e-4)))
    return np.array(X, dtype=np.float32), np.array(t, dtype=np.float32)


class CostModel:
    """Learned schedule: predicts log time, chooses the argmin candidate.

    margin > 0 makes the choice conservative: the model's argmin replaces the
    fixed rule's configuration only when it predicts at least that relative
    saving (a prediction error of a few percent otherwise trades the rule's
    configuration for one that is no faster)."""

    def __init__(self, seed=1, margin=0.0):
        self.net = Mlp(N_FEATURES, seed)
        self.margin = margin

    def fit(self, X, t, epochs=300, batch=256, lr=2e-3, seed=7):
        return self.net.train(X, t, epochs=epochs, batch=batch, lr=lr, seed=seed)

    def choose(self, reqs):
        """Chosen configuration per request (one batched forward pass)."""
        cands = [candidates(r) for r in reqs]
        rows = [features(r, c) for r, cs in zip(reqs, cands) for c in cs]
        pred = self.net.predict(np.array(rows, dtype=np.float32))
        keep = math.log(1.0 - self.margin) if self.margin > 0 else 0.0
        out, k = [], 0
        for r, cs in zip(reqs, cands):
            p = pred[k:k + len(cs)]
            i = int(np.argmin(p))
            if self.margin > 0:
                dk = default_config(r).key()
                j = next((n for n, c in enumerate(cs) if c.key() == dk), None)
                if j is not None and p[i] - p[j] > keep:
                    i = j
            out.append(cs[i])
            k += len(cs)
        return out


def regret(tuner, reqs, chosen):
    """Per-request regret t(chosen) / t(best) - 1 against the exhaustive tuner,
    and the total-time ratios of the default rule and of the choices."""
    reg, t_best, t_chosen, t_default = [], 0.0, 0.0, 0.0
    for r, c in zip(reqs, chosen):
        _, b = tuner.best(r)
        tc = tuner.time(r, c)
        td = tuner.time(r, default_config(r))
        reg.append(tc / b - 1.0)
        t_best += b
        t_chosen += tc
        t_default += td
    reg = np.array(reg)
    return {
        "requests": len(reqs),
        "mean_regret": float(reg.mean()), "median_regret": float(np.median(reg)),
        "p90_regret": float(np.quantile(reg, 0.9)), "max_regret": float(reg.max()),
        "total_ms_best": t_best, "total_ms_chosen": t_chosen, "total_ms_default": t_default,
        "gain_over_default": t_default / t_chosen,
        "total_regret": t_chosen / t_best - 1.0,
    }
