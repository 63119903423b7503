"""Autotuner and learned schedule for the multiplication path.

The reference picks its transform parameters with a fixed heuristic
(mpn_ctx_best_profile, src/fft_small/mpn_mul.c:1248-1340) and routes small
operands to GMP by size thresholds (src/mpn_extras/mul.c:52-75).  Here the
choice per request is a gpu_mul_config:

    route   transform or basecase (schoolbook, shorter operand <= 1024 limbs)
    np      prime count (the minimum, or one more)
    logM    transform length (the minimum, or twice it)
    logC    four-step row length (the longest allowed, or 2x / 4x / 8x shorter)
    flags   THREE: a 3 2^(logM-2)-point transform (radix-3 column stage) where
            the product fits it; SPLIT: chunks of the long operand against one
            transform of the short one (unbalanced products)

Every valid configuration gives the same exact product; only time differs.

* ``candidates`` enumerates the configurations of a request;
* ``Autotuner`` measures them on the device (gpu_mul_time_config, CUDA
  events, median of a few runs) -- the exhaustive tuner, which is both the
  fallback and the yardstick of the learned model (its regret);
* ``CostModel`` is the learned part: an MLP (16 inputs -> 3 x 64 -> 1, fp32,
  the library's own CUDA training and inference kernels) that predicts the
  log device time of (request, configuration); ``choose`` takes the argmin
  over a request's candidates in one batched forward pass;
* ``regret`` compares chosen configurations with the exhaustive optimum;
* ``reference_rule`` is the reference's own profile choice
  (mpn_ctx_best_profile, src/fft_small/mpn_mul.c:1248-1340) ported to this
  configuration space: the least score (1 - ratio/4) np depth L_t over single
  transforms, L_t the transform's points (truncated where a 3 2^k length
  fits), depth = ceil(log2 L_t), ratio = L_t / 2^depth.

A request is (kind, an, bn, aw, bw): kind 0 is an mpn product of an x bn
limbs (aw = bw = 1), kind 1 an integer-polynomial product of an x bn
coefficients of aw and bw limbs.
"""
import math

import numpy as np

from . import (FLAG_ROWS16, FLAG_ROWS32, FLAG_SPLIT, FLAG_THREE, MulConfig, ROUTE_BASECASE, ROUTE_NTT,
               GpuFftSmallError, Mlp, resolve_config)
from . import reference_rule as _reference_rule

BASECASE_MAX = 4096          # short operand of the basecase route, single products
BASECASE_BATCH_MAX = 1024    # ... in a planned batch
N_FEATURES = 26


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


def candidates(r, flags=True):
    """All configurations the tuner considers for request r (resolved).
    flags=False leaves out the flagged configurations (THREE, SPLIT, the row
    pass's width) and keeps the basecase route to the batch limit: planned
    batches run every class with plain transforms."""
    kind, an, bn, aw, bw = _req(r)
    base = default_config(r)
    out = []
    if kind == 0 and min(an, bn) <= (BASECASE_MAX if flags else BASECASE_BATCH_MAX):
        out.append(MulConfig(ROUTE_BASECASE, 0, 0, 0))
    seen = set()
    for dnp in (0, 1):
        for dm in (0, 1):
            np_, logM = base.np + dnp, base.logM + dm
            # the rule's row length for this length, then the longest rows
            # and 2x / 4x / 8x shorter
            try:
                rule_logC = [resolve_config(kind, an, bn, MulConfig(ROUTE_NTT, np_, logM, 0), aw, bw).logC]
            except GpuFftSmallError:
                rule_logC = []
            for logC in rule_logC + [min(logM, 14) - dc for dc in (0, 1, 2, 3)]:
                if (np_, logM, logC) in seen:
                    continue
                seen.add((np_, logM, logC))
                try:
                    out.append(resolve_config(kind, an, bn, MulConfig(ROUTE_NTT, np_, logM, logC), aw, bw))
                except GpuFftSmallError:
                    pass
    if flags:
        # 3 2^k lengths for both kinds; splitting for mpn products only
        for fl in ((FLAG_THREE, FLAG_SPLIT) if kind == 0 else (FLAG_THREE,)):
            try:
                out.append(resolve_config(kind, an, bn, MulConfig(ROUTE_NTT, base.np, base.logM, 0, fl), aw, bw))
            except GpuFftSmallError:
                pass
    if flags and kind == 0:
        # the row pass at 16 and at 32 points per thread (the launch rule
        # picks one of them by the warps the launch has)
        for fl in (FLAG_ROWS16, FLAG_ROWS32):
            try:
                out.append(resolve_config(kind, an, bn, MulConfig(ROUTE_NTT, base.np, base.logM, base.logC, fl)))
            except GpuFftSmallError:
                pass
    return out


def transform_points(cfg):
    """Points of the transform a resolved configuration runs (one transform;
    a split product's chunks are not counted)."""
    if cfg.route != ROUTE_NTT:
        return 0
    return 3 << (cfg.logM - 2) if cfg.flags & FLAG_THREE else 1 << cfg.logM


def reference_rule(r):
    """The reference's profile choice (mpn_ctx_best_profile,
    src/fft_small/mpn_mul.c:1248-1340) in this configuration space, from the
    library's host-C port (gpu_mul_reference_rule): the least score
    (1 - ratio/4) np depth L_t over single transforms with the longest rows,
    L_t the transform's points (3 2^k where the product fits), depth =
    ceil(log2 L_t), ratio = L_t / 2^depth."""
    kind, an, bn, aw, bw = _req(r)
    return _reference_rule(kind, an, bn, aw, bw)


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
        lt = math.log2(transform_points(cfg))
        f[10] = cfg.np - base.np
        f[11] = cfg.logM - base.logM
        f[12] = lt / 25
        f[13] = cfg.logC / 14
        f[14] = (lt - cfg.logC) / 11
        f[15] = math.log2(pts) / 25 - lt / 25
        f[16] = 1.0 if cfg.flags & FLAG_THREE else 0.0
        f[17] = 1.0 if cfg.flags & FLAG_SPLIT else 0.0
        f[18] = 1.0 if cfg.flags & FLAG_ROWS16 else 0.0
        f[19] = 1.0 if cfg.flags & FLAG_ROWS32 else 0.0
        # the column length selects the kernel variants (no column pass, one
        # thread per short column, 32-point columns in registers, strided
        # passes, constant-stride instances): one indicator per group
        logR = round(lt) - cfg.logC if not cfg.flags & FLAG_THREE else 0
        for i, (lo, hi) in enumerate(((0, 0), (1, 4), (5, 5), (6, 8), (9, 10), (11, 11))):
            f[20 + i] = 1.0 if lo <= logR <= hi else 0.0
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
            # planned batches take no flags, and basecase products only up to
            # a short operand of BASECASE_BATCH_MAX limbs: other
            # configurations run per instance, so they are timed alone
            batchable = not cfg.flags and not (cfg.route == ROUTE_BASECASE and min(an, bn) > BASECASE_BATCH_MAX)
            if self.batched and kind == 0 and batchable:
                self.cache[key] = self.ctx.time_batched(an, bn, cfg, batch_copies(an, bn), self.reps)
            else:
                self.cache[key] = self.ctx.time_config(kind, an, bn, cfg, aw, bw, self.reps)
        return self.cache[key]

    def table(self, r, flags=True):
        """[(cfg, ms)] for every candidate of r."""
        return [(c, self.time(r, c)) for c in candidates(r, flags)]

    def best(self, r, flags=True):
        return min(self.table(r, flags), key=lambda x: x[1])


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

    def choose_classes(self, reqs, margin=0.05, margin_fmpz=None):
        """Configurations for requests run as one planned batch (plain
        transforms), decided per class: the requests whose fixed-rule
        configuration is the same form a class, and the class moves as a
        whole to the configuration whose predicted total time over its
        requests is least, where that total is at least `margin` below the
        rule's.  Summing over a class averages out the model's per-request
        error, and moving a class whole keeps the batch's classes as
        populated as the rule's.  Integer-polynomial classes (products
        that run one after another, never batched) take margin_fmpz
        (default: the model's decision margin)."""
        if margin_fmpz is None:
            margin_fmpz = self.margin
        cands = [candidates(r, False) for r in reqs]
        rows = [features(r, c) for r, cs in zip(reqs, cands) for c in cs]
        pred = np.exp(self.net.predict(np.array(rows, dtype=np.float32)).astype(np.float64))
        groups = {}
        k = 0
        for n, (r, cs) in enumerate(zip(reqs, cands)):
            groups.setdefault((r[0],) + default_config(r).key(), []).append(
                (n, {c.key(): (c, pred[k + i]) for i, c in enumerate(cs)}))
            k += len(cs)
        out = [default_config(r) for r in reqs]
        for gk, members in groups.items():
            dk = gk[1:]
            common = set(members[0][1])
            for _, m in members[1:]:
                common &= set(m)
            if dk not in common:
                continue
            tot = {key: sum(m[key][1] for _, m in members) for key in common}
            best = min(tot, key=tot.get)
            if tot[best] <= (1.0 - (margin if gk[0] == 0 else margin_fmpz)) * tot[dk]:
                for n, m in members:
                    out[n] = m[best][0]
        return out

    def choose_stream(self, reqs, class_margin=0.05, flag_margin=None, alone_points=1 << 20):
        """Configurations for a mixed request stream: plain transforms chosen
        per class of the fixed rule (choose_classes; mpn requests then share
        planned batches as under the rule), and a request moved to a THREE
        (3 2^k-point) or, for mpn, SPLIT configuration only where the model
        predicts at least flag_margin (default: the model's decision margin)
        below the class choice -- for an mpn request (which then runs alone)
        also only where its transform has at least `alone_points` points (a
        product that fills the GPU by itself, so leaving the batch costs
        nothing).  The row-pass width flags stay with the launch rule."""
        if flag_margin is None:
            flag_margin = self.margin
        out = self.choose_classes(reqs, class_margin)
        # integer-polynomial products run alone anyway: any size may move
        idx = [n for n, r in enumerate(reqs) if r[0] == 1 or transform_points(out[n]) >= alone_points]
        flagged = [[c for c in candidates(reqs[n], True) if c.flags & (FLAG_THREE | FLAG_SPLIT)] for n in idx]
        rows, own = [], []
        for n, fl in zip(idx, flagged):
            if fl:
                rows.append(features(reqs[n], out[n]))
                rows += [features(reqs[n], c) for c in fl]
                own.append((n, fl))
        if not rows:
            return out
        pred = self.net.predict(np.array(rows, dtype=np.float32))
        keep = math.log(1.0 - flag_margin)
        k = 0
        for n, fl in own:
            base, p = pred[k], pred[k + 1:k + 1 + len(fl)]
            i = int(np.argmin(p))
            if p[i] - base <= keep:
                out[n] = fl[i]
            k += 1 + len(fl)
        return out

    def choose(self, reqs, flags=True, min_class=0):
        """Chosen configuration per request (one batched forward pass);
        flags=False chooses among plain transforms only (planned batches).

        min_class > 0: the requests are run as planned batches, whose
        products share launches by configuration class; the model is trained
        on the marginal cost of a product inside a populated class, so a
        choice that leaves a request in a class of fewer than min_class
        products of this request list (where that cost does not hold) falls
        back to the fixed rule.  Configurations that run per instance
        (flags, a basecase product beyond a batch's limit) are exempt."""
        out = self._choose(reqs, flags)
        if min_class > 0:
            for _ in range(2):
                count = {}
                for r, c in zip(reqs, out):
                    k = _class_key(r, c)
                    if k is not None:
                        count[k] = count.get(k, 0) + 1
                out = [default_config(r) if (k := _class_key(r, c)) is not None and count[k] < min_class
                       and c.key() != default_config(r).key() else c for r, c in zip(reqs, out)]
        return out

    def _choose(self, reqs, flags):
        cands = [candidates(r, flags) for r in reqs]
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


def _class_key(r, c):
    """The planned-batch class of mpn request r under configuration c (None
    for requests that run per instance, and for integer polynomials)."""
    kind, an, bn, _, _ = _req(r)
    if kind != 0 or c.flags or (c.route == ROUTE_BASECASE and min(an, bn) > BASECASE_BATCH_MAX):
        return None
    return (c.route, c.np, c.logM, c.logC)


def regret(tuner, reqs, chosen, flags=True):
    """Per-request regret t(chosen) / t(best) - 1 against the exhaustive tuner
    (over the same candidate space, flags as for candidates), and the
    total-time ratios of the fixed rule, of the reference's rule
    (reference_rule; flags=False keeps it to plain transforms) and of the
    choices."""
    reg, t_best, t_chosen, t_default, t_ref = [], 0.0, 0.0, 0.0, 0.0
    for r, c in zip(reqs, chosen):
        _, b = tuner.best(r, flags)
        tc = tuner.time(r, c)
        td = tuner.time(r, default_config(r))
        rc = reference_rule(r) if flags else default_config(r)
        tr = tuner.time(r, rc)
        reg.append(tc / b - 1.0)
        t_best += b
        t_chosen += tc
        t_default += td
        t_ref += tr
    reg = np.array(reg)
    return {
        "requests": len(reqs),
        "mean_regret": float(reg.mean()), "median_regret": float(np.median(reg)),
        "p90_regret": float(np.quantile(reg, 0.9)), "max_regret": float(reg.max()),
        "total_ms_best": t_best, "total_ms_chosen": t_chosen, "total_ms_default": t_default,
        "total_ms_reference_rule": t_ref,
        "gain_over_default": t_default / t_chosen,
        "gain_over_reference_rule": t_ref / t_chosen,
        "total_regret": t_chosen / t_best - 1.0,
    }
