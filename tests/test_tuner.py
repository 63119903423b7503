"""Host logic of the autotuner and the learned schedule (no GPU needed):
candidate enumeration, configuration validation, feature encoding and the
request-stream generator."""
import math

import numpy as np
import pytest

import flint_b200 as FB
from flint_b200 import tuner
from flint_b200.workload import request_stream


REQS = [(0, 1, 1), (0, 64, 64), (0, 1000, 3), (0, 3000, 2000), (0, 1 << 14, 1 << 14), (0, 40000, 30000),
        (0, 1 << 20, 1 << 14), (0, 1 << 22, 1 << 22),
        (1, 256, 300, 2, 2), (1, 1 << 16, 1 << 16, 65, 65), (1, 5000, 40, 10, 3)]


@pytest.mark.parametrize("r", REQS)
def test_candidates_are_valid_and_include_default(r):
    cs = tuner.candidates(r)
    keys = [c.key() for c in cs]
    assert len(set(keys)) == len(keys)
    assert tuner.default_config(r).key() in keys
    kind, an, bn = r[:3]
    has_bc = any(c.route == FB.ROUTE_BASECASE for c in cs)
    assert has_bc == (kind == 0 and min(an, bn) <= tuner.BASECASE_MAX)
    has_bc_batch = any(c.route == FB.ROUTE_BASECASE for c in tuner.candidates(r, flags=False))
    assert has_bc_batch == (kind == 0 and min(an, bn) <= tuner.BASECASE_BATCH_MAX)
    for c in cs:
        if c.route == FB.ROUTE_NTT and c.flags & FB.FLAG_THREE:
            assert c.logC == 13                  # 3 2^k-point transforms: 2^13-point rows
        elif c.route == FB.ROUTE_NTT:
            assert max(5, c.logM - 11) <= c.logC <= min(c.logM, 14)
            assert c.logM >= 14 or c.logM - c.logC <= 4
        f = tuner.features(r, c)
        assert f.shape == (tuner.N_FEATURES,) and np.isfinite(f).all()


def test_invalid_configs_are_rejected():
    with pytest.raises(FB.GpuFftSmallError):
        FB.resolve_config(0, 5000, 5000, FB.MulConfig(FB.ROUTE_BASECASE, 0, 0, 0))   # > 4096
    assert FB.resolve_config(0, 4096, 10 ** 6, FB.MulConfig(FB.ROUTE_BASECASE, 0, 0, 0)).route == FB.ROUTE_BASECASE
    with pytest.raises(FB.GpuFftSmallError):
        FB.resolve_config(0, 100, 100, FB.MulConfig(FB.ROUTE_NTT, 4, 0, 0))          # too few primes
    with pytest.raises(FB.GpuFftSmallError):
        FB.resolve_config(0, 100, 100, FB.MulConfig(FB.ROUTE_NTT, 0, 7, 0))          # too short
    with pytest.raises(FB.GpuFftSmallError):
        FB.resolve_config(0, 1 << 20, 1, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 8))        # rows too short
    with pytest.raises(FB.GpuFftSmallError):
        FB.resolve_config(1, 10, 10, FB.MulConfig(FB.ROUTE_BASECASE, 0, 0, 0), 2, 2)
    with pytest.raises(FB.GpuFftSmallError):                                         # 64 columns of
        FB.resolve_config(0, 600, 500, FB.MulConfig(FB.ROUTE_NTT, 0, 11, 5))          # 32 below 2^14
    assert FB.resolve_config(0, 600, 500, FB.MulConfig(FB.ROUTE_NTT, 0, 11, 7)).logC == 7
    c = FB.resolve_config(0, 1 << 20, 1 << 20)
    assert c.key() == (FB.ROUTE_NTT, 5, 21, 13, 0)       # 2^13-point rows from 2^15 to 2^24
    assert FB.resolve_config(0, 1 << 24, 1 << 24).key() == (FB.ROUTE_NTT, 5, 25, 14, 0)
    assert FB.resolve_config(0, 5000, 3000).key() == (FB.ROUTE_NTT, 5, 13, 13, 0)


def test_request_stream_shape():
    rs = request_stream(11, 4000)
    mpn = [r for r in rs if r[0] == 0]
    fz = [r for r in rs if r[0] == 1]
    assert abs(len(mpn) - len(fz)) < 300
    la = np.log2([r[1] for r in mpn])
    assert 6 - 1e-9 <= la.min() and la.max() <= 22 + 1e-9
    # bn = round(an / 2^V) >= 1: rounding moves the ratio by at most a factor 1.5
    ratios = np.log2([r[1] / r[2] for r in mpn])
    assert ratios.min() >= -0.6 and ratios.max() <= 6.6
    ws = [r[3] for r in fz]
    assert min(ws) >= 2 and max(ws) <= 65
    assert all(2 ** 8 - 1 <= r[1] <= 2 ** 16 + 1 and 2 ** 8 - 1 <= r[2] <= 2 ** 16 + 1 for r in fz)


def test_configuration_flags():
    """THREE and SPLIT resolve where the product allows them and are refused
    elsewhere; the reference rule (host-C port of mpn_ctx_best_profile) takes
    the 3 2^k length where it fits."""
    three = FB.resolve_config(0, 3 << 22, 3 << 22, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_THREE))
    assert three.key() == (FB.ROUTE_NTT, 5, 25, 13, FB.FLAG_THREE)
    assert FB.resolve_config(0, 1 << 24, 1 << 20,
                             FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_SPLIT)).flags == FB.FLAG_SPLIT
    for an, bn, fl in [(1 << 24, 1 << 24, FB.FLAG_THREE),        # L = 2^25 - 1: no 3 2^23 fit
                       (1000, 1000, FB.FLAG_THREE),               # below the radix-3 kernels
                       (3 << 22, 3 << 22, FB.FLAG_THREE | FB.FLAG_SPLIT),
                       (1 << 20, 1 << 20, FB.FLAG_SPLIT),         # balanced: does not split
                       (1 << 16, 1 << 16, FB.FLAG_ROWS16 | FB.FLAG_ROWS32),
                       (100, 100, FB.FLAG_ROWS16),                # rows of 2^8 points
                       (1 << 24, 1 << 20, FB.FLAG_ROWS16 | FB.FLAG_SPLIT),
                       (100, 100, 64)]:                           # unknown flag
        with pytest.raises(FB.GpuFftSmallError):
            FB.resolve_config(0, an, bn, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, fl))
    with pytest.raises(FB.GpuFftSmallError):                     # six primes: no cube roots
        FB.resolve_config(0, 3 << 22, 3 << 22, FB.MulConfig(FB.ROUTE_NTT, 6, 0, 0, FB.FLAG_THREE))
    with pytest.raises(FB.GpuFftSmallError):                     # too short for the radix-3 kernels
        FB.resolve_config(1, 300, 200, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_THREE), 2, 2)
    # integer polynomials: a chunk product of 8999 x 63 positions fits 3 2^18
    fz3 = FB.resolve_config(1, 4500, 4500, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_THREE), 32, 32)
    assert fz3.key() == (FB.ROUTE_NTT, 5, 20, 13, FB.FLAG_THREE)
    for fl in (FB.FLAG_SPLIT, FB.FLAG_ROWS16):                  # the only flag they take is THREE
        with pytest.raises(FB.GpuFftSmallError):
            FB.resolve_config(1, 4500, 4500, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, fl), 32, 32)
    assert tuner.reference_rule((1, 4500, 4500, 32, 32)).flags == FB.FLAG_THREE
    for fl in (FB.FLAG_ROWS16, FB.FLAG_ROWS32):                  # row pass width: kept as given
        assert FB.resolve_config(0, 1 << 16, 1 << 16, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, fl)).flags == fl
    assert tuner.reference_rule((0, 3 << 22, 3 << 22)).flags == FB.FLAG_THREE
    assert tuner.reference_rule((0, 1 << 24, 1 << 24)).key() == (FB.ROUTE_NTT, 5, 25, 14, 0)
    assert tuner.reference_rule((1, 300, 200, 3, 3)).flags == 0
    keys = [c.key() for c in tuner.candidates((0, 3 << 22, 3 << 22))]
    assert (FB.ROUTE_NTT, 5, 25, 13, FB.FLAG_THREE) in keys
    assert all(c.flags == 0 for c in tuner.candidates((0, 3 << 22, 3 << 22), flags=False))


def test_min_class_falls_back_to_rule():
    """A learned choice that leaves a request in a batch class of fewer than
    min_class products falls back to the fixed rule; per-instance
    configurations (flags) are kept."""
    reqs = [(0, 1 << 12, 1 << 12)] * 20 + [(0, 1 << 14, 1 << 13)] * 3 + [(0, 3 << 20, 3 << 20)]
    alt = FB.resolve_config(0, 1 << 12, 1 << 12, FB.MulConfig(FB.ROUTE_NTT, 6, 0, 0))
    alt2 = FB.resolve_config(0, 1 << 14, 1 << 13, FB.MulConfig(FB.ROUTE_NTT, 6, 0, 0))
    three = FB.resolve_config(0, 3 << 20, 3 << 20, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_THREE))
    m = tuner.CostModel.__new__(tuner.CostModel)
    m._choose = lambda rs, flags: [alt] * 20 + [alt2] * 3 + [three]
    out = m.choose(reqs, min_class=16)
    assert all(c.key() == alt.key() for c in out[:20])                     # a class of 20: kept
    assert all(c.key() == tuner.default_config(reqs[20]).key() for c in out[20:23])   # 3: rule
    assert out[23].key() == three.key()                                      # per instance: kept
    assert [c.key() for c in m.choose(reqs)] == [c.key() for c in [alt] * 20 + [alt2] * 3 + [three]]


class _FakeNet:
    """Predicts log time from the row-length feature alone: scale * logC/14."""

    def __init__(self, scale):
        self.scale = scale

    def predict(self, X):
        return (self.scale * X[:, 13]).astype(np.float32)


def test_choose_classes_moves_whole_classes():
    """Planned-batch choice per class of the fixed rule: every request of a
    class moves to the configuration of least predicted total, and only when
    that total saves at least the margin."""
    reqs = [(0, 100000 + 37 * k, 60000 + 11 * k) for k in range(12)] + [(0, 3000, 2000)] * 5
    m = tuner.CostModel.__new__(tuner.CostModel)
    m.margin = 0.10
    m.net = _FakeNet(-3.0)                 # longer rows predicted faster
    out = m.choose_classes(reqs, margin=0.05)
    for r, c in zip(reqs, out):
        # the predicted-fastest candidate: the longest rows on offer
        assert c.logC == max(x.logC for x in tuner.candidates(r, flags=False) if x.route == FB.ROUTE_NTT)
    # each class of the rule moves whole: one configuration per class
    assert len({c.key() for c in out[:12]}) == 1 and len({c.key() for c in out[12:]}) == 1
    m.net = _FakeNet(-0.01)                # a saving below the margin: the rule stays
    assert [c.key() for c in m.choose_classes(reqs, margin=0.05)] == \
        [tuner.default_config(r).key() for r in reqs]


class _FakeFlagNet:
    """Predicts log time: `three` for THREE configurations, 0 otherwise."""

    def __init__(self, three):
        self.three = three

    def predict(self, X):
        return (self.three * X[:, 16]).astype(np.float32)


def test_choose_stream_flag_override():
    """In a stream, an mpn request moves to a flagged configuration only where
    the predicted saving over its class's choice reaches the margin;
    integer-polynomial requests take no flags."""
    reqs = [(0, 3 << 20, 3 << 20), (0, 1000, 900), (1, 300, 200, 2, 2), (0, 3 << 10, 3 << 10)]
    m = tuner.CostModel.__new__(tuner.CostModel)
    m.margin = 0.10
    m.net = _FakeFlagNet(-0.3)             # THREE predicted 26% faster
    out = m.choose_stream(reqs, class_margin=0.05)
    assert out[0].flags == FB.FLAG_THREE
    assert out[1].key() == tuner.default_config(reqs[1]).key() and out[2].flags == 0
    assert out[3].flags == 0               # a small product stays in the batch
    m.net = _FakeFlagNet(-0.05)            # 5% faster: below the margin
    assert m.choose_stream(reqs, class_margin=0.05)[0].flags == 0
