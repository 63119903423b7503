"""The learned schedule: the cost model's CUDA kernels against the NumPy
oracle, training, and the trained model against the exhaustive autotuner and
against the fixed rule it replaces.  The model only picks among valid
configurations, so results stay exact whatever it predicts (the config tests
check every candidate)."""
import numpy as np
import pytest

import flint_b200 as FB
from flint_b200 import tuner
from flint_b200.workload import request_stream
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 31, 32, 33, 500])
def test_forward_and_gradient_match_oracle(n):
    rng = np.random.default_rng(n)
    net = FB.Mlp(16, seed=5)
    P = net.params().astype(np.float64)
    X = rng.normal(0, 1, (n, 16)).astype(np.float32)
    t = rng.normal(0, 1, n).astype(np.float32)
    y_ref, _ = mlp_ref.forward(P, X)
    y = net.predict(X)
    assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4)
    g, loss = net.gradient(X, t)
    g_ref = mlp_ref.gradient(P, X, t)
    assert abs(loss - mlp_ref.loss(P, X, t)) <= 1e-4 * max(1.0, abs(loss))
    # fp32 kernels against the float64 oracle: relative to the gradient's scale
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale + 1e-7
    # deterministic: the same call gives the same bits
    g2, _ = net.gradient(X, t)
    assert (g2 == g).all()
    net.close()


def test_parameters_round_trip_and_init_is_seeded():
    a, b, c = FB.Mlp(16, seed=1), FB.Mlp(16, seed=1), FB.Mlp(16, seed=2)
    assert (a.params() == b.params()).all() and not (a.params() == c.params()).all()
    p = np.arange(a.nparams, dtype=np.float32) * 1e-4
    a.set_params(p)
    assert (a.params() == p).all()
    assert a.nparams == mlp_ref.offsets(16)["total"]


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(0)
    X = rng.uniform(-1, 1, (2048, 16)).astype(np.float32)
    t = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2).astype(np.float32)
    net = FB.Mlp(16, seed=3)
    _, loss0 = net.gradient(X, t)
    loss = net.train(X, t, epochs=150, batch=128, lr=2e-3)
    assert loss < 0.05 * loss0
    # the training loop's own result equals the oracle's loss of the final parameters
    assert abs(loss - mlp_ref.loss(net.params(), X, t)) <= 1e-3 * max(loss, 1e-3)


def test_learned_schedule_regret_and_gain(ctx):
    """Train on autotuner timings of a request sample, evaluate on held-out
    requests: regret against the exhaustive tuner, gain over the fixed rule."""
    reqs = request_stream(2024, 220, mpn_log=(6.0, 18.0), fmpz_len_log=(8.0, 12.0),
                          fmpz_bits=(64, 1024))
    train, test = reqs[:160], reqs[160:]
    tun = tuner.Autotuner(ctx, reps=3)
    X, t = tuner.dataset(tun, train)
    model = tuner.CostModel(seed=11)
    model.fit(X, t, epochs=400, batch=256, lr=2e-3)
    chosen = model.choose(test)
    rep = tuner.regret(tun, test, chosen)
    print("learned schedule:", rep)
    assert rep["gain_over_default"] > 1.0
    assert rep["total_regret"] < 0.25


def test_learned_schedule_gain_over_reference_rule(ctx):
    """The method without the model, as the reference makes it: its own
    profile choice (mpn_ctx_best_profile, ported to host C as
    gpu_mul_reference_rule).  On held-out requests that include products
    above 2^19 coefficients (where 3 2^k lengths and split products apply),
    the trained model takes less total time than that rule."""
    reqs = request_stream(2031, 200, mpn_log=(10.0, 21.0), mpn_ratio_log=(0.0, 5.0),
                          fmpz_len_log=(8.0, 12.0), fmpz_bits=(64, 1024))
    train, test = reqs[:150], reqs[150:]
    tun = tuner.Autotuner(ctx, reps=3)
    X, t = tuner.dataset(tun, train)
    model = tuner.CostModel(seed=13)
    model.fit(X, t, epochs=400, batch=256, lr=2e-3)
    rep = tuner.regret(tun, test, model.choose(test))
    print("learned vs reference rule:", rep)
    assert rep["gain_over_reference_rule"] > 1.0
    assert rep["total_regret"] < 0.25
