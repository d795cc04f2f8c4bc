"""GPU: the learned tuner's MLP kernels and proposals.

* forward pass and gradients of the device kernels vs the numpy float64
  oracle (oracle/mlp_oracle.py), FP32 tolerances stated below;
* full-batch Adam training on the device reduces the loss;
* proposals pass the endpoint-coverage check or fall back to the reference
  heuristic; every proposal gives the exact M(X);
* with the committed trained weights the proposal beats the reference's
  default heuristic at X = 3*10^16 (the gain of the learned part).
"""
import json
import os

import numpy as np
import pytest

import dr_b200
import mlp_oracle as mo

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(dr_b200.__file__), "tuner_weights.json")
FWD_TOL = 1e-4   # |y_gpu - y_oracle| <= FWD_TOL * (1 + |y|)   (FP32 vs float64)
GRAD_TOL = 2e-3  # |g_gpu - g_oracle| <= GRAD_TOL * max|g_oracle|


def test_forward_matches_oracle(engine):
    rng = np.random.default_rng(3)
    mlp = dr_b200.MLP(engine, seed=7)
    P = mlp.get_weights().astype(np.float64)
    x = rng.normal(0, 1, (33, 4)).astype(np.float32)
    y = mlp.forward(x)
    yo, _ = mo.forward(P, x.astype(np.float64))
    assert np.all(np.abs(y - yo) <= FWD_TOL * (1 + np.abs(yo)))


def test_gradients_match_oracle(engine):
    rng = np.random.default_rng(4)
    mlp = dr_b200.MLP(engine, seed=11)
    w = rng.normal(0, 0.2, mlp.n_params).astype(np.float32)
    mlp.set_weights(w)
    x = rng.normal(0, 1, (50, 4)).astype(np.float32)
    t = rng.normal(0, 1, (50, 4)).astype(np.float32)
    g, loss = mlp.grad(x, t)
    go = mo.grad(w.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    lo = mo.loss(w.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lo) <= 1e-4 * (1 + abs(lo))
    assert np.max(np.abs(g - go)) <= GRAD_TOL * np.max(np.abs(go))


def test_training_reduces_loss(engine):
    rng = np.random.default_rng(5)
    mlp = dr_b200.MLP(engine, seed=13)
    x = rng.uniform(-1, 1, (200, 4)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]), x[:, 1] * x[:, 2], np.abs(x[:, 3]), x[:, 0] - x[:, 3]], 1).astype(np.float32)
    _, l0 = mlp.grad(x, t)
    l1 = mlp.train(x, t, 1500, 3e-3)
    assert l1 < 0.1 * l0, (l0, l1)


def test_proposal_and_fallback(engine):
    mlp = dr_b200.MLP(engine, seed=17)
    for X in (10**11, 10**14, 10**16):
        p, fb = mlp.propose(X, 160 * 2**30)
        assert dr_b200.check_params(X, p) == 0
        assert engine.mertens(X, p).M == {10**11: -87856, 10**14: -875575, 10**16: -3195437}[X]
    # a budget no table fits: the proposal fails the check and the reference heuristic is used
    p, fb = mlp.propose(10**16, 1 << 20)
    ref = dr_b200.default_params(10**16, dr_b200.POLICY_REFERENCE)
    assert fb and (p.u_total, p.u_dense, p.cx, p.mu_limit) == (ref.u_total, ref.u_dense, ref.cx, ref.mu_limit)


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="trained weights not committed")
def test_trained_tuner_beats_default_heuristic(engine):
    """At X = 3*10^16 (M pinned by the reference engine's own run,
    tests/golden/m30000000000000000.json) the proposal of the committed weights
    is at least 5% faster on the device than the reference's default heuristic."""
    with open(WEIGHTS) as f:
        w = np.array(json.load(f)["weights"], dtype=np.float32)
    mlp = dr_b200.MLP(engine)
    mlp.set_weights(w)
    X = 3 * 10**16
    p, fb = mlp.propose(X, 160 * 2**30)
    assert not fb
    d = dr_b200.default_params(X, dr_b200.POLICY_REFERENCE)

    def t(params):
        best = None
        for _ in range(2):
            r = engine.mertens(X, params)
            assert r.M == -1493402
            v = r.stats.table_ms + r.stats.plan_ms + r.stats.sums_ms
            best = v if best is None else min(best, v)
        return best

    td, tm = t(d), t(p)
    assert tm < 0.95 * td, (tm, td)
