"""Stochastic dynamics: a plugin that draws its own randoms from the Philox
counter and key the library hands to the dynamics callable (the reference's
contract, shaders/mppi_rollout.metal:89-90 and mppi_reduce.metal:212-214,
used by its WEZ example, wez_environment.metal:166-173).  Rollout counter
(step, k*H*P + t + 0x80000000); propagation counter (step, 0x80000000) with
seed = agent index.  Checked against the FP64 oracle's restatement of the
same model (ORACLE_MODEL_GUST)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import backend_for, oracle_problem, rel_err
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


def _event_fraction(oracle, step, key, K, H):
    """Share of samples whose gust event fires within the horizon (from the
    counters alone: the event never depends on the state)."""
    k = np.repeat(np.arange(K, dtype=np.uint64), H)
    t = np.tile(np.arange(H, dtype=np.uint64), K)
    c1 = ((k * H + t + 0x80000000 + 0x1000) & 0xFFFFFFFF).astype(np.uint32)
    c0 = np.full(c1.shape, step, np.uint32)
    w = oracle.philox(c0, c1, np.full(c1.shape, key, np.uint32))
    u = (w[:, 0].astype(np.float32) + np.float32(0.5)) * np.float32(2.0 ** -32)
    fired = (u < np.float32(0.02)).reshape(K, H).any(axis=1)
    return float(fired.mean())


def test_stochastic_rollout_matches_oracle(oracle):
    w = models.gust_batch(seed=1, N=1, K=1024, H=30)
    b = backend_for(w)
    x0 = np.array([1.0, -2.0, 0.3, 0.0, 0.0], np.float32)
    u_nom = (np.random.default_rng(0).normal(size=60) * 0.3).astype(np.float32)
    u, diag = b.dispatch_rollout(5, x0, u_nom)
    costs = b.last_costs()[0]
    p = oracle_problem(w)
    ref = oracle.rollout(p, 5, w.seed, x0, u_nom)
    assert rel_err(costs, ref) <= 1e-5
    frac = _event_fraction(oracle, 5, w.seed, 1024, 30)
    assert 0.2 < frac < 0.8, frac  # the random event really splits the samples
    wts, _ = oracle.weights(costs.astype(np.float64), w.lam)
    u_ref = oracle.update(p, 5, w.seed, wts, u_nom)
    assert np.abs(u - u_ref).max() <= 1e-4


def test_stochastic_batch_closed_loop_matches_oracle(oracle):
    w = models.gust_batch(seed=2, N=8, K=512, H=20, T=15)
    b = backend_for(w)
    r = b.simulate_batch(8, 15, 0, w.x0)
    ref = oracle.simulate_batch(oracle_problem(w), 8, 15, 0, w.seed, w.x0)
    assert np.abs(r["states"] - ref["states"]).max() <= 1e-3
    assert np.abs(r["controls"] - ref["controls"]).max() <= 1e-3
    assert np.abs(r["terminal"] - ref["terminal"]).max() <= 1e-3
    # propagation draws with seed = agent index: identical agents diverge
    same = np.repeat(w.x0[:1], 8, axis=0)
    r2 = b.simulate_batch(8, 15, 0, same)
    assert not np.allclose(r2["terminal"][0], r2["terminal"][1])


def test_stochastic_same_seed_is_bit_identical():
    w = models.gust_batch(seed=3, N=4, K=256, H=16, T=10)
    a = backend_for(w).simulate_batch(4, 10, 0, w.x0)
    c = backend_for(w).simulate_batch(4, 10, 0, w.x0)
    assert np.array_equal(a["states"], c["states"])
    d = backend_for(w, seed=w.seed + 1).simulate_batch(4, 10, 0, w.x0)
    assert not np.array_equal(a["states"], d["states"])
