"""The combine fused into the rollout launch (each agent's last rollout CTA
runs the agent's weighted update, diagnostics, propagate and shift) against
the separate combine kernel (MPPI_B200_SEPARATE_COMBINE=1, read when a
backend is created): closed loops of uniform batches, uneven batches and a
proposal closed loop give the same bits, and a single step's u_next and
diagnostics are the same too."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import backend_for
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


def _separate(fn):
    """Runs fn() with backends created under MPPI_B200_SEPARATE_COMBINE=1."""
    old = os.environ.get("MPPI_B200_SEPARATE_COMBINE")
    os.environ["MPPI_B200_SEPARATE_COMBINE"] = "1"
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["MPPI_B200_SEPARATE_COMBINE"]
        else:
            os.environ["MPPI_B200_SEPARATE_COMBINE"] = old


def _uniform_loop(w):
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    kps = b.launch_info()["kernels_per_step"]
    b.close()
    return r, kps


def _assert_same(r1, r2):
    for key in r1:
        if isinstance(r1[key], np.ndarray):
            assert np.array_equal(r1[key], r2[key]), key


@pytest.mark.parametrize("K", [1000, 4096])
def test_fused_combine_matches_separate_uniform(K):
    w = models.unicycle_batch(seed=21, N=24, K=K, H=20, T=12)
    fused, kf = _uniform_loop(w)
    sep, ks = _separate(lambda: _uniform_loop(w))
    assert kf == 1 and ks == 2
    _assert_same(fused, sep)


def test_fused_combine_matches_separate_uneven():
    w = models.bicycle_uneven(seed=5, N=9, T=4, k_range=(100, 1500), h_range=(6, 28))

    def run():
        b = backend_for(w)
        r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                             cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
                             sigma=w.agent_sigma, sample_counts=w.agent_K, horizons=w.agent_H)
        b.close()
        return r

    _assert_same(run(), _separate(run))


def test_fused_combine_matches_separate_single_step():
    w = models.unicycle_single(seed=3, K=1024, H=30)
    x0 = np.array([0.5, -1.0, 0.2, 0.0], np.float32)
    u_nom = np.linspace(-0.2, 0.3, w.horizon * w.control_dim).astype(np.float32)

    def step():
        b = backend_for(w)
        out = b.dispatch_rollout(4, x0, u_nom)
        b.close()
        return out

    (u1, d1), (u2, d2) = step(), _separate(step)
    assert np.array_equal(u1, u2) and np.array_equal(d1, d2)
