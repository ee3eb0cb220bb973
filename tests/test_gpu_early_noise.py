"""Early noise: without a proposal and with the whole horizon staged, the
128-sample rollout draws its noise before it waits for the previous launch
(mppi_rollout_early[_fused]_b128).  Only the time of the draw moves, so the
results must be the same bits as the kernels that draw after the wait
(MPPI_B200_NO_EARLY_NOISE=1): closed loops in both combine forms, and a
single control step's costs and update.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import backend_for
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _one_thread_forms(monkeypatch):
    # the one-thread 128-sample forms (the cooperative ones always draw early)
    monkeypatch.setenv("MPPI_B200_COOP", "0")
    monkeypatch.setenv("MPPI_B200_WS", "0")


def _loop(w):
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    info = b.launch_info()
    b.close()
    return r, info


@pytest.mark.parametrize("combine", ["MPPI_B200_FUSED_COMBINE", "MPPI_B200_SEPARATE_COMBINE"])
def test_early_noise_closed_loop_same_bits(monkeypatch, combine):
    w = models.unicycle_batch(seed=41, N=12, K=1024, H=30, T=8)
    monkeypatch.setenv(combine, "1")
    early, info = _loop(w)
    assert info["stage_rows"] >= w.horizon * w.control_dim and info["block"] == 128
    monkeypatch.setenv("MPPI_B200_NO_EARLY_NOISE", "1")
    late, _ = _loop(w)
    for k in early:
        assert np.array_equal(early[k], late[k]), k


def test_early_noise_single_step_same_bits(monkeypatch):
    w = models.unicycle_batch(seed=42, N=1, K=4096, H=50, T=1)
    x0 = w.x0[0]
    u_nom = np.linspace(-0.5, 0.5, w.horizon * w.control_dim).astype(np.float32)

    def step():
        b = backend_for(w)
        b.bind_params(w.model_params, w.cost_params[0])
        u, d = b.dispatch_rollout(5, x0, u_nom)
        c = b.last_cost_pairs()[0]
        b.close()
        return u, d, c

    u1, d1, c1 = step()
    monkeypatch.setenv("MPPI_B200_NO_EARLY_NOISE", "1")
    u2, d2, c2 = step()
    assert np.array_equal(u1, u2) and np.array_equal(np.asarray(d1), np.asarray(d2))
    assert np.array_equal(c1, c2)
