"""Uneven batches on the GPU: agents with their own sample count, horizon
and full noise covariance in one persistent launch per pass, against the FP64
oracle agent by agent; and the invariances the design promises (an uneven
batch of equal shapes is bit-identical to the uniform path; the tuned grid
size and staging mode do not change a bit)."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from helpers import abs_err, backend_for
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu
TOL_U = 1e-4


def small_uneven(seed=5, N=6, T=3):
    w = models.bicycle_uneven(seed=seed, N=N, T=T, k_range=(100, 700), h_range=(6, 28))
    w.lam = 50.0  # well-conditioned weights for the FP32 / FP64 comparison
    return w


def run_uneven(w, backend=None):
    b = backend or backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma,
                         sample_counts=w.agent_K, horizons=w.agent_H)
    return b, r


def oracle_agent(oracle, w, a):
    p = pyoracle.Problem(w.oracle_model, w.state_dim, w.control_dim, int(w.agent_H[a]),
                         int(w.agent_K[a]), w.lam, w.agent_sigma[a].astype(float),
                         w.u_min.astype(float), w.u_max.astype(float),
                         sigma_inv=np.linalg.inv(w.agent_sigma[a].reshape(2, 2)).ravel(),
                         cov_full=True, model_params=w.model_params, cost_params=w.cost_params[a])
    return oracle.simulate(p, w.num_steps, 0, w.seed + a, w.x0[a],
                           np.zeros(int(w.agent_H[a]) * w.control_dim))


def test_uneven_batch_matches_oracle_per_agent(oracle):
    w = small_uneven()
    b, r = run_uneven(w)
    assert b.tuning_info()["num_work"] == int(sum((k + 127) // 128 for k in w.agent_K))
    for a in range(w.num_agents):
        o = oracle_agent(oracle, w, a)
        assert abs_err(r["controls"][:, a], o["controls"]) < TOL_U, a
        assert abs_err(r["states"][:, a], o["states"]) < TOL_U, a
        assert abs_err(r["terminal"][a], o["x_final"]) < TOL_U, a


def test_uneven_with_equal_shapes_is_bitwise_uniform():
    w = small_uneven(seed=9, N=4)
    w.agent_K = np.full(w.num_agents, w.sample_count, np.uint32)
    w.agent_H = np.full(w.num_agents, w.horizon, np.uint32)
    b = backend_for(w)
    _, ru = run_uneven(w, b)
    ro = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                          cost_stride=w.cost_stride, sigma=w.agent_sigma)
    if b.launch_info()["block"] != 128:
        pytest.skip("uniform path chose another CTA size for this shape")
    for k in ("states", "controls", "costs", "terminal"):
        assert np.array_equal(ru[k], ro[k]), k


@pytest.mark.parametrize("grid,rows", [("0", ""), ("148", ""), ("592", "8")])
def test_tuned_geometry_does_not_change_results(monkeypatch, grid, rows):
    w = small_uneven(seed=11, N=5)
    _, ref = run_uneven(w)
    monkeypatch.setenv("MPPI_B200_UNEVEN_GRID", grid)
    if rows:
        monkeypatch.setenv("MPPI_B200_UNEVEN_STAGE_ROWS", rows)
    b, r = run_uneven(w)
    info = b.tuning_info()
    assert info["grid"] == int(grid)
    for k in ("states", "controls", "costs", "terminal"):
        assert np.array_equal(r[k], ref[k]), k


def test_uneven_rejects_out_of_range_shapes():
    from mppi_metal_b200.backend import BackendError
    w = small_uneven(N=3)
    ks = w.agent_K.copy()
    ks[1] = w.sample_count + 1
    b = backend_for(w)
    with pytest.raises(BackendError, match="sample_counts"):
        b.simulate_batch(3, 2, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma, sample_counts=ks,
                         horizons=w.agent_H)
