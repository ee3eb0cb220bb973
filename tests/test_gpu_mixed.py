"""Half-precision noise mode (DriverConfig::NumericMode kFp16 / kMixed).

The noise is drawn with the SM's approximate transcendentals and rounded
once to FP16; rollout and update use that rounded value.  Checked against
the oracle restating the same method (its FP64 noise rounded to FP16), on the
quadrotor model (m = 4: one Philox call per step, its two words split into
four 16-bit uniforms):
  shaped noise      within one FP16 rounding step of the oracle's, plus
                    2e-3 * sigma absolute (approximate log near u1 -> 1)
  costs, u_next     on the device's own noise, the oracle's rollout reproduces
                    the device's costs to 1e-5 relative (99 % of the samples:
                    a tumbling quadrotor is chaotic, so FP32 and FP64 dynamics
                    part ways on the few samples that tumble), and the oracle's
                    update on the device's costs reproduces u_next to 1e-4
  closed loop       mixed mode's executed closed-loop cost is statistically
                    indistinguishable from the FP32 mode's (within 5 %).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import abs_err, backend_for, oracle_problem, rel_err
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


def quad(mode: int, N=1, K=2048, H=40, T=1, seed=3):
    w = models.quadrotor_batch(seed=seed, N=N, K=K, H=H, T=T)
    w.numeric_mode = mode
    return w


@pytest.mark.parametrize("mode", [1, 2])
def test_half_noise_matches_rounded_oracle(oracle, mode):
    w = quad(mode, K=512)
    b = backend_for(w)
    p = oracle_problem(w)
    _, eps = b.sample_noise(step=4, agent=0, k0=0, count=512)
    worst = 0.0
    for k in range(0, 512, 5):
        _, e_o = oracle.noise(p, 4, w.seed, k)
        tol = np.abs(e_o) * 2.0 ** -10 + 2e-3 * float(w.sigma[0])
        worst = max(worst, float(np.max(np.abs(eps[k] - e_o) / tol)))
    assert worst <= 1.0
    # the values are FP16 numbers
    assert np.array_equal(eps.astype(np.float16).astype(np.float32), eps)


def test_half_noise_costs_and_update_on_device_noise(oracle):
    w = quad(2, K=2048, H=40)
    w.lam = 200.0
    b = backend_for(w)
    b.bind_params(w.model_params, w.cost_params[0])
    p = oracle_problem(w)
    un = np.full(40 * 4, 2.45, np.float32)
    u_out, _ = b.dispatch_rollout(6, w.x0[0], un)
    _, eps = b.sample_noise(step=6, agent=0, k0=0, count=w.sample_count)
    costs = b.last_costs()[0]
    c_o = oracle.rollout_eps(p, w.x0[0], un, eps)
    r = np.abs(costs - c_o) / np.abs(c_o)
    assert np.quantile(r, 0.99) < 1e-5 and np.median(r) < 1e-6
    w_o, _ = oracle.weights(costs, w.lam)
    assert abs_err(u_out, oracle.update_eps(p, w_o, un, eps)) < 1e-4


def test_mixed_mode_closed_loop_cost_matches_fp32():
    costs = {}
    for mode in (0, 2):
        w = quad(mode, N=8, K=4096, H=50, T=40, seed=21)
        b = backend_for(w)
        r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                             cost_params=w.cost_params_packed, cost_stride=w.cost_stride)
        costs[mode] = models.executed_cost(w, r["states"], r["controls"], r["terminal"])
    rel = abs(costs[2].mean() - costs[0].mean()) / costs[0].mean()
    assert rel < 0.05, (costs[0].mean(), costs[2].mean())


def test_quadrotor_fp32_matches_oracle(oracle):
    """FP32 mode.  Random thrusts can tumble a quadrotor, and a tumbling rigid
    body amplifies FP32-vs-FP64 rounding chaotically, so per-sample costs are
    compared in distribution (99 % of the samples to 1e-5 relative, on the
    device's own noise and end to end) and u_next stage-isolated (the
    oracle's weights and update on the device's costs and noise)."""
    w = quad(0, K=1024, H=50)
    w.lam = 200.0
    b = backend_for(w)
    p = oracle_problem(w)
    un = np.full(50 * 4, 2.45, np.float32)
    u_out, _ = b.dispatch_rollout(2, w.x0[0], un)
    costs = b.last_costs()[0]
    _, eps = b.sample_noise(step=2, agent=0, k0=0, count=w.sample_count)
    c_o = oracle.rollout_eps(p, w.x0[0], un, eps)
    assert np.quantile(np.abs(costs - c_o) / np.abs(c_o), 0.99) < 1e-5
    w_o, _ = oracle.weights(costs, w.lam)
    assert abs_err(u_out, oracle.update_eps(p, w_o, un, eps)) < 1e-4
    o = oracle.step(p, 2, w.seed, w.x0[0], un)
    r = np.abs(costs - o["costs"]) / np.abs(o["costs"])
    assert np.quantile(r, 0.99) < 1e-5


@pytest.mark.parametrize("seed", [3, 8])
def test_quadrotor_fp32_well_conditioned_every_sample(oracle, seed):
    """FP32 quadrotor pinned by its maximum: a well-conditioned case (hover
    nominal, sigma 0.1, H 30, lambda 1 as configured) where no sample
    tumbles.  End to end against the oracle on the same seed: every
    sample's cost to 1e-5 relative, u_next to 1e-4, weights to 1e-5 and ESS
    to 1e-5 relative, for two warm-started steps."""
    w = quad(0, K=2048, H=30, seed=seed)
    assert w.lam == 1.0
    w.sigma = np.full(4, 0.1, np.float32)
    w.sigma_inv = (1.0 / w.sigma ** 2).astype(np.float32)
    b = backend_for(w)
    p = oracle_problem(w)
    hover = float(w.u_max[0]) / 2.0
    un = np.full(w.horizon * 4, hover, np.float32)
    for step in (0, 1):
        u_out, diag = b.dispatch_rollout(step, w.x0[0], un)
        o = oracle.step(p, step, w.seed, w.x0[0], un)
        assert rel_err(b.last_costs()[0], o["costs"]) <= 1e-5
        assert abs_err(u_out, o["u_out"]) <= 1e-4
        assert abs_err(b.last_weights()[0], o["weights"]) <= 1e-5
        assert rel_err([diag[2]], [o["diag"][2]]) <= 1e-5
        un = np.concatenate([u_out[4:], u_out[-4:]]).astype(np.float32)
