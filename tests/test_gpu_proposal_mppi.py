"""GPU parity of proposal-MPPI: the plugin's feature callable, the recorded
u* history, and a control step whose samples partly draw around the
network's prediction, all against the CPU oracle.

Tolerances as in the plain parity tests: features 1e-5 absolute (FP32
against float64; obstacle ranking may differ only on near-ties), per-sample
costs 1e-5 relative, u_next 1e-4 absolute (the update checked on the
device's own costs).
"""
from __future__ import annotations

import numpy as np
import pytest

import mlp_oracle as mo
from helpers import backend_for, oracle_problem, rel_err
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FEATURES = "mppi_proposal_features"


def _batch_backend(w):
    b = backend_for(w, bind=False)
    b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
              cost_stride=w.cost_stride, model_params=w.model_params, model_stride=0,
              sigma=w.agent_sigma)
    return b


def test_features_match_oracle():
    w = models.unicycle_batch(seed=3, N=64, K=256, H=16, T=2)
    b = _batch_backend(w)
    b.set_features(FEATURES, 31)
    rng = np.random.default_rng(0)
    R = 64 * 4
    st = np.zeros((R, 4), np.float32)
    st[:, :2] = rng.uniform(-10, 10, (R, 2))
    st[:, 2] = rng.uniform(-np.pi, np.pi, R)
    st[:, 3] = rng.uniform(0, 15, R)
    f = b.features(st, agents_mod=64)
    ref = np.stack([mo.unicycle_features(st[r], w.cost_params[r % 64]) for r in range(R)])
    d = np.abs(f - ref).max(axis=1)
    assert f.shape == (R, 31)
    assert np.mean(d <= 1e-5) >= 0.99, np.sort(d)[-5:]
    # the state and goal features never depend on the ranking
    assert np.abs(f[:, :7] - ref[:, :7]).max() <= 1e-5


def test_missing_feature_callable_is_named():
    from mppi_metal_b200.backend import BackendError
    w = models.unicycle_batch(seed=3, N=4, K=128, H=8, T=1)
    b = backend_for(w)
    with pytest.raises(BackendError) as e:
        b.set_features("no_such_features", 31)
    assert "no_such_features" in e.value.msg and e.value.code == 3


def test_recorded_ustar_matches_the_applied_controls():
    w = models.unicycle_batch(seed=4, N=16, K=512, H=20, T=6)
    b = backend_for(w, bind=False)
    b.set_record_ustar(True)
    b.prepare(16, 6, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              model_params=w.model_params, sigma=w.agent_sigma)
    b.run(0)
    r = b.fetch()
    us = b.fetch_ustar()
    assert us.shape == (6, 16, 20, 2)
    assert np.array_equal(us[:, :, 0, :], r["controls"])
    last = us[-1]
    shifted = np.concatenate([last[:, 1:], last[:, -1:]], axis=1).reshape(16, -1)
    assert np.array_equal(shifted, r["u_nom"])


def _proposal_case(samples: int):
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=5, N=1, K=1024, H=64, T=1)
    b = backend_for(w)
    b.set_features(FEATURES, 31)
    shape = mo.Shape(31, 64, 2)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=1)
    net.set_params(mo.init_params(shape, 4))
    b.set_proposal(net, samples)
    return w, b, net, shape


@pytest.mark.parametrize("samples", [512, 1024])
def test_proposal_step_matches_oracle(oracle, samples):
    w, b, net, shape = _proposal_case(samples)
    x0 = w.x0[0].copy()
    rng = np.random.default_rng(6)
    u_nom = (rng.normal(size=64 * 2) * 0.3).astype(np.float32)
    step = 7
    u_out, diag = b.dispatch_rollout(step, x0, u_nom)
    costs = b.last_costs()[0]
    # the network's output on the same features (same kernels, same bits)
    feats = b.features(x0[None, :], agents_mod=1)
    out = net.forward(torch.from_numpy(np.ascontiguousarray(feats)).cuda()).cpu().numpy()[0]
    mu = out[:128].astype(np.float64)
    ps = np.exp(np.clip(out[128:130].astype(np.float32), -3.0, 1.0)).astype(np.float64)
    p = oracle_problem(w)
    eps = np.zeros((1024, 64, 2))
    sh = (mu - u_nom.astype(np.float64)).reshape(64, 2)
    for k in range(1024):
        n, e = oracle.noise(p, step, w.seed, k)
        eps[k] = sh + ps * n if k < samples else e
    ref = oracle.rollout_eps(p, x0, u_nom, eps)
    assert rel_err(costs, ref) <= 1e-5
    wts, _ = oracle.weights(costs.astype(np.float64), w.lam)
    u_ref = oracle.update_eps(p, wts, u_nom, eps)
    assert np.abs(u_out - u_ref).max() <= 1e-4
    assert diag[0] == pytest.approx(costs.min(), rel=1e-6)


def test_detaching_restores_the_plain_path():
    w, b, net, shape = _proposal_case(512)
    x0 = w.x0[0].copy()
    u_nom = np.zeros(128, np.float32)
    b.set_proposal(None)
    u1, _ = b.dispatch_rollout(3, x0, u_nom)
    plain = backend_for(w)
    u2, _ = plain.dispatch_rollout(3, x0, u_nom)
    assert np.array_equal(u1, u2)


def test_proposal_batch_closed_loop_runs():
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=7, N=130, K=256, H=64, T=5)
    b = backend_for(w, bind=False)
    b.set_features(FEATURES, 31)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=2)
    b.set_proposal(net, 128)
    b.prepare(130, 5, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              model_params=w.model_params, sigma=w.agent_sigma)
    b.run(0)
    r1 = b.fetch()
    assert np.all(np.isfinite(r1["states"])) and np.all(np.isfinite(r1["controls"]))
    # replay of the captured graph gives the same bits
    b.prepare(130, 5, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              model_params=w.model_params, sigma=w.agent_sigma)
    b.run(0)
    r2 = b.fetch()
    assert np.array_equal(r1["states"], r2["states"])


def test_driver_api_runs_the_proposal():
    """DriverOptions.proposal through the public MPPIDriver API gives the same
    closed loop, bit for bit, as the backend path."""
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200._lib import plugin_path
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=8, N=32, K=256, H=64, T=4)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=3)
    cfg = D.DriverConfig(4, 2, 64, 256, w.lam,
                         D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, w.sigma, w.sigma_inv, 2),
                         D.ControlBounds(w.u_min, w.u_max, 2))
    drv = D.MPPIDriver(cfg, D.DriverOptions(proposal=net, proposal_samples=128))
    err = D.ErrorRef()
    spec = D.ModelPluginSpec(plugin_path(w.plugin),
                             D.CallableNames("mppi_dynamics", "mppi_stage_cost",
                                             "mppi_terminal_cost"),
                             D.ParamLayout(len(w.model_params), 4, w.cost_stride, 4),
                             D.RngConfig(w.seed))
    assert drv.initialize(spec, err), err.value
    assert drv.set_problem_params(D.ProblemParams(D.ByteView.of(w.model_params),
                                                  D.ByteView.of(w.cost_params[0])), err), err.value
    outs = D.BatchSimulationResults(np.zeros((4, 32, 4), np.float32),
                                    np.zeros((4, 32, 2), np.float32), np.zeros((4, 32), np.float32),
                                    np.zeros((32, 4), np.float32), 32, 4)
    ap = D.BatchAgentParams(cost_params=w.cost_params_packed, cost_params_stride=w.cost_stride,
                            sigma=w.agent_sigma)
    assert drv.simulate_batch(32, 4, w.x0, outs, ap, err), err.value
    b = backend_for(w, bind=True)
    b.set_features(FEATURES, 31)
    b.set_proposal(net, 128)
    b.prepare(32, 4, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              sigma=w.agent_sigma)
    b.run(0)
    r = b.fetch()
    assert np.array_equal(outs.states_out, r["states"])
    assert np.array_equal(outs.controls_out, r["controls"])


def test_fused_next_step_features_match_the_feature_kernel():
    """In the captured closed loop each combine also evaluates the next
    step's features; chaining one-step loops (each starting with the
    separate feature kernel) must give the same trajectory bit for bit."""
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=9, N=16, K=256, H=64, T=4)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=4)

    def backend():
        b = backend_for(w, bind=True)
        b.set_features(FEATURES, 31)
        b.set_proposal(net, 128)
        return b

    b = backend()
    b.prepare(16, 4, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              sigma=w.agent_sigma)
    b.run(0)
    whole = b.fetch()
    c = backend()
    x, un, states = w.x0, None, []
    for s in range(4):
        c.prepare(16, 1, x, un, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
                  sigma=w.agent_sigma)
        c.run(s)
        r = c.fetch()
        states.append(r["states"][0])
        x, un = r["x"], r["u_nom"]
    assert np.array_equal(whole["states"], np.stack(states))
    assert np.array_equal(whole["terminal"], x)


def test_quadrotor_features_match_oracle():
    w = models.quadrotor_batch(seed=5, N=16, K=256, H=20, T=2)
    b = _batch_backend(w)
    b.set_features(FEATURES, 29)
    rng = np.random.default_rng(1)
    R = 16 * 4
    st = np.zeros((R, 12), np.float32)
    st[:, :3] = rng.uniform(-5, 5, (R, 3))
    st[:, 3:] = rng.normal(size=(R, 9)) * 0.5
    f = b.features(st, agents_mod=16)
    ref = np.stack([mo.quadrotor_features(st[r], w.cost_params[r % 16]) for r in range(R)])
    d = np.abs(f - ref).max(axis=1)
    assert f.shape == (R, 29)
    assert np.mean(d <= 1e-5) >= 0.99, np.sort(d)[-5:]
    assert np.abs(f[:, :13] - ref[:, :13]).max() <= 1e-5


def test_short_network_horizon_shifts_only_its_steps(oracle):
    """A network predicting fewer steps than the horizon: proposal samples
    get the mean shift on those steps only (checked against the oracle on
    the device's noise layout)."""
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=6, N=1, K=512, H=40, T=1)
    b = backend_for(w)
    b.set_features(FEATURES, 31)
    shape = mo.Shape(31, 16, 2)
    net = ProposalNet(31, 16, 2, max_batch=128, seed=1)
    net.set_params(mo.init_params(shape, 8))
    b.set_proposal(net, 256)
    x0 = w.x0[0].copy()
    u_nom = (np.random.default_rng(2).normal(size=80) * 0.3).astype(np.float32)
    u_out, _ = b.dispatch_rollout(3, x0, u_nom)
    costs = b.last_costs()[0]
    feats = b.features(x0[None, :], agents_mod=1)
    out = net.forward(torch.from_numpy(np.ascontiguousarray(feats)).cuda()).cpu().numpy()[0]
    ps = np.exp(np.clip(out[32:34].astype(np.float32), -3.0, 1.0)).astype(np.float64)
    sh = np.zeros((40, 2))
    sh[:16] = out[:32].astype(np.float64).reshape(16, 2) - u_nom[:32].astype(np.float64).reshape(16, 2)
    p = oracle_problem(w)
    eps = np.zeros((512, 40, 2))
    for k in range(512):
        n, e = oracle.noise(p, 3, w.seed, k)
        eps[k] = sh + ps * n if k < 256 else e
    ref = oracle.rollout_eps(p, x0, u_nom, eps)
    assert rel_err(costs, ref) <= 1e-5


def test_proposal_with_uneven_shapes_matches_uniform(monkeypatch):
    """A proposal attached to an uneven batch whose agents all have the same
    K and H (the persistent work-list kernel) gives the uniform batch's
    bits; with truly uneven shapes it stays deterministic across the
    autotuner's choices.  (The uniform batch is pinned to one thread per
    sample: the cooperative form it would pick at this size sums costs in
    its own order.)"""
    from mppi_metal_b200.proposal import ProposalNet
    monkeypatch.setenv("MPPI_B200_COOP", "0")
    w = models.unicycle_batch(seed=11, N=12, K=384, H=64, T=3)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=5)

    def run(ks=None, hs=None):
        b = backend_for(w, bind=True)
        b.set_features(FEATURES, 31)
        b.set_proposal(net, 128)
        b.prepare(12, 3, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
                  sigma=w.agent_sigma, sample_counts=ks, horizons=hs)
        b.run(0)
        return b, b.fetch()

    b_u, uniform = run()
    if b_u.launch_info()["block"] != 128:
        pytest.skip("uniform path chose another CTA size for this shape")
    _, ragged = run(np.full(12, 384, np.uint32), np.full(12, 64, np.uint32))
    for k in ("states", "controls", "costs", "terminal"):
        assert np.array_equal(uniform[k], ragged[k]), k
    ks = np.array([128, 384, 200, 256] * 3, np.uint32)
    hs = np.array([64, 32, 48, 16] * 3, np.uint32)
    _, r1 = run(ks, hs)
    _, r2 = run(ks, hs)
    assert np.array_equal(r1["states"], r2["states"])
    assert np.all(np.isfinite(r1["states"]))


def test_proposal_in_mixed_numeric_mode_matches_oracle(oracle):
    """FP16 noise mode: the proposal draw (mu - u_nom) + exp(s) n is rounded
    to FP16 like the plain draw, on the fast-transcendental normals."""
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=12, N=1, K=512, H=32, T=1)
    w.numeric_mode = 2
    b = backend_for(w)
    b.set_features(FEATURES, 31)
    shape = mo.Shape(31, 32, 2)
    net = ProposalNet(31, 32, 2, max_batch=128, seed=6)
    net.set_params(mo.init_params(shape, 9))
    b.set_proposal(net, 256)
    x0 = w.x0[0].copy()
    u_nom = (np.random.default_rng(3).normal(size=64) * 0.3).astype(np.float32)
    u_out, _ = b.dispatch_rollout(4, x0, u_nom)
    costs = b.last_costs()[0]
    feats = b.features(x0[None, :], agents_mod=1)
    out = net.forward(torch.from_numpy(np.ascontiguousarray(feats)).cuda()).cpu().numpy()[0]
    ps = np.exp(np.clip(out[64:66].astype(np.float32), -3.0, 1.0)).astype(np.float32)
    sh = (out[:64] - u_nom).astype(np.float32).reshape(32, 2)
    p = oracle_problem(w)
    # the device's own normals of this step (fast Box-Muller) and, for the
    # plain samples, its own FP16-rounded draws
    nrm, plain_eps = b.sample_noise(4, 0, 0, 512)
    eps = np.zeros((512, 32, 2))
    for k in range(512):
        if k < 256:  # fmaf(scale, n, shift) in FP32, then rounded to FP16
            e = (ps.astype(np.float64) * nrm[k] + sh.astype(np.float64)).astype(np.float32)
            eps[k] = e.astype(np.float16).astype(np.float64)
        else:
            eps[k] = plain_eps[k]
    ref = oracle.rollout_eps(p, x0, u_nom, eps)
    assert rel_err(costs, ref) <= 1e-5
