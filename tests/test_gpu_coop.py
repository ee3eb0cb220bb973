"""The cooperative rollout form (plugins that split their stage cost with
MPPI_STAGE_COST_SPLIT; the unicycle splits its obstacle terms in 4 parts).

Four lanes share a sample: they step the same dynamics on the same staged
noise and each accumulates one part of the stage cost; the parts are summed
at the end.  The backend uses it for launch shapes whose one-thread form
would have at most one 128-sample CTA per four SMs (32-sample CTAs there);
MPPI_B200_COOP=1 pins it for every shape (128-sample CTAs for large ones),
MPPI_B200_COOP=0 off.  Pinned on here unless a test says otherwise.
Checked here:
  * the shape rule and the pins;
  * against the FP64 oracle: costs 1e-5 relative, u_next 1e-4, weights 1e-5
    (a single agent); batch closed loops at lambda = 1 (both CTA sizes) as
    close to the oracle as the reference's own FP32 kernels (see
    test_gpu_lambda_one.py);
  * against the one-thread-per-sample form (MPPI_B200_COOP=0): the same
    values up to the order of the cost sums (1e-6 relative on costs);
  * its fused and separate combines give the same bits, and the closed loop
    is reproducible;
  * with a learned proposal attached (the proposal workload's shape).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import abs_err, backend_for, oracle_problem, rel_err
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cooperative(monkeypatch):
    monkeypatch.setenv("MPPI_B200_COOP", "1")


def _env(pairs, fn):
    old = {k: os.environ.get(k) for k in pairs}
    os.environ.update(pairs)
    try:
        return fn()
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _step(w, x0, u_nom, step=3):
    b = backend_for(w)
    u, d = b.dispatch_rollout(step, x0, u_nom)
    out = (u, d, b.last_costs()[0], b.last_weights()[0], b.launch_info()["form"])
    b.close()
    return out


def test_cooperative_form_follows_shape_rule_and_pins(monkeypatch):
    single = models.unicycle_single(seed=0, K=1024, H=30)
    u0 = np.zeros(60, np.float32)
    assert _step(single, single.x0[0], u0)[4]["cooperative"]
    monkeypatch.setenv("MPPI_B200_COOP", "0")
    assert not _step(single, single.x0[0], u0)[4]["cooperative"]
    monkeypatch.delenv("MPPI_B200_COOP")
    assert _step(single, single.x0[0], u0)[4]["cooperative"]  # few CTAs: by default
    big = models.unicycle_batch(seed=3, N=48, K=1024, H=20, T=2)

    def form():
        b = backend_for(big)
        b.prepare(big.num_agents, big.num_steps, big.x0, cost_params=big.cost_params_packed,
                  cost_stride=big.cost_stride, sigma=big.agent_sigma)
        b.run(0)
        f = b.launch_info()["form"]
        b.close()
        return f

    assert not form()["cooperative"]  # many CTAs: the one-thread form
    monkeypatch.setenv("MPPI_B200_COOP", "1")
    assert form()["cooperative"]


@pytest.mark.parametrize("K,H", [(1024, 30), (777, 17)])
def test_cooperative_step_matches_oracle(oracle, K, H):
    w = models.unicycle_single(seed=4, K=K, H=H)
    x0 = np.array([1.5, -0.5, 0.4, 0.0], np.float32)
    u_nom = (np.random.default_rng(K).normal(size=H * 2) * 0.3).astype(np.float32)
    u, d, costs, wts, form = _step(w, x0, u_nom)
    assert form["cooperative"]
    o = oracle.step(oracle_problem(w), 3, w.seed, x0, u_nom)
    assert rel_err(costs, o["costs"]) <= 1e-5
    assert abs_err(u, o["u_out"]) <= 1e-4
    assert abs_err(wts, o["weights"]) <= 1e-5
    assert rel_err([d[2]], [o["diag"][2]]) <= 1e-5


def test_cooperative_matches_one_thread_per_sample():
    w = models.unicycle_single(seed=6, K=2048, H=30)
    x0 = np.array([-3.0, 2.0, -0.7, 0.0], np.float32)
    u_nom = np.linspace(-0.4, 0.4, 60).astype(np.float32)
    uc, dc, cc, _, fc = _step(w, x0, u_nom)
    up, dp, cp, _, fp = _env({"MPPI_B200_COOP": "0"}, lambda: _step(w, x0, u_nom))
    assert fc["cooperative"] and not fp["cooperative"]
    assert rel_err(cc, cp) <= 1e-6
    assert abs_err(uc, up) <= 1e-5


def _loop(w):
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    f = b.launch_info()["form"]
    b.close()
    return r, f


def test_cooperative_cta_size_follows_the_launch_shape():
    # few CTAs: 32 samples per CTA (an agent's samples over more SMs); many:
    # 128 samples per CTA (as many partial records as the one-thread form)
    small = models.unicycle_batch(seed=34, N=2, K=1024, H=20, T=2)
    large = models.unicycle_batch(seed=35, N=48, K=1024, H=20, T=2)
    for w, block in ((small, 32), (large, 128)):
        b = backend_for(w)
        b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
                  cost_stride=w.cost_stride, sigma=w.agent_sigma)
        b.run(0)
        info = b.launch_info()
        b.close()
        assert info["form"]["cooperative"] and info["block"] == block, info


def test_cooperative_fused_and_separate_combine_same_bits():
    w = models.unicycle_batch(seed=31, N=3, K=1000, H=24, T=10)
    fused, ff = _env({"MPPI_B200_FUSED_COMBINE": "1"}, lambda: _loop(w))
    sep, fs = _env({"MPPI_B200_SEPARATE_COMBINE": "1"}, lambda: _loop(w))
    assert ff["cooperative"] and fs["cooperative"]
    assert ff["fused_combine"] and not fs["fused_combine"]
    for k in fused:
        assert np.array_equal(fused[k], sep[k]), k
    again, _ = _loop(w)
    for k in fused:
        assert np.array_equal(fused[k], again[k]), k


@pytest.mark.parametrize("N,H,T,block", [(4, 30, 6, 32), (48, 20, 3, 128)])
def test_cooperative_closed_loop_matches_oracle(oracle, N, H, T, block):
    import pyoracle
    if not pyoracle.ref_available("unicycle_obstacles"):
        pytest.skip("oracle/_ref (the reference kernels for the CPU) not built")
    w = models.unicycle_batch(seed=32, N=N, K=1024, H=H, T=T)
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    f, blk = b.launch_info()["form"], b.launch_info()["block"]
    b.close()
    assert f["cooperative"] and blk == block
    p = oracle_problem(w)
    o = oracle.simulate_batch(p, w.num_agents, w.num_steps, 0, w.seed, w.x0,
                              cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride,
                              sigma_packed=w.agent_sigma.astype(float))
    rr = pyoracle.RefKernels("unicycle_obstacles").simulate_batch(
        p, w.num_agents, w.num_steps, 0, w.seed, w.x0, sigma_packed=w.agent_sigma,
        cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride,
        model_params_packed=w.model_params, model_stride=0, nthreads=8)
    for k in ("controls", "states"):
        lib, ref = abs_err(r[k], o[k]), abs_err(rr[k], o[k])
        print(f"cooperative closed loop {k}: library {lib:.2e}, reference FP32 kernels {ref:.2e}")
        assert lib <= max(1e-4, 3.0 * ref)


def test_cooperative_with_proposal_matches_one_thread_per_sample():
    pytest.importorskip("torch")
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=33, N=12, K=256, H=64, T=4)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=9)

    def run():
        b = backend_for(w, bind=False)
        b.set_features("mppi_proposal_features", 31)
        b.set_proposal(net, 128)
        b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
                  cost_stride=w.cost_stride, model_params=w.model_params, sigma=w.agent_sigma)
        b.run(0)
        r, f = b.fetch(), b.launch_info()["form"]
        b.set_proposal(None)
        b.close()
        return r, f

    rc, fc = run()
    rp, fp = _env({"MPPI_B200_COOP": "0"}, run)
    assert fc["cooperative"] and not fp["cooperative"]
    assert abs_err(rc["controls"], rp["controls"]) <= 1e-4
    assert abs_err(rc["states"], rp["states"]) <= 1e-4
