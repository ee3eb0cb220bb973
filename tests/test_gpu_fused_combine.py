"""The combine fused into the rollout launch (each agent's last rollout CTA
runs the agent's weighted update, diagnostics, propagate and shift) against
the separate combine kernel: closed loops of uniform batches (up to 157
rollout CTAs per agent, past one CTA's worth of records) and of uneven
batches give the same bits, and so do a single step's u_next and
diagnostics.  The same holds for the warp-specialised rollout (a second set
of warps draws the noise ahead), with either combine.  The backend picks the
form per launch shape by timing; MPPI_B200_FUSED_COMBINE=1 /
MPPI_B200_SEPARATE_COMBINE=1 and MPPI_B200_WS=1 / 0 (read when a backend is
created) pin it here.  Programmatic dependent launch, on by default, is
checked against plain launches (MPPI_B200_NO_PDL=1) the same way.
These tests compare the forms with one thread per sample; the cooperative
form, which the backend picks by launch shape for plugins with a split stage
cost, is pinned off here (MPPI_B200_COOP=0) and tested in test_gpu_coop.py."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import backend_for, nonholonomic_example
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _one_thread_per_sample(monkeypatch):
    monkeypatch.setenv("MPPI_B200_COOP", "0")


def _with_env(name, fn, value="1"):
    old = os.environ.get(name)
    os.environ[name] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


def _separate(fn):
    """Runs fn() with backends that use the separate combine kernel."""
    return _with_env("MPPI_B200_SEPARATE_COMBINE", fn)


def _fused(fn):
    """Runs fn() with backends that use the fused form, untimed."""
    return _with_env("MPPI_B200_FUSED_COMBINE", fn)


def _ws(fn):
    """Runs fn() with backends that use the warp-specialised rollout."""
    return _with_env("MPPI_B200_WS", fn)


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


@pytest.mark.parametrize("N,K", [(24, 1000), (24, 4096), (3, 20000)])
def test_fused_combine_matches_separate_uniform(N, K):
    w = models.unicycle_batch(seed=21, N=N, K=K, H=20, T=12)
    fused, kf = _fused(lambda: _uniform_loop(w))
    sep, ks = _separate(lambda: _uniform_loop(w))
    assert kf == 1 and ks == 2
    _assert_same(fused, sep)
    auto, _ = _uniform_loop(w)  # the timed choice, either form: the same bits
    _assert_same(auto, sep)


def test_fused_combine_matches_separate_uneven():
    w = models.bicycle_uneven(seed=5, N=9, T=4, k_range=(100, 1500), h_range=(6, 28))

    def run():
        b = backend_for(w)
        r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                             cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
                             sigma=w.agent_sigma, sample_counts=w.agent_K, horizons=w.agent_H)
        b.close()
        return r

    _assert_same(_fused(run), _separate(run))


def test_fused_combine_matches_separate_single_step():
    w = models.unicycle_single(seed=3, K=1024, H=30)
    x0 = np.array([0.5, -1.0, 0.2, 0.0], np.float32)
    u_nom = np.linspace(-0.2, 0.3, w.horizon * w.control_dim).astype(np.float32)

    def step():
        b = backend_for(w)
        out = b.dispatch_rollout(4, x0, u_nom)
        b.close()
        return out

    (u1, d1), (u2, d2) = _fused(step), _separate(step)
    assert np.array_equal(u1, u2) and np.array_equal(d1, d2)


def test_fused_combine_matches_separate_quadrotor():
    # the propagate's dynamics are one compiled function for both forms; an
    # inlined copy per kernel had contracted multiply-adds differently
    w = models.quadrotor_batch(seed=28, N=3, K=700, H=37, T=6)
    _assert_same(_fused(lambda: _uniform_loop(w))[0], _separate(lambda: _uniform_loop(w))[0])


@pytest.mark.parametrize("N,K,H", [(24, 1000, 20), (3, 20000, 20), (8, 256, 64)])
def test_warp_specialised_rollout_matches_plain(N, K, H):
    w = models.unicycle_batch(seed=22, N=N, K=K, H=H, T=8)
    plain, _ = _separate(lambda: _uniform_loop(w))
    ws_sep, _ = _ws(lambda: _separate(lambda: _uniform_loop(w)))
    ws_fused, kf = _ws(lambda: _fused(lambda: _uniform_loop(w)))
    assert kf == 1
    _assert_same(ws_sep, plain)
    _assert_same(ws_fused, plain)


def test_warp_specialised_single_step_matches_plain():
    w = models.unicycle_single(seed=3, K=1024, H=30)
    x0 = np.array([0.5, -1.0, 0.2, 0.0], np.float32)
    u_nom = np.linspace(-0.2, 0.3, w.horizon * w.control_dim).astype(np.float32)

    def step():
        b = backend_for(w)
        out = b.dispatch_rollout(4, x0, u_nom)
        b.close()
        return out

    (u1, d1), (u2, d2) = _ws(lambda: _fused(step)), _separate(step)
    assert np.array_equal(u1, u2) and np.array_equal(d1, d2)


def test_programmatic_dependent_launch_matches_plain_launches():
    # the loop-constant prologue runs before griddepcontrol.wait; everything
    # the previous launch writes is read after it: same bits either way
    w = models.unicycle_batch(seed=23, N=6, K=1000, H=24, T=10)
    pdl, _ = _uniform_loop(w)
    plain, _ = _with_env("MPPI_B200_NO_PDL", lambda: _uniform_loop(w))
    _assert_same(pdl, plain)


@pytest.mark.parametrize("grid", ["0", "148"])
def test_programmatic_dependent_launch_matches_plain_launches_uneven(grid):
    # one CTA per work item (grid 0): dependent launches; a persistent grid
    # (its queue counter reset before each launch): plain launches either way
    w = models.bicycle_uneven(seed=6, N=9, T=5, k_range=(100, 1500), h_range=(6, 28))

    def run():
        b = backend_for(w)
        r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                             cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
                             sigma=w.agent_sigma, sample_counts=w.agent_K, horizons=w.agent_H)
        b.close()
        return r

    pdl = _with_env("MPPI_B200_UNEVEN_GRID", run, value=grid)
    plain = _with_env("MPPI_B200_UNEVEN_GRID",
                      lambda: _with_env("MPPI_B200_NO_PDL", run), value=grid)
    _assert_same(pdl, plain)


def test_warp_specialised_proposal_loop_matches_plain():
    # the noise warps also draw the proposal samples (mean shift and scales
    # from the network's output): same bits as the plain form
    pytest.importorskip("torch")
    from mppi_metal_b200.proposal import ProposalNet
    w = models.unicycle_batch(seed=24, N=12, K=256, H=64, T=4)
    net = ProposalNet(31, 64, 2, max_batch=256, seed=7)

    def run():
        b = backend_for(w, bind=False)
        b.set_features("mppi_proposal_features", 31)
        b.set_proposal(net, 128)
        b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
                  cost_stride=w.cost_stride, model_params=w.model_params, sigma=w.agent_sigma)
        b.run(0)
        r = b.fetch()
        b.set_proposal(None)
        b.close()
        return r

    ws = _ws(lambda: _fused(run))
    plain = _with_env("MPPI_B200_WS", lambda: _separate(run), value="0")
    _assert_same(ws, plain)



def test_step_form_reported():
    w = models.unicycle_batch(seed=27, N=4, K=512, H=30, T=2)

    def run():
        b = backend_for(w)
        b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
        info = b.launch_info()
        b.close()
        return info["form"]

    assert _ws(lambda: _fused(run)) == {"fused_combine": True, "warp_specialised": True,
                                        "cooperative": False}
    assert _with_env("MPPI_B200_WS", lambda: _separate(run), value="0") == \
        {"fused_combine": False, "warp_specialised": False, "cooperative": False}


def _quad_mixed():
    w = models.quadrotor_batch(seed=29, N=2, K=600, H=30, T=5)
    w.numeric_mode = 2
    return w


# Every shipped plugin, at sizes where all four step forms apply (128-sample
# CTAs, whole horizon staged): each form is a separately compiled kernel, and
# the compiler could contract a plugin's multiply-adds differently in each.
PLUGIN_WORKLOADS = {
    "unicycle_obstacles": lambda: models.unicycle_batch(seed=29, N=6, K=600, H=24, T=5),
    "unicycle_control_cost": lambda: models.unicycle_single(seed=29, K=600, H=24, T=5),
    "quadrotor": lambda: models.quadrotor_batch(seed=29, N=2, K=600, H=30, T=5),
    "quadrotor_mixed": _quad_mixed,
    "bicycle_full_cov": lambda: models.bicycle_uneven(seed=29, N=5, T=5, k_range=(600, 600),
                                                      h_range=(24, 24)),
    "gust_integrator": lambda: models.gust_batch(seed=29, N=5, K=600, H=24, T=5),
    "double_integrator": lambda: models.double_integrator_test(K=600, H=24),
    "nonholonomic_vehicle": lambda: nonholonomic_example(K=600, H=24),
}


@pytest.mark.parametrize("name", sorted(PLUGIN_WORKLOADS))
def test_every_step_form_same_bits_per_plugin(name):
    w = PLUGIN_WORKLOADS[name]()

    def run():
        b = backend_for(w)
        r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                             cost_params=w.cost_params_packed or None, cost_stride=w.cost_stride,
                             sigma=w.agent_sigma)
        form = b.launch_info()["form"]
        b.close()
        return r, form

    base, f0 = _with_env("MPPI_B200_WS", lambda: _separate(run), value="0")
    assert f0 == {"fused_combine": False, "warp_specialised": False, "cooperative": False}
    for ws, pin in ((False, _fused), (True, _separate), (True, _fused)):
        r, f = _with_env("MPPI_B200_WS", lambda: pin(run), value="1" if ws else "0")
        assert f == {"fused_combine": pin is _fused, "warp_specialised": ws,
                     "cooperative": False}
        _assert_same(r, base)


def test_every_step_form_same_bits_quadrotor_proposal():
    # with a network attached the combine also computes the next step's
    # features (one compiled copy of the feature callable for every kernel);
    # the network predicts the first 16 of the 24 steps
    pytest.importorskip("torch")
    from mppi_metal_b200.proposal import ProposalNet
    w = models.quadrotor_batch(seed=30, N=3, K=512, H=24, T=4)
    net = ProposalNet(29, 16, 4, max_batch=128, seed=8)

    def run():
        b = backend_for(w, bind=False)
        b.set_features("mppi_proposal_features", 29)
        b.set_proposal(net, 256)
        b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
                  cost_stride=w.cost_stride, model_params=w.model_params, sigma=w.agent_sigma)
        b.run(0)
        r = b.fetch()
        form = b.launch_info()["form"]
        b.set_proposal(None)
        b.close()
        return r, form

    base, f0 = _with_env("MPPI_B200_WS", lambda: _separate(run), value="0")
    assert f0 == {"fused_combine": False, "warp_specialised": False, "cooperative": False}
    for ws, pin in ((False, _fused), (True, _separate), (True, _fused)):
        r, f = _with_env("MPPI_B200_WS", lambda: pin(run), value="1" if ws else "0")
        assert f == {"fused_combine": pin is _fused, "warp_specialised": ws,
                     "cooperative": False}
        _assert_same(r, base)
