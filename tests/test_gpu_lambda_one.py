"""End-to-end parity at the benchmark configurations' own temperature, lambda = 1.

At lambda = 1 with costs of order 1e3-1e4 the softmax weights change by
their own size for a cost change of one unit, so these tests pin the whole
chain -- rollout costs, the CTA minima, the rescaled sums, the update --
against the FP64 oracle on the configurations as they are benchmarked, with
no temperature override:

* the single-agent configuration (unicycle, K 1024, H 30, 8 static
  obstacles, control cost on, lambda 1, Philox seed 0, x0 = 0) through the
  public driver API, MPPIDriver::step, for the first five closed-loop steps;
* agents shaped like the batched configuration (K 4096, H 50, 16 moving
  obstacles, per-agent sigma, lambda 1), step by step and through the batch
  closed loop -- measured against the reference's own FP32 kernels as well
  (below);
* the executed closed-loop cost of that batch against the reference's own
  kernels compiled for the CPU (the matched-cost figure the benchmark
  reports).

Each step hands the device and the oracle the same inputs (the state and
the warm-started nominal the driver used), so every step is compared on its
own; the next state comes from the oracle's dynamics with the device's
first control.  Bars: u_next 1e-4 absolute,
weights 1e-5 absolute, ESS 1e-5 relative; the best cost to 1e-6 relative.

The single-agent configuration meets them.  The batched configuration's
agents cannot in general, in any FP32 implementation: their positions reach
|x| ~ 10, where a float carries about 1e-6, and the obstacle term weighs
the penetration 1000-fold, so the costs of the samples that graze an
obstacle carry errors of order 1e-3 -- at lambda = 1 weight errors of order
1e-4.  The reference's own kernels (FP32, compiled for the CPU, oracle/_ref)
miss the bars on most of these agents (u_next errors up to 8e-4 on the
first eight).  There the test asserts that the library is as close to the
FP64 oracle as the reference is: each error within the bar or within 3x the
reference kernels' error on the same inputs.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from helpers import abs_err, backend_for, oracle_problem, rel_err
from mppi_metal_b200 import driver as D
from mppi_metal_b200 import models
from mppi_metal_b200._lib import plugin_path

pytestmark = pytest.mark.gpu

TOL_U = 1e-4
TOL_W = 1e-5
TOL_ESS = 1e-5
STEPS = 5


def _driver(w: models.Workload, cost_blob: bytes) -> D.MPPIDriver:
    cfg = D.DriverConfig(w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam,
                         D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, w.sigma, w.sigma_inv,
                                              w.control_dim),
                         D.ControlBounds(w.u_min, w.u_max, w.control_dim))
    drv = D.MPPIDriver(cfg, D.DriverOptions(control_cost=w.control_cost))
    err = D.ErrorRef()
    spec = D.ModelPluginSpec(plugin_path(w.plugin),
                             D.CallableNames("mppi_dynamics", "mppi_stage_cost",
                                             "mppi_terminal_cost"),
                             D.ParamLayout(len(w.model_params), 4, len(cost_blob), 4),
                             D.RngConfig(w.seed))
    assert drv.initialize(spec, err), err.value
    assert drv.set_problem_params(D.ProblemParams(D.ByteView.of(w.model_params),
                                                  D.ByteView.of(cost_blob)), err), err.value
    return drv


def _shift(u: np.ndarray, m: int) -> np.ndarray:
    """The driver's warm start: shift left by one step, hold the last."""
    return np.concatenate([u[m:], u[-m:]]).astype(np.float32)


def _check_step(oracle, p, b, s, key, x, u_nom, u_dev, diag_dev, worst):
    o = oracle.step(p, s, key, x, u_nom)
    worst["u"] = max(worst["u"], abs_err(u_dev, o["u_out"]))
    worst["ess"] = max(worst["ess"], rel_err([diag_dev[2]], [o["diag"][2]]))
    worst["best"] = max(worst["best"], rel_err([diag_dev[0]], [o["diag"][0]]))
    worst["mean"] = max(worst["mean"], rel_err([diag_dev[1]], [o["diag"][1]]))
    # the same step on the backend, for the weights (same library, same bits)
    u_b, d_b = b.dispatch_rollout(s, x, u_nom)
    assert np.array_equal(u_b, u_dev) and np.array_equal(d_b, np.asarray(diag_dev, np.float32))
    worst["w"] = max(worst["w"], abs_err(b.last_weights()[0], o["weights"]))
    return o


def _assert_worst(worst, label):
    msg = f"{label}: " + ", ".join(f"{k} {v:.2e}" for k, v in worst.items())
    print(msg)
    assert worst["u"] <= TOL_U, msg
    assert worst["w"] <= TOL_W, msg
    assert worst["ess"] <= TOL_ESS, msg
    assert worst["best"] <= 1e-6, msg
    assert worst["mean"] <= 1e-5, msg


def test_single_agent_configuration_driver_steps(oracle):
    """Single-agent configuration exactly (seed 0, x0 = 0, control cost on,
    lambda 1) through MPPIDriver::step, five closed-loop steps."""
    w = models.unicycle_single(seed=0, K=1024, H=30)
    assert w.lam == 1.0 and w.control_cost and w.seed == 0
    drv = _driver(w, w.cost_params[0])
    b = backend_for(w)
    p = oracle_problem(w)
    n, m, HM = w.state_dim, w.control_dim, w.horizon * w.control_dim
    err = D.ErrorRef()
    x = w.x0[0].astype(np.float32)
    u_nom = np.zeros(HM, np.float32)
    worst = dict(u=0.0, w=0.0, ess=0.0, best=0.0, mean=0.0)
    for s in range(STEPS):
        u = np.zeros(HM, np.float32)
        diag = D.StepDiagnostics()
        assert drv.step(D.StepInputs(D.StateView(x, n)), D.MutableControlSequenceView(u, w.horizon, m),
                        diag, err), err.value
        dd = [diag.best_cost, diag.mean_cost, diag.effective_sample_size]
        _check_step(oracle, p, b, s, w.seed, x, u_nom, u, dd, worst)
        x = oracle.dynamics(p, x, u[:m]).astype(np.float32)
        u_nom = _shift(u, m)
    _assert_worst(worst, "single-agent configuration")


REF_FACTOR = 3.0


def _ref_kernels():
    if not pyoracle.ref_available("unicycle_obstacles"):
        pytest.skip("oracle/_ref (the reference kernels for the CPU) not built")
    return pyoracle.RefKernels("unicycle_obstacles")


def _assert_like_reference(worst, ref_worst, label):
    msg = (f"{label}: library " + ", ".join(f"{k} {v:.2e}" for k, v in worst.items()) +
           " | reference FP32 kernels " + ", ".join(f"{k} {v:.2e}" for k, v in ref_worst.items()))
    print(msg)
    bars = {"u": TOL_U, "w": TOL_W, "ess": TOL_ESS}
    for k, bar in bars.items():
        assert worst[k] <= max(bar, REF_FACTOR * ref_worst[k]), msg


@pytest.mark.parametrize("agent", [0, 1, 2, 3])
def test_batched_configuration_agents_step_by_step(oracle, agent):
    """Agents of the batched configuration (K 4096, H 50, 16 moving
    obstacles, their own sigma and key seed + agent), lambda 1; each step
    also through the reference's FP32 kernels on the same inputs."""
    ref = _ref_kernels()
    wb = models.unicycle_batch(seed=0, N=4, K=4096, H=50, T=STEPS)
    assert wb.lam == 1.0
    w = models.Workload(wb.name, wb.plugin, wb.oracle_model, wb.state_dim, wb.control_dim,
                        wb.horizon, wb.sample_count, wb.lam, wb.agent_sigma[agent],
                        (1.0 / wb.agent_sigma[agent] ** 2).astype(np.float32), wb.u_min, wb.u_max,
                        1, STEPS, wb.x0[agent:agent + 1], wb.model_params,
                        [wb.cost_params[agent]], None, seed=wb.seed + agent)
    b = backend_for(w)
    p = oracle_problem(w)
    m, HM = w.control_dim, w.horizon * w.control_dim
    x = w.x0[0].astype(np.float32)
    u_nom = np.zeros(HM, np.float32)
    worst = dict(u=0.0, w=0.0, ess=0.0, best=0.0, mean=0.0)
    ref_worst = dict(u=0.0, w=0.0, ess=0.0)
    b2 = backend_for(w)
    for s in range(STEPS):
        u, diag = b2.dispatch_rollout(s, x, u_nom)
        o = _check_step(oracle, p, b, s, w.seed, x, u_nom, u, diag, worst)
        r = ref.step(p, s, w.seed, x, u_nom, nthreads=8)
        ref_worst["u"] = max(ref_worst["u"], abs_err(r["u_out"], o["u_out"]))
        ref_worst["w"] = max(ref_worst["w"], abs_err(r["weights"], o["weights"]))
        ref_worst["ess"] = max(ref_worst["ess"], rel_err([r["diag"][2]], [o["diag"][2]]))
        x = oracle.dynamics(p, x, u[:m]).astype(np.float32)
        u_nom = _shift(u, m)
    assert worst["best"] <= 1e-5 and worst["mean"] <= 1e-5, worst  # per-sample cost bar
    _assert_like_reference({k: worst[k] for k in ("u", "w", "ess")}, ref_worst,
                           f"batched configuration, agent {agent}")


def test_batched_configuration_closed_loop_matches_oracle(oracle):
    """The batch closed loop itself (one launch per step, propagate and warm
    start on the device) for 8 agents x 5 steps against the oracle's batch
    closed loop: the device propagates in FP32, the oracle in FP64, so the
    trajectories may part by rounding only."""
    ref = _ref_kernels()
    w = models.unicycle_batch(seed=0, N=8, K=4096, H=50, T=STEPS)
    b = backend_for(w)
    p = oracle_problem(w)
    r = b.simulate_batch(w.num_agents, STEPS, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    o = oracle.simulate_batch(p, w.num_agents, STEPS, 0, w.seed, w.x0,
                              cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride,
                              sigma_packed=w.agent_sigma.astype(float))
    rr = ref.simulate_batch(p, w.num_agents, STEPS, 0, w.seed, w.x0, sigma_packed=w.agent_sigma,
                            cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride,
                            model_params_packed=w.model_params, model_stride=0, nthreads=8)
    lib = {"u": abs_err(r["controls"], o["controls"]), "x": abs_err(r["states"], o["states"])}
    refe = {"u": abs_err(rr["controls"], o["controls"]), "x": abs_err(rr["states"], o["states"])}
    print(f"batch closed loop: library controls {lib['u']:.2e}, states {lib['x']:.2e} | "
          f"reference FP32 kernels controls {refe['u']:.2e}, states {refe['x']:.2e}")
    for k in lib:
        assert lib[k] <= max(TOL_U, REF_FACTOR * refe[k]), (lib, refe)


@pytest.mark.skipif(not pyoracle.ref_available("unicycle_obstacles"),
                    reason="oracle/_ref (the reference kernels for the CPU) not built")
def test_batched_configuration_cost_matches_reference_kernels():
    """Executed closed-loop cost of 16 agents x 2 steps of the batched
    configuration: the library on the GPU against the reference's own
    kernels (FP32, CPU) on the same agents, seeds and steps."""
    from mppi_metal_b200 import models as M
    w = M.unicycle_batch(seed=1000, N=16, K=4096, H=50, T=2)
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, 2, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride, sigma=w.agent_sigma)
    ref = pyoracle.RefKernels("unicycle_obstacles")
    p = oracle_problem(w)
    rr = ref.simulate_batch(p, w.num_agents, 2, 0, w.seed, w.x0, sigma_packed=w.agent_sigma,
                            cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride,
                            model_params_packed=w.model_params, model_stride=0, nthreads=4)
    gpu = M.unicycle_executed_cost(r["states"], r["controls"], r["terminal"], w.cost_params)
    cpu = M.unicycle_executed_cost(rr["states"], rr["controls"], rr["terminal"], w.cost_params)
    per_agent = float(np.max(np.abs(gpu - cpu) / np.abs(cpu)))
    mean_gap = abs(gpu.mean() - cpu.mean()) / abs(cpu.mean())
    print(f"executed cost vs reference kernels: per agent {per_agent:.2e}, mean {mean_gap:.2e}")
    assert per_agent <= 1e-5
    assert mean_gap <= 1e-6
