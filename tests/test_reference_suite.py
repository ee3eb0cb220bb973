"""The reference's behavioural test suite, test for test, on this backend.

Each test mirrors one function of the reference's tests/mppi_driver_tests.cpp
(named in its docstring) through the Python mirror of MPPIDriver, which
calls the C ABI (include/mppi_b200/mppi_driver_c.h) -> C++ MPPIDriver ->
CUDA backend.  Validation-only tests need no GPU (validation runs before the
backend is touched); the rest are marked gpu.  The test plugin is the CUDA
form of the reference's shaders/test_user_dynamics.metal.
"""
from __future__ import annotations

import numpy as np
import pytest

from mppi_metal_b200 import driver as D
from mppi_metal_b200._lib import plugin_path

TEST_PLUGIN = plugin_path("double_integrator")


class ValidConfigFixture:
    """tests/mppi_driver_tests.cpp:42-72."""

    def __init__(self):
        self.sigma = np.array([1.0, 1.0], np.float32)
        self.sigma_inv = np.array([1.0, 1.0], np.float32)
        self.u_min = np.array([-1.0, -1.0], np.float32)
        self.u_max = np.array([1.0, 1.0], np.float32)
        self.config = D.DriverConfig(
            state_dim=4, control_dim=2, horizon=10, sample_count=64, lambda_=1.0,
            noise=D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, self.sigma, self.sigma_inv, 2),
            bounds=D.ControlBounds(self.u_min, self.u_max, 2))


def make_initialized_driver(layout: D.ParamLayout | None = None, stage_cost: str = ""):
    """tests/mppi_driver_tests.cpp:448-465."""
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    model = D.ModelPluginSpec(TEST_PLUGIN, D.CallableNames(stage_cost=stage_cost),
                              layout or D.ParamLayout())
    err = D.ErrorRef()
    assert drv.initialize(model, err), err.value
    return drv


def _fail_init(mutate, needle: str | None):
    f = ValidConfigFixture()
    mutate(f)
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    assert not drv.initialize(D.ModelPluginSpec(), err)
    if needle is not None:
        assert needle in err.value


# ---- dimension validation (mppi_driver_tests.cpp:78-128) --------------------
def test_zero_state_dim():
    _fail_init(lambda f: setattr(f.config, "state_dim", 0), "state_dim")


def test_zero_control_dim():
    _fail_init(lambda f: setattr(f.config, "control_dim", 0), "control_dim")


def test_zero_horizon():
    _fail_init(lambda f: setattr(f.config, "horizon", 0), "horizon")


def test_zero_sample_count():
    _fail_init(lambda f: setattr(f.config, "sample_count", 0), "sample_count")


# ---- noise validation (:134-172) ---------------------------------------------
def test_noise_dim_mismatch():
    _fail_init(lambda f: setattr(f.config.noise, "control_dim", 99), "control_dim")


def test_null_sigma():
    _fail_init(lambda f: setattr(f.config.noise, "sigma", None), "sigma")


def test_null_sigma_inv():
    _fail_init(lambda f: setattr(f.config.noise, "sigma_inv", None), "sigma_inv")


# ---- bounds validation (:178-232) ---------------------------------------------
def test_bounds_dim_mismatch():
    _fail_init(lambda f: setattr(f.config.bounds, "control_dim", 99), "control_dim")


def test_null_u_min():
    _fail_init(lambda f: setattr(f.config.bounds, "u_min", None), "u_min")


def test_null_u_max():
    _fail_init(lambda f: setattr(f.config.bounds, "u_max", None), "u_max")


def test_u_min_greater_than_u_max():
    def m(f):
        f.config.bounds.u_min = np.array([-1.0, 5.0], np.float32)
        f.config.bounds.u_max = np.array([1.0, -5.0], np.float32)
    _fail_init(m, "u_min")


# ---- init against the backend (:238-338) ----------------------------------------
@pytest.mark.gpu
def test_valid_config_passes_validation():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    assert drv.initialize(D.ModelPluginSpec(TEST_PLUGIN), err), err.value


def test_null_error_pointer():
    f = ValidConfigFixture()
    f.config.state_dim = 0
    drv = D.MPPIDriver(f.config)
    assert not drv.initialize(D.ModelPluginSpec(), None)


@pytest.mark.gpu
def test_deep_copy_survives_source_destruction():
    cfg = D.DriverConfig(4, 2, 10, 64, 1.0)
    sigma = np.array([1.0, 1.0], np.float32)
    cfg.noise = D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, sigma, sigma.copy(), 2)
    cfg.bounds = D.ControlBounds(-np.ones(2, np.float32), np.ones(2, np.float32), 2)
    drv = D.MPPIDriver(cfg)
    # the source arrays are overwritten after construction
    cfg.noise.sigma[:] = np.nan
    cfg.bounds.u_min[:] = 5.0
    err = D.ErrorRef()
    assert drv.initialize(D.ModelPluginSpec(TEST_PLUGIN), err), err.value


def test_init_nonexistent_plugin():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    assert not drv.initialize(D.ModelPluginSpec("/nonexistent/path.cu"), err)


def test_init_empty_plugin_path():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    assert not drv.initialize(D.ModelPluginSpec(""), err)
    assert "empty" in err.value


def test_init_missing_dynamics_callable():
    """Needs no GPU here: the plugin is compiled (NVRTC) before the device is
    touched only when a device exists, so this runs on either machine; with
    a device the error names the missing callable."""
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    model = D.ModelPluginSpec(TEST_PLUGIN, D.CallableNames(dynamics="nonexistent_fn"))
    assert not drv.initialize(model, err)


@pytest.mark.gpu
def test_init_missing_dynamics_callable_names_it():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    err = D.ErrorRef()
    model = D.ModelPluginSpec(TEST_PLUGIN, D.CallableNames(dynamics="nonexistent_fn"))
    assert not drv.initialize(model, err)
    assert "nonexistent_fn" in err.value


# ---- reset (:344-441) ---------------------------------------------------------------
def test_reset_no_arg_succeeds():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    err = D.ErrorRef()
    assert drv.reset(error=err)


def test_reset_no_arg_null_error_pointer():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    assert drv.reset(None, None)


def test_reset_with_nominal_succeeds():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    view = D.ControlSequenceView(np.full(20, 0.5, np.float32), 10, 2)
    assert drv.reset(view, D.ErrorRef())


def test_reset_horizon_mismatch():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    err = D.ErrorRef()
    assert not drv.reset(D.ControlSequenceView(np.zeros(100, np.float32), 11, 2), err)
    assert "horizon" in err.value


def test_reset_control_dim_mismatch():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    err = D.ErrorRef()
    assert not drv.reset(D.ControlSequenceView(np.zeros(100, np.float32), 10, 3), err)
    assert "control_dim" in err.value


def test_reset_null_data_with_nonzero_dims():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    err = D.ErrorRef()
    assert not drv.reset(D.ControlSequenceView(None, 10, 2), err)
    assert "null" in err.value


def test_reset_null_error_pointer_with_bad_shape():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    assert not drv.reset(D.ControlSequenceView(None, 999, 999), None)


# ---- set_problem_params (:467-549) ------------------------------------------------
def test_set_params_before_init():
    drv = D.MPPIDriver(ValidConfigFixture().config)
    err = D.ErrorRef()
    assert not drv.set_problem_params(D.ProblemParams(), err)
    assert "not initialized" in err.value


@pytest.mark.gpu
def test_set_params_zero_layout_zero_params():
    drv = make_initialized_driver()
    err = D.ErrorRef()
    assert drv.set_problem_params(D.ProblemParams(), err), err.value


@pytest.mark.gpu
def test_set_params_model_size_mismatch():
    drv = make_initialized_driver(D.ParamLayout(model_params_size=16))
    assert not drv.set_problem_params(D.ProblemParams(D.ByteView.of(bytes(8))), D.ErrorRef())


@pytest.mark.gpu
def test_set_params_cost_size_mismatch():
    drv = make_initialized_driver(D.ParamLayout(cost_params_size=32))
    pp = D.ProblemParams(cost_params=D.ByteView.of(bytes(16)))
    assert not drv.set_problem_params(pp, D.ErrorRef())


@pytest.mark.gpu
def test_set_params_null_data_nonzero_bytes():
    drv = make_initialized_driver(D.ParamLayout(model_params_size=16))
    assert not drv.set_problem_params(D.ProblemParams(D.ByteView(None, 16)), D.ErrorRef())


@pytest.mark.gpu
def test_set_params_matching_layout():
    drv = make_initialized_driver(D.ParamLayout(model_params_size=16, cost_params_size=8))
    pp = D.ProblemParams(D.ByteView.of(bytes(16)), D.ByteView.of(bytes(8)))
    err = D.ErrorRef()
    assert drv.set_problem_params(pp, err), err.value


@pytest.mark.gpu
def test_set_params_layout_requires_but_zero_provided():
    drv = make_initialized_driver(D.ParamLayout(model_params_size=16))
    assert not drv.set_problem_params(D.ProblemParams(), D.ErrorRef())


# ---- step (:555-692) ---------------------------------------------------------------
def test_step_before_init():
    f = ValidConfigFixture()
    drv = D.MPPIDriver(f.config)
    u = np.zeros(20, np.float32)
    inputs = D.StepInputs(D.StateView(np.zeros(4, np.float32), 4))
    assert not drv.step(inputs, D.MutableControlSequenceView(u, 10, 2), D.StepDiagnostics(),
                        D.ErrorRef())


@pytest.mark.gpu
def test_step_null_x0():
    drv = make_initialized_driver()
    u = np.zeros(20, np.float32)
    assert not drv.step(D.StepInputs(D.StateView(None, 4)), D.MutableControlSequenceView(u, 10, 2),
                        None, D.ErrorRef())


@pytest.mark.gpu
def test_step_x0_dim_mismatch():
    drv = make_initialized_driver()
    u = np.zeros(20, np.float32)
    inputs = D.StepInputs(D.StateView(np.zeros(4, np.float32), 99))
    assert not drv.step(inputs, D.MutableControlSequenceView(u, 10, 2), None, D.ErrorRef())


@pytest.mark.gpu
def test_step_null_output():
    drv = make_initialized_driver()
    inputs = D.StepInputs(D.StateView(np.zeros(4, np.float32), 4))
    assert not drv.step(inputs, D.MutableControlSequenceView(None, 10, 2), None, D.ErrorRef())


@pytest.mark.gpu
def test_step_succeeds():
    drv = make_initialized_driver()
    u = np.full(20, -999.0, np.float32)
    err = D.ErrorRef()
    inputs = D.StepInputs(D.StateView(np.ones(4, np.float32), 4))
    assert drv.step(inputs, D.MutableControlSequenceView(u, 10, 2), D.StepDiagnostics(), err), \
        err.value
    assert np.all(u != -999.0)


@pytest.mark.gpu
def test_step_override_shape_mismatch():
    drv = make_initialized_driver()
    u = np.zeros(20, np.float32)
    inputs = D.StepInputs(D.StateView(np.zeros(4, np.float32), 4),
                          D.ControlSequenceView(np.zeros(100, np.float32), 99, 99))
    assert not drv.step(inputs, D.MutableControlSequenceView(u, 10, 2), None, D.ErrorRef())


@pytest.mark.gpu
def test_step_mppi_moves_toward_origin():
    drv = make_initialized_driver(stage_cost="mppi_stage_cost")
    u = np.zeros(20, np.float32)
    diag = D.StepDiagnostics()
    err = D.ErrorRef()
    inputs = D.StepInputs(D.StateView(np.array([1, 1, 0, 0], np.float32), 4))
    assert drv.step(inputs, D.MutableControlSequenceView(u, 10, 2), diag, err), err.value
    assert u[0] < 0.0 and u[1] < 0.0
    assert diag.best_cost > 0.0
    assert diag.mean_cost >= diag.best_cost
    assert diag.effective_sample_size > 0.0


@pytest.mark.gpu
def test_step_rng_determinism():
    d1 = make_initialized_driver(stage_cost="mppi_stage_cost")
    d2 = make_initialized_driver(stage_cost="mppi_stage_cost")
    u1 = np.zeros(20, np.float32)
    u2 = np.zeros(20, np.float32)
    inputs = D.StepInputs(D.StateView(np.array([1, 1, 0, 0], np.float32), 4))
    d1.step(inputs, D.MutableControlSequenceView(u1, 10, 2), None, None)
    d2.step(inputs, D.MutableControlSequenceView(u2, 10, 2), None, None)
    assert np.array_equal(u1, u2)


# ---- simulate (:694-811) -----------------------------------------------------------
@pytest.mark.gpu
def test_simulate_multi_step_parity():
    d1 = make_initialized_driver(stage_cost="mppi_stage_cost")
    d2 = make_initialized_driver(stage_cost="mppi_stage_cost")
    N, H, C, S = 5, 10, 2, 4
    x = np.array([1, 1, 0, 0], np.float32)
    hs, hc, hk = np.zeros((N, S)), np.zeros((N, C)), np.zeros(N)
    u = np.zeros(H * C, np.float32)
    for i in range(N):
        diag = D.StepDiagnostics()
        d1.step(D.StepInputs(D.StateView(x.copy(), S)), D.MutableControlSequenceView(u, H, C),
                diag, None)
        hs[i], hc[i], hk[i] = x, u[:C], diag.best_cost
        dt = np.float32(0.1)
        x = np.array([x[0] + x[2] * dt, x[1] + x[3] * dt, x[2] + u[0] * dt, x[3] + u[1] * dt],
                     np.float32)
    res = D.SimulationResults(np.zeros((N, S), np.float32), np.zeros((N, C), np.float32),
                              np.zeros(N, np.float32), N)
    err = D.ErrorRef()
    assert d2.simulate(N, D.StepInputs(D.StateView(np.array([1, 1, 0, 0], np.float32), S)), res,
                       err), err.value
    assert np.max(np.abs(hs - res.states_out)) <= 1e-4
    assert np.max(np.abs(hc - res.controls_out)) <= 1e-4
    assert np.max(np.abs(hk - res.costs_out)) <= 1e-4


@pytest.mark.gpu
def test_simulate_batch_parity():
    d1 = make_initialized_driver(stage_cost="mppi_stage_cost")
    d2 = make_initialized_driver(stage_cost="mppi_stage_cost")
    T, C, S = 5, 2, 4
    x0 = np.array([1, 1, 0, 0], np.float32)
    r1 = D.SimulationResults(np.zeros((T, S), np.float32), np.zeros((T, C), np.float32),
                             np.zeros(T, np.float32), T)
    err = D.ErrorRef()
    assert d1.simulate(T, D.StepInputs(D.StateView(x0, S)), r1, err), err.value
    r2 = D.BatchSimulationResults(np.zeros((T, 1, S), np.float32), np.zeros((T, 1, C), np.float32),
                                  np.zeros((T, 1), np.float32), None, 1, T)
    assert d2.simulate_batch(1, T, x0, r2, error=err), err.value
    assert np.max(np.abs(r1.states_out - r2.states_out[:, 0])) <= 1e-4
    assert np.max(np.abs(r1.controls_out - r2.controls_out[:, 0])) <= 1e-4
    assert np.max(np.abs(r1.costs_out - r2.costs_out[:, 0])) <= 1e-4


X0_FOUR = np.array([[1, 1, 0, 0], [-1, 1, 0, 0], [1, -1, 0, 0], [-1, -1, 0, 0]], np.float32)


@pytest.mark.gpu
def test_simulate_batch_multi_agent():
    drv = make_initialized_driver(stage_cost="mppi_stage_cost")
    N, T, C, S = 4, 5, 2, 4
    r = D.BatchSimulationResults(np.zeros((T, N, S), np.float32), np.zeros((T, N, C), np.float32),
                                 np.zeros((T, N), np.float32), None, N, T)
    err = D.ErrorRef()
    assert drv.simulate_batch(N, T, X0_FOUR, r, error=err), err.value
    first = r.states_out[0]
    assert all(not np.array_equal(first[a], first[0]) for a in range(1, N))
    assert np.all(r.costs_out > 0.0)


@pytest.mark.gpu
def test_simulate_batch_terminal_states_match_post_propagation_state():
    a = make_initialized_driver(stage_cost="mppi_stage_cost")
    b = make_initialized_driver(stage_cost="mppi_stage_cost")
    N, T, S = 3, 6, 4
    x0 = np.array([[1, 1, 0, 0], [-1.5, 0.5, 0, 0], [0.5, -1, 0, 0]], np.float32)
    term = np.zeros((N, S), np.float32)
    err = D.ErrorRef()
    assert a.simulate_batch(N, T, x0, D.BatchSimulationResults(terminal_states_out=term,
                                                               num_agents=N, num_steps=T),
                            error=err), err.value
    ext = np.zeros((T + 1, N, S), np.float32)
    assert b.simulate_batch(N, T + 1, x0, D.BatchSimulationResults(states_out=ext, num_agents=N,
                                                                   num_steps=T + 1), error=err)
    assert np.max(np.abs(ext[T] - term)) <= 1e-4


@pytest.mark.gpu
def test_simulate_batch_terminal_only_matches_reference():
    a = make_initialized_driver(stage_cost="mppi_stage_cost")
    b = make_initialized_driver(stage_cost="mppi_stage_cost")
    N, T, S = 4, 5, 4
    st = np.zeros((T, N, S), np.float32)
    t_ref = np.zeros((N, S), np.float32)
    err = D.ErrorRef()
    assert a.simulate_batch(N, T, X0_FOUR, D.BatchSimulationResults(st, None, None, t_ref, N, T),
                            error=err), err.value
    t_only = np.zeros((N, S), np.float32)
    assert b.simulate_batch(N, T, X0_FOUR, D.BatchSimulationResults(terminal_states_out=t_only,
                                                                    num_agents=N, num_steps=T),
                            error=err), err.value
    assert np.max(np.abs(t_ref - t_only)) <= 1e-4


@pytest.mark.gpu
def test_simulate_batch_all_optional_outputs_null_succeeds():
    drv = make_initialized_driver(stage_cost="mppi_stage_cost")
    x0 = np.array([[1, 0, 0, 0], [-1, 0, 0, 0]], np.float32)
    err = D.ErrorRef()
    assert drv.simulate_batch(2, 4, x0, D.BatchSimulationResults(num_agents=2, num_steps=4),
                              error=err), err.value


@pytest.mark.gpu
def test_simulate_batch_controls_and_costs_only():
    drv = make_initialized_driver(stage_cost="mppi_stage_cost")
    N, T, C = 3, 5, 2
    x0 = np.array([[1, 1, 0, 0], [-1, 1, 0, 0], [0, -1, 0, 0]], np.float32)
    ctl = np.zeros((T, N, C), np.float32)
    cst = np.zeros((T, N), np.float32)
    err = D.ErrorRef()
    assert drv.simulate_batch(N, T, x0, D.BatchSimulationResults(None, ctl, cst, None, N, T),
                              error=err), err.value
    assert np.all(ctl >= -1.0001) and np.all(ctl <= 1.0001)
    assert np.all(cst > 0.0)
