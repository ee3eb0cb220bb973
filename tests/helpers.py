"""Builders shared by the tests: one problem description feeds the CUDA
backend (product) and the FP64 oracle (checker)."""
from __future__ import annotations

import numpy as np

import pyoracle
from mppi_metal_b200 import models
from mppi_metal_b200.backend import Backend


def oracle_problem(w: models.Workload, use_stage=True, use_terminal=True,
                   cost_params: bytes | None = None) -> pyoracle.Problem:
    return pyoracle.Problem(
        w.oracle_model, w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam,
        np.asarray(w.sigma, np.float64), np.asarray(w.u_min, np.float64),
        np.asarray(w.u_max, np.float64), sigma_inv=np.asarray(w.sigma_inv, np.float64),
        cov_full=w.cov_full, control_cost=w.control_cost, use_stage=use_stage,
        use_terminal=use_terminal, noise_half=w.numeric_mode != 0, model_params=w.model_params,
        cost_params=cost_params if cost_params is not None
        else (w.cost_params[0] if w.cost_params else b""))


def backend_for(w: models.Workload, use_stage=True, use_terminal=True, bind=True,
                seed: int | None = None) -> Backend:
    b = Backend(w.plugin, w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam,
                w.sigma, w.u_min, w.u_max, sigma_inv=w.sigma_inv, cov_full=w.cov_full,
                control_cost=w.control_cost,
                stage_cost="mppi_stage_cost" if use_stage else "",
                terminal_cost="mppi_terminal_cost" if use_terminal else "",
                model_params_size=len(w.model_params),
                cost_params_size=len(w.cost_params[0]) if w.cost_params else 0,
                seed=w.seed if seed is None else seed, numeric_mode=w.numeric_mode)
    if bind and (w.model_params or w.cost_params):
        b.bind_params(w.model_params or None, w.cost_params[0] if w.cost_params else None)
    return b


def nonholonomic_example(K=256, H=20) -> models.Workload:
    """The reference example's problem (examples/nonholonomic_vehicle_batch/main.cpp:24-91)."""
    mp = models.NonholonomicModelParams(2.0, 0.05)
    cp = models.NonholonomicCostParams(5.0, 5.0, 0.2, 10.0, 0.0, 0.1)
    return models.Workload(
        "nonholonomic_example", "nonholonomic_vehicle", "nonholonomic_vehicle", 4, 2, H, K,
        1.0, np.array([2.0, 1.0], np.float32), np.array([0.5, 1.0], np.float32),
        np.array([-3.0, -1.5], np.float32), np.array([3.0, 1.5], np.float32), 1, 5,
        np.zeros((1, 4), np.float32), models.blob(mp), [models.blob(cp)], None)


def rel_err(a, b, floor=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def abs_err(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))
