"""The checker itself, pinned before it is trusted (CPU only).

The FP64 oracle (oracle/mppi_oracle.c) is compared with the reference's own
kernels, which oracle/Makefile compiles from the reference's Metal sources
for the CPU; their outputs are committed as golden vectors in tests/golden/
(made by tests/golden/make_golden.py), so this runs wherever the reference
tree is absent too.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from helpers import abs_err, nonholonomic_example, oracle_problem, rel_err
from mppi_metal_b200 import models


def test_philox_words_bit_exact_against_reference(oracle, golden):
    g = golden("philox_ref.npz")
    assert np.array_equal(oracle.philox(g["ctr0"], g["ctr1"], g["key"]), g["words"])


def test_philox_known_value_of_reference_source(oracle):
    # philox2x32_10((0, 0), 0) from the reference's shaders/philox.h
    assert [hex(v) for v in oracle.philox([0], [0], [0])[0]] == ["0xff1dae59", "0x6cd10df2"]


def test_box_muller_against_reference(oracle, golden):
    # the reference evaluates theta = 2 pi u2 and the transcendentals in
    # float; the oracle in double: agreement to a few float ulps
    g = golden("philox_ref.npz")
    ours = oracle.box_muller(g["words"])
    assert abs_err(ours, g["normals"]) < 5e-6


def test_uniform_map_is_open_interval(oracle):
    lib = oracle.lib
    lib.oracle_uint_to_01.restype = __import__("ctypes").c_float
    lo = lib.oracle_uint_to_01(0)
    hi = lib.oracle_uint_to_01(0xFFFFFFFF)
    assert 0.0 < lo < 1e-9
    assert hi == 1.0  # float(2^32 - 1) rounds to 2^32, as in the reference


def test_step_double_integrator_against_reference(oracle, golden):
    g = golden("step_double_integrator.npz")
    w = models.double_integrator_test()
    o = oracle.step(oracle_problem(w, use_terminal=False), 0, 0, g["x0"], g["u_nom"])
    assert rel_err(o["costs"], g["costs"]) < 2e-6
    assert abs_err(o["weights"], g["weights"]) < 2e-6
    assert abs_err(o["u_out"], g["u_out"]) < 1e-5
    assert rel_err(o["diag"], g["diag"]) < 1e-5


def test_simulate_double_integrator_against_reference(oracle, golden):
    g = golden("step_double_integrator.npz")
    w = models.double_integrator_test()
    p = oracle_problem(w, use_terminal=False)
    o = oracle.simulate(p, 5, 0, 0, g["x0"], g["u_nom"])
    assert abs_err(o["states"], g["sim_states"]) < 1e-5
    assert abs_err(o["controls"], g["sim_controls"]) < 1e-5
    assert abs_err(o["costs"], g["sim_costs"]) < 1e-4
    ob = oracle.simulate_batch(p, 4, 5, 0, 0, g["batch_x0"])
    assert abs_err(ob["states"], g["batch_states"]) < 1e-5
    assert abs_err(ob["controls"], g["batch_controls"]) < 1e-5
    assert abs_err(ob["terminal"], g["batch_terminal"]) < 1e-5


def test_step_nonholonomic_against_reference(oracle, golden):
    g = golden("step_nonholonomic.npz")
    w = nonholonomic_example()
    p = oracle_problem(w)
    o = oracle.step(p, int(g["step"]), int(g["seed"]), g["x0"], g["u_nom"])
    assert rel_err(o["costs"], g["costs"]) < 1e-5
    assert abs_err(o["u_out"], g["u_out"]) < 1e-4
    s = oracle.simulate(p, 6, 0, int(g["seed"]), g["x0"], g["u_nom"])
    assert abs_err(s["controls"], g["sim_controls"]) < 1e-4


def test_step_unicycle_against_reference(oracle, golden):
    g = golden("step_unicycle.npz")
    w = models.unicycle_single(seed=0, K=int(g["K"]), H=int(g["H"]))
    w.lam = float(g["lam"])
    w.control_cost = False
    o = oracle.step(oracle_problem(w), 0, 0, g["x0"], g["u_nom"])
    assert rel_err(o["costs"], g["costs"]) < 1e-5
    assert abs_err(o["u_out"], g["u_out"]) < 1e-4


@pytest.mark.skipif(not pyoracle.ref_available("double_integrator"),
                    reason="oracle/_ref not built (needs the reference tree)")
def test_oracle_against_live_reference_kernels_random_inputs(oracle):
    """Fresh random problems through the reference's own kernels (FP32)."""
    ref = pyoracle.RefKernels("double_integrator")
    rng = np.random.default_rng(99)
    for trial in range(5):
        K, H = int(rng.integers(8, 300)), int(rng.integers(1, 25))
        w = models.double_integrator_test(K=K, H=H)
        p = oracle_problem(w, use_terminal=bool(trial % 2))
        x0 = rng.uniform(-2, 2, 4).astype(np.float32)
        un = rng.uniform(-1, 1, H * 2).astype(np.float32)
        step, seed = int(rng.integers(0, 1000)), int(rng.integers(0, 2 ** 32))
        a = oracle.step(p, step, seed, x0, un)
        b = ref.step(p, step, seed, x0, un)
        assert rel_err(a["costs"], b["costs"]) < 1e-5
        assert abs_err(a["u_out"], b["u_out"]) < 1e-4


def test_weights_properties(oracle):
    rng = np.random.default_rng(3)
    c = rng.uniform(0, 100, 1000)
    w, d = oracle.weights(c, 10.0)
    assert abs(w.sum() - 1.0) < 1e-12
    assert d[0] == c.min() and abs(d[1] - c.mean()) < 1e-9
    assert abs(d[2] - 1.0 / np.sum(w * w)) < 1e-9
    # shift invariance: adding a constant to every cost leaves the weights
    w2, _ = oracle.weights(c + 1234.5, 10.0)
    assert abs_err(w, w2) < 1e-12


def test_full_covariance_noise_has_requested_covariance(oracle):
    w = models.double_integrator_test(K=1, H=4000)
    cov = np.array([[0.30, 0.12], [0.12, 0.20]])
    p = oracle_problem(w)
    p.cov_full = True
    p.sigma = cov
    p.sigma_inv = np.linalg.inv(cov)
    _, e = oracle.noise(p, 0, 5, 0)
    emp = np.cov(e.T)
    assert np.max(np.abs(emp - cov)) < 0.03


def test_wez_oracle_carries_a_45_float_state(oracle):
    """The WEZ model's state (45 float slots: floats, a bool and per-adversary
    uint16 / bool fields) through the oracle's closed loop: the packed words
    keep valid fields (bools 0 / 1, step counters), and engagement zones
    switch on."""
    from mppi_metal_b200 import models
    w = models.wez_batch(seed=11, N=3, K=256, H=12, T=8)
    r = oracle.simulate_batch(oracle_problem(w), w.num_agents, w.num_steps, 0, w.seed, w.x0,
                              cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride)
    st = r["states"].astype(np.float32)
    adv_words = np.ascontiguousarray(st[..., [9 + 5 * i for i in range(models.WEZ_ADVERSARIES)]])
    bits = adv_words.view(np.uint32)
    assert np.all(((bits >> 16) & 0xFF) <= 1) and np.all((bits >> 24) <= 1)
    assert np.count_nonzero((bits >> 16) & 0xFF) > 0
    cont = [0, 1, 2, 3] + [5 + 5 * i + j for i in range(8) for j in range(4)]
    assert np.all(np.isfinite(st[..., cont]))
    # the first state is the workload's x0, bit for bit
    assert np.array_equal(st[0].view(np.uint32), w.x0.view(np.uint32))
