"""The WEZ plugin (plugins/wez_environment.cu): the reference's stochastic
example model (examples/wez_environment_batch/wez_environment.metal) with a
180-byte state -- 45 float slots holding floats, a bool and per-adversary
uint16 / bool fields -- beyond the reference's 128-byte state buffer, and
adversary activations drawn inside the dynamics from the callable's Philox
counter and key.

Checked against the FP64 oracle's restatement (ORACLE_MODEL_WEZ), which
carries the packed fields as the bits of their float slots:
  * per-sample costs of one step to 1e-5 relative, u_next to 1e-4;
  * batch closed loops: continuous state fields and controls to 1e-3 (the
    stochastic model's closed-loop bar), the packed fields (captured,
    activation, step counters) bit for bit;
  * the reference's example program, compiled unchanged, runs to completion
    on the library and writes its trajectory CSV.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import abs_err, backend_for, oracle_problem, rel_err
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu

# float slots of the state that hold floats (ego x, y, theta, v and each
# adversary's x, y, theta, v); the others hold packed integer / bool fields
CONT = np.array([i for i in range(models.WEZ_STATE_DIM) if i < 4 or (i >= 5 and (i - 5) % 5 < 4)])
PACKED = np.array([i for i in range(models.WEZ_STATE_DIM) if i not in set(CONT.tolist())])


def _activations(states: np.ndarray) -> int:
    bits = np.ascontiguousarray(states[..., PACKED[1:]], np.float32).view(np.uint32)
    return int(np.count_nonzero((bits >> 16) & 0xFF))


def test_wez_step_matches_oracle(oracle):
    w = models.wez_batch(seed=None, N=1, K=1024, H=20, T=1)
    b = backend_for(w)
    p = oracle_problem(w)
    x0 = w.x0[0]
    u_nom = (np.random.default_rng(3).normal(size=w.horizon * 2) * 0.5).astype(np.float32)
    for step in (0, 7):
        u, diag = b.dispatch_rollout(step, x0, u_nom)
        o = oracle.step(p, step, w.seed, x0, u_nom)
        assert rel_err(b.last_costs()[0], o["costs"]) <= 1e-5
        assert abs_err(u, o["u_out"]) <= 1e-4
        assert rel_err([diag[2]], [o["diag"][2]]) <= 1e-5


def test_wez_closed_loop_matches_oracle(oracle):
    w = models.wez_batch(seed=11, N=6, K=512, H=20, T=12)
    b = backend_for(w)
    r = b.simulate_batch(w.num_agents, w.num_steps, 0, w.x0, cost_params=w.cost_params_packed,
                         cost_stride=w.cost_stride)
    o = oracle.simulate_batch(oracle_problem(w), w.num_agents, w.num_steps, 0, w.seed, w.x0,
                              cost_params_packed=w.cost_params_packed, cost_stride=w.cost_stride)
    assert abs_err(r["states"][..., CONT], o["states"][..., CONT]) <= 1e-3
    assert abs_err(r["controls"], o["controls"]) <= 1e-3
    got = np.ascontiguousarray(r["states"][..., PACKED], np.float32).view(np.uint32)
    ref = np.ascontiguousarray(o["states"][..., PACKED].astype(np.float32)).view(np.uint32)
    assert np.array_equal(got, ref)
    assert _activations(r["states"]) > 0  # engagement zones really switch on


def test_wez_example_agents_diverge_by_key():
    # the example's agents are identical but for their key (seed + agent)
    w = models.wez_batch(seed=None, N=4, K=128, H=20, T=30)
    r = backend_for(w).simulate_batch(4, 30, 0, w.x0)
    assert not np.allclose(r["states"][-1, 0, :4], r["states"][-1, 1, :4])


EX = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "examples"


def test_wez_reference_example_runs(tmp_path):
    exe = EX / "wez_environment_batch"
    if not exe.exists():
        pytest.skip("wez_environment_batch not built (make -C oracle ref_examples)")
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    lines = (tmp_path / "trajectory_batch.csv").read_text().splitlines()
    header = lines[0].split(",")
    assert header[:10] == ["sim_id", "step", "x", "y", "theta", "v", "a_cmd", "omega_cmd",
                           "captured", "best_cost"]
    assert len(header) == 10 + 4 * models.WEZ_ADVERSARIES
    data = np.genfromtxt(tmp_path / "trajectory_batch.csv", delimiter=",", skip_header=1)
    # two runs of 256 agents x 100 steps
    assert data.shape == (2 * 256 * 100, len(header))
    assert np.all(np.isfinite(data))
    assert np.all(np.abs(data[:, 6]) <= 3.0 + 1e-4) and np.all(np.abs(data[:, 7]) <= 1.5 + 1e-4)
