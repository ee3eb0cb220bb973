"""Generates the golden vectors in tests/golden/ from the REFERENCE's own code.

The reference's shader sources (shaders/philox.h, shaders/mppi_rollout.metal,
shaders/mppi_reduce.metal) and plugins compile as C++ through
oracle/ref_shim and run on the CPU as oracle/_ref/libmppi_ref_<plugin>.so
(see oracle/Makefile).  This script drives them through oracle/pyoracle.py
and stores their outputs, so the FP64 oracle and the GPU path are pinned to
what the reference computes, on machines where the reference tree is absent.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))

from pyoracle import Problem, RefKernels  # noqa: E402

from mppi_metal_b200 import models  # noqa: E402

OUT = Path(__file__).resolve().parent


def philox_cases():
    rng = np.random.default_rng(1234)
    edge = np.array([
        [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1],
        [0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF], [0x80000000, 0x80000000, 0],
        [7, 0x80000000 + 3, 42], [123456789, 987654321, 0xDEADBEEF],
    ], dtype=np.uint32)
    rand = rng.integers(0, 2 ** 32, size=(248, 3), dtype=np.uint64).astype(np.uint32)
    return np.concatenate([edge, rand])


def problem_of(w: models.Workload, use_stage=True, use_terminal=True, K=None, H=None) -> Problem:
    return Problem(w.oracle_model, w.state_dim, w.control_dim, H or w.horizon,
                   K or w.sample_count, w.lam, np.asarray(w.sigma, np.float64),
                   np.asarray(w.u_min, np.float64), np.asarray(w.u_max, np.float64),
                   sigma_inv=np.asarray(w.sigma_inv, np.float64), use_stage=use_stage,
                   use_terminal=use_terminal, model_params=w.model_params,
                   cost_params=w.cost_params[0] if w.cost_params else b"")


def main() -> None:
    # ---- Philox words and Box-Muller pairs (shaders/philox.h) ---------------
    ref = RefKernels("double_integrator")
    cases = philox_cases()
    words = ref.philox(cases[:, 0], cases[:, 1], cases[:, 2])
    normals = ref.box_muller(words)
    np.savez_compressed(OUT / "philox_ref.npz", ctr0=cases[:, 0], ctr1=cases[:, 1],
                        key=cases[:, 2], words=words, normals=normals)

    # ---- one control step, reference test fixture (double integrator) ------
    w = models.double_integrator_test()
    p = problem_of(w, use_stage=True, use_terminal=False)
    x0 = w.x0[0]
    un = np.zeros(w.horizon * w.control_dim, np.float32)
    r = ref.step(p, 0, 0, x0, un)
    sim = ref.simulate(p, 5, 0, 0, x0, un)
    x0b = np.array([[1, 1, 0, 0], [-1, 1, 0, 0], [1, -1, 0, 0], [-1, -1, 0, 0]], np.float32)
    simb = ref.simulate_batch(p, 4, 5, 0, 0, x0b)
    np.savez_compressed(OUT / "step_double_integrator.npz", x0=x0, u_nom=un, seed=0, step=0,
                        costs=r["costs"], weights=r["weights"], u_out=r["u_out"],
                        diag=r["diag"], sim_states=sim["states"], sim_controls=sim["controls"],
                        sim_costs=sim["costs"], batch_x0=x0b, batch_states=simb["states"],
                        batch_controls=simb["controls"], batch_costs=simb["costs"],
                        batch_terminal=simb["terminal"])

    # ---- the reference example model (nonholonomic vehicle, K 256, H 20) ----
    refn = RefKernels("nonholonomic_vehicle")
    mp = models.NonholonomicModelParams(2.0, 0.05)
    cp = models.NonholonomicCostParams(5.0, 5.0, 0.2, 10.0, 0.0, 0.1)
    pn = Problem("nonholonomic_vehicle", 4, 2, 20, 256, 1.0, np.array([2.0, 1.0]),
                 np.array([-3.0, -1.5]), np.array([3.0, 1.5]), sigma_inv=np.array([0.5, 1.0]),
                 model_params=models.blob(mp), cost_params=models.blob(cp))
    x0n = np.zeros(4, np.float32)
    un = np.zeros(40, np.float32)
    rn = refn.step(pn, 3, 7, x0n, un)
    simn = refn.simulate(pn, 6, 0, 7, x0n, un)
    np.savez_compressed(OUT / "step_nonholonomic.npz", x0=x0n, u_nom=un, seed=7, step=3,
                        model_params=np.frombuffer(models.blob(mp), np.uint8),
                        cost_params=np.frombuffer(models.blob(cp), np.uint8),
                        costs=rn["costs"], weights=rn["weights"], u_out=rn["u_out"],
                        diag=rn["diag"], sim_states=simn["states"],
                        sim_controls=simn["controls"], sim_costs=simn["costs"])

    # ---- unicycle among obstacles (benchmark model, reference kernels) -----
    refu = RefKernels("unicycle_obstacles")
    wu = models.unicycle_single(seed=0, K=256, H=30)
    wu.lam = 50.0  # well-conditioned weights for a float-vs-double comparison
    pu = problem_of(wu)
    x0u = wu.x0[0]
    un = np.zeros(60, np.float32)
    ru = refu.step(pu, 0, 0, x0u, un)
    np.savez_compressed(OUT / "step_unicycle.npz", x0=x0u, u_nom=un, seed=0, step=0, lam=wu.lam,
                        K=256, H=30, model_params=np.frombuffer(wu.model_params, np.uint8),
                        cost_params=np.frombuffer(wu.cost_params[0], np.uint8),
                        costs=ru["costs"], weights=ru["weights"], u_out=ru["u_out"],
                        diag=ru["diag"])
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
