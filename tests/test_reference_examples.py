"""The reference's example applications (examples/*/main.cpp of
MarshallVielmetti/mppi_metal), compiled unchanged against this project's
headers and libmppi_b200.so (oracle/Makefile target `ref_examples`; the
binaries travel with the tree).  Each must run to completion on the B200
backend and write the reference's trajectory CSV format
(sim_id,step,x,y,theta,v,a_cmd,omega_cmd,best_cost), which the reference's
plotting script reads.  The concurrent example runs one driver per host
thread (the reference's concurrency model) on per-driver CUDA streams."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

EX = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "examples"
HEADER = "sim_id,step,x,y,theta,v,a_cmd,omega_cmd,best_cost"

pytestmark = pytest.mark.gpu


def _run(name: str, cwd: Path) -> str:
    exe = EX / name
    if not exe.exists():
        pytest.skip(f"{name} not built (make -C oracle ref_examples)")
    r = subprocess.run([str(exe)], cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def _csv(path: Path) -> np.ndarray:
    lines = path.read_text().splitlines()
    assert lines[0] == HEADER
    data = np.genfromtxt(path, delimiter=",", skip_header=1)
    assert data.ndim == 2 and data.shape[1] == 9
    assert np.all(np.isfinite(data))
    return data


def test_batch_example(tmp_path):
    out = _run("nonholonomic_vehicle_batch", tmp_path)
    data = _csv(tmp_path / "trajectory_batch.csv")
    sims = np.unique(data[:, 0])
    assert len(sims) == 512
    m = re.search(r"(\d+)/512 agents reached the goal", out)
    assert m, out[-500:]
    # bounds of the example's controls: |a| <= 3, |omega| <= 1.5
    assert np.all(np.abs(data[:, 6]) <= 3.0 + 1e-4) and np.all(np.abs(data[:, 7]) <= 1.5 + 1e-4)


@pytest.mark.parametrize("name", ["nonholonomic_vehicle", "nonholonomic_vehicle_concurrent"])
def test_single_and_concurrent_examples(tmp_path, name):
    # both programs run 1000 simulations (their loop bound), one driver per
    # host thread, and log every one of them
    out = _run(name, tmp_path)
    data = _csv(tmp_path / "trajectory.csv")
    assert len(np.unique(data[:, 0])) == 1000
    assert len(re.findall(r"Finished simulation \d+", out)) == 1000
