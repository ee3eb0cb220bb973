"""The multi-process path on CPU (gloo, world size 2): agent sharding with
no data-path collective, the barrier, and the max-over-ranks timing that
bench.py reports.  Two spawned processes rendezvous on 127.0.0.1."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    from mppi_metal_b200 import dist
    R = dist.env()
    dist.init(R, "gloo", timeout_s=60)
    import bench
    import pyoracle
    w = bench.workload_for_rank(R.rank, "batch")
    # the data path of a rank touches only its own agents: a short closed
    # loop of its first agent on the CPU restatement, no collective
    from mppi_metal_b200 import models  # noqa: F401
    p = pyoracle.Problem(w.oracle_model, 4, 2, 8, 64, w.lam, w.agent_sigma[0].astype(float),
                         w.u_min.astype(float), w.u_max.astype(float),
                         model_params=w.model_params, cost_params=w.cost_params[0])
    r = pyoracle.Oracle().simulate(p, 3, 0, w.seed, w.x0[0], np.zeros(16))
    dist.barrier(R)
    t = 1.0 + R.rank  # this rank's "device time"
    q.put({"rank": R.rank, "seed": w.seed, "x0": w.x0[:3].tolist(),
           "traj": r["states"].tolist(), "max": dist.max_over_ranks(R, t),
           "rate": dist.aggregate_rate(R, 100.0, t),
           "shard": list(dist.shard(257, R))})
    dist.barrier(R)
    dist.finish(R)


def test_two_ranks_shard_agents_and_reduce_times():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        d = q.get(timeout=240)
        out[d["rank"]] = d
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = out[0], out[1]
    assert a["seed"] != b["seed"] and a["x0"] != b["x0"]      # disjoint agent sets
    assert a["traj"] != b["traj"]                             # independent data paths
    assert a["max"] == b["max"] == 2.0                        # max over ranks
    assert a["rate"] == b["rate"] == 100.0                    # 2 ranks x 100 units / 2 s
    assert a["shard"] + b["shard"] == list(range(257))        # contiguous, complete
    assert len(a["shard"]) == 129 and len(b["shard"]) == 128


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def _library_worker(rank: int, world: int, port: int, q) -> None:
    """A rank of the weak-scaling path on the library: its own agents (seed
    per rank), one batch closed loop on cuda:0, gloo for the barrier and the
    max over ranks only."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT / "oracle"))
    from mppi_metal_b200 import dist, models
    from helpers import backend_for
    R = dist.env()
    dist.init(R, "gloo", timeout_s=120)
    w = models.unicycle_batch(seed=dist.agent_seed(500, R), N=4, K=512, H=16, T=3)
    b = backend_for(w)
    b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
              cost_stride=w.cost_stride, sigma=w.agent_sigma)
    dist.barrier(R)
    b.run(0)
    ms = b.last_run_ms()
    r = b.fetch()
    dist.barrier(R)
    q.put({"rank": R.rank, "controls": r["controls"].tolist(), "ms": ms,
           "max_ms": dist.max_over_ranks(R, ms)})
    dist.barrier(R)
    b.close()
    dist.finish(R)


@pytest.mark.gpu
def test_two_ranks_run_the_library_on_their_own_agents():
    # both ranks share this run's one GPU: their kernels are independent
    # replicas (no rank waits on another's kernel); the host-side gloo group
    # carries only the barrier and the max of the device times
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_library_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        d = q.get(timeout=600)
        out[d["rank"]] = d
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0]["max_ms"] == out[1]["max_ms"] == max(out[0]["ms"], out[1]["ms"])
    # each rank's results are the single-process results of the same agents
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import backend_for
    from mppi_metal_b200 import models
    for rank in (0, 1):
        w = models.unicycle_batch(seed=500 + rank, N=4, K=512, H=16, T=3)
        r = backend_for(w).simulate_batch(w.num_agents, w.num_steps, 0, w.x0,
                                          cost_params=w.cost_params_packed,
                                          cost_stride=w.cost_stride, sigma=w.agent_sigma)
        assert np.array_equal(np.asarray(out[rank]["controls"], np.float32), r["controls"])
    assert out[0]["controls"] != out[1]["controls"]
