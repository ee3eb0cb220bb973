"""MPPI rollout throughput on B200 — one JSON line.

Workload (the batched configuration): 256 independent kinematic-unicycle
agents per GPU in one launch per pass, K = 4096 samples, horizon H = 50,
FP32, each agent with its own seeded start, goal, 16 moving circular
keep-out regions and per-dimension sigma U[0.2, 0.8]; 300 closed-loop
control steps.  One benchmark step = one such closed loop
(MPPIDriver::simulate_batch): 256 x 300 control steps of
rollout -> weights -> update -> propagate & shift.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload NAME] [--workloads all|none]

value : rollout-steps/s over all ranks, inputs resident in HBM (device
        time, CUDA events on the library's stream, max over ranks)
e2e   : the same metric through the public C ABI call with host buffers
        (host->device inputs and device->host histories inside the timing)
workloads : on one GPU the default line also carries every other
        configuration, each measured the same way (at most 5 timed loops):
        the single agent, the uneven bicycle batch, the quadrotor batch in
        FP32 and mixed mode, and the learned proposal against plain MPPI
        (unicycle K 256 / 1024 vs K 4096; quadrotor K 4096 vs K 65536) with
        its speed-up and closed-loop cost ratio.  --workload NAME measures
        one of them alone as the line.
--impl reference : the reference's own kernels (its Metal shader sources
        compiled for the CPU, oracle/_ref) on the host cores, on a bounded
        sample of the same workload.
Multi-GPU: agents are independent, so ranks run disjoint agent sets with no
collective on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import select
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "rollout-steps/s and control steps/s per B200 at matched closed-loop cost"
AGENTS_PER_GPU = 256
K_SAMPLES = 4096
HORIZON = 50
CLOSED_LOOP_STEPS = 300
L2_FLUSH_BYTES = 256 << 20

# Rollout-kernel instructions per rollout-step (warp-level instructions issued
# per sample-timestep, i.e. / 32 lanes) and DRAM bytes (read + write) per
# launch, from ncu captures of the same kernel builds (profiles/
# rollout_kernels_all_workloads.txt): smsp__inst_executed.sum / rollout-steps
# of the launch.  Used only to express the live-timed kernel against the SM
# issue-rate roofline.
ROLLOUT_COUNTERS = {
    # workload: (warp-inst per rollout-step, DRAM bytes per launch) of the
    # kernel rollout_kernel_name() names for the workload's launch shape
    "batch": (492249088 / 52428800, 267776),          # 9.39  mppi_rollout_early_b128
    "uneven": (182619694 / 16410677, 128085),         # 11.13 mppi_rollout_work_b128
    "single": (584832 / 30720, 51328),                # 19.04 mppi_rollout_coop32 (4 lanes/sample)
    "quadrotor/fp32": (6955357806 / 209715200, 235904),   # 33.17 mppi_rollout_b128
    "quadrotor/mixed": (6147972631 / 209715200, 438528),  # 29.32 mppi_rollout_b128 (16-bit uniforms)
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", choices=["full", "kernels"], default="full",
                    help="kernels: only launch the rollout and combine kernels of the "
                         "workload `--iters` times each (small capture target for ncu)")
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--workload", choices=WORKLOADS, default="batch",
                    help="batch (default, the headline configuration), uneven, single, "
                         "quadrotor, proposal, quadrotor_proposal")
    ap.add_argument("--numeric", choices=["fp32", "mixed"], default="fp32",
                    help="numeric mode of the quadrotor workload")
    ap.add_argument("--workloads", choices=["all", "none"], default="all",
                    help="with the default (batch) workload on one GPU: also measure every "
                         "other configuration and report them under `workloads`")
    ap.add_argument("--proposal-weights", default="",
                    help="proposal workload: load the network from this .npz instead of "
                         "training it on the GPU first (python -m mppi_metal_b200.proposal)")
    return ap.parse_args()


def dist_env():
    from mppi_metal_b200 import dist
    r = dist.env()
    return r.rank, r.world, r.local_rank


WORKLOADS = ("batch", "uneven", "single", "quadrotor", "proposal", "quadrotor_proposal")


def workload_for_rank(rank: int, name: str = "batch", numeric: str = "fp32"):
    """batch  : 256 unicycle agents per GPU, K 4096, H 50, 300 closed-loop steps
                (the headline configuration);
    uneven : 64 kinematic-bicycle instances per GPU, K log-uniform [1024, 16384],
                H log-uniform [16, 96], full 2x2 covariance, 100 closed-loop steps;
    single : one unicycle agent, K 1024, H 30, 8 static obstacles, control
                cost on, 200 closed-loop steps from x0 = 0, Philox seed 0;
    quadrotor : 32 quadrotors, n 12, m 4, dt 0.01, H 100, K 65536, 32
                spherical obstacles each, 20 closed-loop steps, in the numeric
                mode `numeric` (fp32, or mixed: FP16 noise)."""
    from mppi_metal_b200 import models
    if name == "quadrotor":
        w = models.quadrotor_batch(seed=3000 + rank, N=32, K=65536, H=100, T=20)
        w.numeric_mode = 2 if numeric == "mixed" else 0
        return w
    if name == "uneven":
        return models.bicycle_uneven(seed=2000 + rank, N=64, T=100)
    if name == "single":
        return models.unicycle_single(seed=0, K=1024, H=30, T=200)
    return models.unicycle_batch(seed=1000 + rank, N=AGENTS_PER_GPU, K=K_SAMPLES, H=HORIZON,
                                 T=CLOSED_LOOP_STEPS)


def agent_shapes(w):
    """(sample counts, horizons) per agent, or (None, None) for a uniform batch."""
    return getattr(w, "agent_K", None), getattr(w, "agent_H", None)


def rollout_steps_per_control_step(w) -> int:
    ks, hs = agent_shapes(w)
    if ks is None:
        return w.num_agents * w.sample_count * w.horizon
    return int(np.sum(ks.astype(np.int64) * hs.astype(np.int64)))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    # 20 ms between samples: the shortest timed regions (the proposal
    # workload's five 300-step loops) last about 0.1 s
    INTERVAL_MS = 20

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", str(self.INTERVAL_MS)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        # the sampler's start-up takes longer than a short timed region: wait
        # for its first sample (taken before the region, not counted)
        ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
        if ready:
            self.proc.stdout.readline()
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return False
        if not select.select([self.proc.stdout], [], [], 0)[0]:
            # a region shorter than the interval: the next sample, at most one
            # interval after its end, stands for it
            select.select([self.proc.stdout], [], [], 1.0)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)
        return False

    def summary(self) -> dict:
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s >= 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def physical_gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ---------------------------------------------------------------------------
# the reference's CPU implementation, bounded sample
# ---------------------------------------------------------------------------
def reference_sample_run(w, agents: int, steps: int, nthreads: int):
    """Runs `agents` x `steps` closed-loop control steps of the workload with
    the reference's kernels on the CPU; returns (seconds, rollout-steps,
    executed closed-loop cost of the sampled agents over those steps)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from mppi_metal_b200 import models
    ref = pyoracle.RefKernels("unicycle_obstacles")
    p = pyoracle.Problem("unicycle_obstacles", w.state_dim, w.control_dim, w.horizon,
                         w.sample_count, w.lam, w.sigma.astype(float), w.u_min.astype(float),
                         w.u_max.astype(float), sigma_inv=w.sigma_inv.astype(float),
                         model_params=w.model_params)
    blobs = w.cost_params[:agents]
    t0 = time.perf_counter()
    r = ref.simulate_batch(p, agents, steps, 0, w.seed, w.x0[:agents],
                           sigma_packed=w.agent_sigma[:agents],
                           cost_params_packed=b"".join(blobs), cost_stride=w.cost_stride,
                           model_params_packed=w.model_params, model_stride=0,
                           nthreads=nthreads)
    dt = time.perf_counter() - t0
    cost = models.unicycle_executed_cost(r["states"], r["controls"], r["terminal"], blobs)
    return dt, agents * steps * w.sample_count * w.horizon, float(cost.mean())


def choose_reference_sample(w, nthreads: int, target_s: float):
    """Sizes the CPU sample (agents at full K and H, 2 closed-loop steps) so one
    reference step takes about target_s seconds."""
    dt, rs, _ = reference_sample_run(w, 1, 1, nthreads)
    per_rs = dt / rs
    agents = int(max(1, min(AGENTS_PER_GPU, target_s / (per_rs * w.sample_count * w.horizon * 2))))
    return agents, 2


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    w = workload_for_rank(0)
    nthreads = os.cpu_count() or 1
    lib = ROOT / "oracle" / "_ref" / "libmppi_ref_unicycle_obstacles.so"
    if not lib.exists():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (the reference's kernels built for the CPU) is missing; "
                          "build it with `make -C oracle ref` where the reference tree exists"}))
        return 0
    agents, steps = choose_reference_sample(w, nthreads, target_s=4.0)
    for _ in range(args.warmup):
        reference_sample_run(w, agents, steps, nthreads)
    times, costs = [], []
    rs = 0
    for _ in range(args.steps):
        dt, rs, c = reference_sample_run(w, agents, steps, nthreads)
        times.append(dt)
        costs.append(c)
    total = sum(times)
    value = rs * len(times) / total
    sample = (f"{agents} of {AGENTS_PER_GPU} agents x {steps} of {CLOSED_LOOP_STEPS} closed-loop "
              f"steps at full K={K_SAMPLES}, H={HORIZON} per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rollout-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": config_block(),
        "control_steps_per_s": value / (K_SAMPLES * HORIZON),
        "closed_loop_cost": {"mean": float(np.mean(costs)), "agents": agents, "steps": steps},
        "cpu_baseline": {"value": value, "unit": "rollout-steps/s", "cores": nthreads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "rollout-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def config_block(name: str = "batch", w=None):
    if name == "quadrotor":
        return {
            "workload": ("quadrotor_batch: 32 quadrotors per GPU (n=12, m=4 rotor thrusts in "
                         "[0, 2*hover]), dt=0.01, H=100, K=65536, waypoint tracking + 32 "
                         "spherical obstacles, 20 closed-loop steps, numeric mode "
                         + ("mixed (fp16 noise)" if w.numeric_mode else "fp32")),
            "agents_per_gpu": 32, "samples": 65536, "horizon": 100, "closed_loop_steps": 20,
            "step": "one simulate_batch closed loop (20 control steps for every agent)",
            "l2": "flushed between timed iterations (256 MiB device write)",
            "parallelism": "agent-sharded replicas, no data-path collective",
        }
    if name == "uneven":
        return {
            "workload": ("bicycle_uneven: 64 kinematic-bicycle instances per GPU, K log-uniform "
                         "[1024,16384], H log-uniform [16,96], full 2x2 covariance per instance "
                         "(eigenvalues U[0.05,0.5]), cubic-spline lane keeping, 100 closed-loop "
                         "steps; one persistent launch per pass, autotuned"),
            "agents_per_gpu": w.num_agents, "rollout_steps_per_control_step":
                rollout_steps_per_control_step(w), "closed_loop_steps": w.num_steps,
            "step": "one simulate_batch closed loop (100 control steps for every agent)",
            "l2": "flushed between timed iterations (256 MiB device write)",
            "parallelism": "agent-sharded replicas, no data-path collective",
        }
    if name == "single":
        return {
            "workload": ("unicycle_single: 1 agent, K=1024, H=30, 8 static obstacles, control "
                         "cost on, 200 closed-loop steps from x0=0, Philox seed 0"),
            "agents_per_gpu": 1, "samples": 1024, "horizon": 30, "closed_loop_steps": 200,
            "step": "one simulate closed loop of 200 control steps",
            "l2": "flushed between timed iterations (256 MiB device write)",
            "parallelism": "replicas only",
        }
    return {
        "workload": (f"unicycle_batch: {AGENTS_PER_GPU} agents per GPU, K={K_SAMPLES}, H={HORIZON}, "
                     f"{CLOSED_LOOP_STEPS} closed-loop steps, 16 moving circular obstacles and "
                     "per-dimension sigma U[0.2,0.8] per agent, lambda=1, dt=0.05"),
        "agents_per_gpu": AGENTS_PER_GPU, "samples": K_SAMPLES, "horizon": HORIZON,
        "closed_loop_steps": CLOSED_LOOP_STEPS,
        "step": "one simulate_batch closed loop (300 control steps for every agent)",
        "l2": "flushed between timed iterations (256 MiB device write)",
        "parallelism": "agent-sharded replicas, no data-path collective",
    }


# ---------------------------------------------------------------------------
# the B200 path
# ---------------------------------------------------------------------------
class Ctx:
    """Rank plumbing shared by every measured workload of one run."""

    def __init__(self):
        import torch
        from mppi_metal_b200 import dist
        self.dist = dist
        self.R = dist.env()
        self.rank, self.world, self.local_rank = self.R.rank, self.R.world, self.R.local_rank
        torch.cuda.set_device(self.local_rank if self.world > 1 else 0)
        dist.init(self.R, "nccl", timeout_s=900)
        self.flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.gpu = physical_gpu_index(self.local_rank)

    def barrier(self):
        self.dist.barrier(self.R, "cuda")

    def max_over_ranks(self, x: float) -> float:
        return self.dist.max_over_ranks(self.R, x, "cuda")

    def flush_l2(self):
        import torch
        self.flush.zero_()
        torch.cuda.synchronize()

    def finish(self):
        self.dist.finish(self.R)


def load_peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def make_driver(w, K=None, options=None):
    """MPPIDriver for a workload through the public API (host buffers)."""
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200._lib import plugin_path
    form = D.CovarianceForm.kFull if w.cov_full else D.CovarianceForm.kDiagonal
    cfg = D.DriverConfig(w.state_dim, w.control_dim, w.horizon, K or w.sample_count, w.lam,
                         D.ControlNoiseConfig(form, w.sigma, w.sigma_inv, w.control_dim),
                         D.ControlBounds(w.u_min, w.u_max, w.control_dim),
                         D.NumericMode(w.numeric_mode))
    drv = D.MPPIDriver(cfg, options or D.DriverOptions(control_cost=w.control_cost))
    err = D.ErrorRef()
    spec = D.ModelPluginSpec(plugin_path(w.plugin),
                             D.CallableNames("mppi_dynamics", "mppi_stage_cost",
                                             "mppi_terminal_cost"),
                             D.ParamLayout(len(w.model_params), 4, w.cost_stride, 4),
                             D.RngConfig(w.seed))
    assert drv.initialize(spec, err), err.value
    assert drv.set_problem_params(D.ProblemParams(D.ByteView.of(w.model_params),
                                                  D.ByteView.of(w.cost_params[0])), err), err.value
    return drv


def timed_e2e(ctx, drv, w, agent_params, steps, warmup):
    """`steps` calls of MPPIDriver::simulate_batch with host buffers (x0, the
    per-agent blobs and sigma go up, the histories come down), after
    `warmup` untimed calls; returns (seconds, outputs of the last call)."""
    from mppi_metal_b200 import driver as D
    N, T = w.num_agents, w.num_steps
    err = D.ErrorRef()
    outs = D.BatchSimulationResults(np.zeros((T, N, w.state_dim), np.float32),
                                    np.zeros((T, N, w.control_dim), np.float32),
                                    np.zeros((T, N), np.float32),
                                    np.zeros((N, w.state_dim), np.float32), N, T)
    for _ in range(warmup):
        assert drv.reset(None, err)
        assert drv.simulate_batch(N, T, w.x0, outs, agent_params, err), err.value
    times = []
    ctx.barrier()
    for _ in range(steps):
        assert drv.reset(None, err)
        t0 = time.perf_counter()
        assert drv.simulate_batch(N, T, w.x0, outs, agent_params, err), err.value
        times.append(time.perf_counter() - t0)
    ctx.barrier()
    return ctx.max_over_ranks(sum(times)), outs


def e2e_bytes(w, ks=None):
    """Host<->device bytes of one simulate_batch call: x0, zero nominals,
    per-agent blobs and sigma up; state, control and cost histories and the
    terminal states down."""
    N, T, HM = w.num_agents, w.num_steps, w.horizon * w.control_dim
    sig_len = (w.control_dim * w.control_dim if w.cov_full else w.control_dim) \
        if w.agent_sigma is not None else 0
    h2d = (N * w.state_dim + N * HM + 4) * 4 + N * ((w.cost_stride + 15) // 16 * 16) \
        + N * sig_len * 4
    if ks is not None:
        work_items = int(sum((int(k) + 127) // 128 for k in ks))
        h2d += 12 * N + 8 * work_items  # per-agent K / H / offsets and the work list
    d2h = (T * N * (w.state_dim + w.control_dim + 1) + N * w.state_dim) * 4
    return h2d, d2h


def rollout_kernel_name(w, geom: dict, ragged: bool) -> str:
    """The rollout kernel the launch-time measurement runs (the form without
    the combine tail) for the prepared launch shape."""
    if ragged:
        return "mppi_rollout_work_b128"
    if geom["form"]["cooperative"]:
        return "mppi_rollout_coop32" if geom["block"] == 32 else "mppi_rollout_coop"
    if geom["block"] == 128 and geom["stage_rows"] >= w.horizon * w.control_dim:
        return "mppi_rollout_early_b128"  # whole horizon staged, no proposal: early noise
    return "mppi_rollout_b%d" % geom["block"]


def measure_workload(ctx, args, name: str, numeric: str, steps: int, warmup: int,
                     with_cpu: bool) -> dict:
    """One plain-MPPI workload: device-resident closed loops (value), the
    same through MPPIDriver::simulate_batch with host buffers (e2e), the
    rollout kernel's live launch time against the issue roofline, and (rank
    0, one GPU, the batched configuration) the reference's CPU kernels."""
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200 import models
    from mppi_metal_b200.backend import Backend

    w = workload_for_rank(ctx.rank, name, numeric)  # per-rank seed: disjoint agents
    N, T = w.num_agents, w.num_steps
    ks, hs = agent_shapes(w)
    rs_per_step = rollout_steps_per_control_step(w) * T  # per bench step (this rank)

    # ---- value: device-resident closed loop ---------------------------------
    b = Backend(w.plugin, w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam, w.sigma,
                w.u_min, w.u_max, sigma_inv=w.sigma_inv, cov_full=w.cov_full,
                control_cost=w.control_cost, model_params_size=len(w.model_params),
                cost_params_size=w.cost_stride, seed=w.seed, numeric_mode=w.numeric_mode)
    b.bind_params(w.model_params, w.cost_params[0])
    b.prepare(N, T, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              sigma=w.agent_sigma, sample_counts=ks, horizons=hs)
    for _ in range(warmup):
        b.run(0)
        b.last_run_ms()
    times = []
    ctx.barrier()
    with ClockSampler(ctx.gpu) as clocks:
        for _ in range(steps):
            ctx.flush_l2()
            b.run(0)
            times.append(b.last_run_ms())
    ctx.barrier()
    total_ms = ctx.max_over_ranks(sum(times))
    value = ctx.world * rs_per_step * steps / (total_ms / 1e3)

    # ---- kernel-level timing for the roofline --------------------------------
    rollout_ms, combine_ms = b.time_passes(20)
    geom = b.launch_info()
    tuning = b.tuning_info()
    b.close()

    # ---- e2e: public API, host buffers ---------------------------------------
    drv = make_driver(w)
    agent_params = D.BatchAgentParams(cost_params=w.cost_params_packed,
                                      cost_params_stride=w.cost_stride, sigma=w.agent_sigma,
                                      sample_counts=ks, horizons=hs)
    e2e_total, outs = timed_e2e(ctx, drv, w, agent_params, steps, warmup)
    # executed closed-loop cost of the last API call (from x0, step index 0)
    cost = models.executed_cost(w, outs.states_out, outs.controls_out, outs.terminal_states_out)
    e2e_value = ctx.world * rs_per_step * steps / e2e_total
    h2d, d2h = e2e_bytes(w, ks)

    # ---- CPU baseline (rank 0, N = 1 only) ------------------------------------
    cpu = None
    if with_cpu and ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        lib = ROOT / "oracle" / "_ref" / "libmppi_ref_unicycle_obstacles.so"
        if lib.exists():
            nthreads = os.cpu_count() or 1
            agents, csteps = choose_reference_sample(w, nthreads, target_s=5.0)
            dt, rs, c = reference_sample_run(w, agents, csteps, nthreads)
            # the GPU's executed cost on the same agents over the same steps
            gpu_c = models.unicycle_executed_cost(
                outs.states_out[:csteps, :agents], outs.controls_out[:csteps, :agents],
                outs.states_out[csteps, :agents], w.cost_params[:agents])
            dt1, rs1, _ = reference_sample_run(w, 2, 2, 1)
            cpu = {"value": rs / dt, "unit": "rollout-steps/s", "cores": nthreads,
                   "kind": "reference",
                   "sample": f"{agents} agents x {csteps} closed-loop steps at full "
                             f"K={K_SAMPLES}, H={HORIZON} (reference kernels compiled for the CPU)",
                   "closed_loop_cost_sample": c,
                   "gpu_closed_loop_cost_same_sample": float(gpu_c.mean()),
                   "one_core": {"value": rs1 / dt1, "unit": "rollout-steps/s",
                                "sample": "2 agents x 2 closed-loop steps, one thread"}}

    rollout_units = rollout_steps_per_control_step(w)  # rollout-steps per rollout launch
    kname = rollout_kernel_name(w, geom, ks is not None)
    key = name + ("/" + numeric if name == "quadrotor" else "")
    inst, dram = ROLLOUT_COUNTERS.get(key, (None, None))
    roof = {"kernel": kname, "bound": "issue",
            "launch_ms": rollout_ms, "combine_launch_ms": combine_ms,
            "rollout_steps_per_launch": rollout_units,
            "traffic": dram, "unit": "Gwarp-inst/s",
            "note": "issue-bound kernel (no HBM or tensor-core bound applies): "
                    "achieved = ncu-counted warp-instructions per rollout-step x "
                    "rollout-steps per launch / live CUDA-event launch time"}
    clk = clocks.summary()
    if inst is not None:
        achieved = inst * rollout_units / (rollout_ms / 1e3) / 1e9
        mhz = clk.get("sm_mhz") or 1965.0
        peak = 148 * 4 * mhz * 1e6 / 1e9
        roof.update({"achieved": achieved, "peak": peak, "frac": achieved / peak,
                     "warp_inst_per_rollout_step": inst,
                     "peak_basis": f"148 SMs x 4 warp-inst/clk x {mhz:.0f} MHz (sampled)"})
    return {
        "metric": METRIC, "value": value, "unit": "rollout-steps/s", "n_gpus": ctx.world,
        "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32" if w.numeric_mode == 0 else "fp32 (fp16 noise)",
        "data": "synthetic (seeded PCG64 workload generator, mppi_metal_b200/models.py)",
        "config": config_block(name, w),
        "control_steps_per_s": value * N / rollout_steps_per_control_step(w),
        "closed_loop_cost": {"mean": float(cost.mean()), "agents": N,
                             "mean_first_agents": float(cost[:8].mean())},
        "e2e": {"value": e2e_value, "unit": "rollout-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e2e_total / steps,
                "control_steps_per_s": e2e_value * N / rollout_steps_per_control_step(w)},
        "gpu_launches": geom["kernels_per_step"] * T * steps,
        "launch_geometry": geom,
        "autotuner": tuning or None,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
    }


def run_b200(args):
    ctx = Ctx()
    try:
        if args.workload in ("proposal", "quadrotor_proposal"):
            line = measure_proposal(ctx, args, args.workload, args.steps, args.warmup)
        else:
            line = measure_workload(ctx, args, args.workload, args.numeric, args.steps,
                                    args.warmup, with_cpu=args.workload == "batch")
            if args.workload == "batch" and args.workloads == "all" and ctx.world == 1:
                line["workloads"] = other_workloads(ctx, args)
        if ctx.rank == 0:
            print(json.dumps(line))
    finally:
        ctx.finish()
    return 0


# Keys of a workload's line kept in the headline line's `workloads` block.
SUMMARY_KEYS = ("value", "unit", "control_steps_per_s", "steps", "warmup", "ms_per_step",
                "dtype", "closed_loop_cost", "e2e", "gpu_launches", "roofline", "clocks",
                "launch_geometry", "autotuner", "plain", "speedup_vs_plain", "arms", "training",
                "kernel_ms_per_pass", "rollout_steps_per_s")


def summarise(line: dict) -> dict:
    out = {k: line[k] for k in SUMMARY_KEYS if k in line and line[k] is not None}
    out["workload"] = line["config"]["workload"]
    return out


def other_workloads(ctx, args) -> dict:
    """Every other configuration, each measured as its own `--workload` line
    would be (device-resident closed loops + the public API with host
    buffers), with at most 5 timed and 3 warm-up loops each, so the default
    run stays within a few minutes.  Runs on one GPU (the scaling runs
    measure the headline configuration)."""
    steps = max(1, min(args.steps, 5))
    warmup = 3
    out = {}
    for key, name, numeric in (("single", "single", "fp32"), ("uneven", "uneven", "fp32"),
                               ("quadrotor_fp32", "quadrotor", "fp32"),
                               ("quadrotor_mixed", "quadrotor", "mixed")):
        out[key] = summarise(measure_workload(ctx, args, name, numeric, steps, warmup,
                                              with_cpu=False))
    qf, qm = out["quadrotor_fp32"], out["quadrotor_mixed"]
    qm["vs_fp32"] = {"value": qm["value"] / qf["value"],
                     "closed_loop_cost": qm["closed_loop_cost"]["mean"]
                     / qf["closed_loop_cost"]["mean"]}
    for key in ("proposal", "quadrotor_proposal"):
        out[key] = summarise(measure_proposal(ctx, args, key, steps, warmup))
    return out

def run_kernels_only(args):
    """Prepares the workload and launches the rollout and combine kernels
    `iters` times each (no closed loop, no host copies in between).  For the
    proposal workload: a 3-step proposal closed loop (features, network,
    rollout, combine) with an untrained network, then one training step on
    8192 random rows (the network kernels' small capture target)."""
    if args.workload == "proposal":
        import torch
        from mppi_metal_b200 import models
        from mppi_metal_b200 import proposal as P
        torch.cuda.set_device(0)
        net = P.ProposalNet(P.UNICYCLE_FEATURES, PROPOSAL_H, 2, max_batch=8192, seed=0)
        w = models.unicycle_batch(seed=4000, N=PROPOSAL_AGENTS, K=PROPOSAL_K, H=PROPOSAL_H, T=3)
        r = P.closed_loop(w, net, PROPOSAL_SAMPLES, repeats=args.iters)
        x = torch.randn(8192, P.UNICYCLE_FEATURES, device="cuda")
        y = torch.randn(8192, PROPOSAL_H * 2, device="cuda")
        loss = net.train_step(x, y, lr=1e-3)
        print(json.dumps({"mode": "kernels", "workload": "proposal", "closed_loop_ms": r["ms"],
                          "train_loss": loss, "train_ms": net.last_train_ms()}))
        return 0
    from mppi_metal_b200.backend import Backend
    w = workload_for_rank(0, args.workload, args.numeric)
    ks, hs = agent_shapes(w)
    b = Backend(w.plugin, w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam, w.sigma,
                w.u_min, w.u_max, sigma_inv=w.sigma_inv, cov_full=w.cov_full,
                control_cost=w.control_cost, model_params_size=len(w.model_params),
                cost_params_size=w.cost_stride, seed=w.seed, numeric_mode=w.numeric_mode)
    b.bind_params(w.model_params, w.cost_params[0])
    b.prepare(w.num_agents, 1, w.x0, cost_params=w.cost_params_packed,
              cost_stride=w.cost_stride, sigma=w.agent_sigma, sample_counts=ks, horizons=hs)
    if ks is not None:
        b.run(0)  # the autotuner picks the persistent-launch geometry on the first run
    r, c = b.time_passes(args.iters)
    print(json.dumps({"mode": "kernels", "workload": args.workload, "rollout_ms": r,
                      "combine_ms": c, "geometry": b.launch_info(),
                      "tuning": b.tuning_info() or None}))
    return 0


# ---------------------------------------------------------------------------
# learned proposal vs plain MPPI
# ---------------------------------------------------------------------------
PROPOSAL_AGENTS = 128
PROPOSAL_K = 256
PROPOSAL_SAMPLES = 128
PROPOSAL_PLAIN_K = 4096
PROPOSAL_H = 64


def proposal_spec(name: str) -> dict:
    """proposal          : 128 unicycle agents x 300 steps, H 64; proposal-MPPI
                          K 256 (128 around the prediction) and K 1024 (512
                          around it) vs plain K 4096
    quadrotor_proposal : 32 quadrotors x 100 steps, H 100; proposal-MPPI K 4096
                          (1024 around the prediction, the network predicts 60
                          steps) vs plain K 65536"""
    from mppi_metal_b200 import models
    from mppi_metal_b200 import proposal as P
    if name == "quadrotor_proposal":
        return dict(agents=32, arms=[(4096, 1024)], plain_K=65536, H=100, T=100, net_H=60,
                    features=P.QUADROTOR_FEATURES, label="quadrotor",
                    make=lambda rank: models.quadrotor_batch(seed=4100 + rank, N=32, K=65536,
                                                             H=100, T=100),
                    train=P.train_quadrotor_proposal,
                    data="plain MPPI K=65536, H=100, 4 seeds x 256 agents x 100 steps",
                    desc="32 quadrotors per GPU (n=12, m=4, dt=0.01, 32 spherical obstacles)")
    return dict(agents=PROPOSAL_AGENTS, arms=[(PROPOSAL_K, PROPOSAL_SAMPLES), (1024, 512)],
                plain_K=PROPOSAL_PLAIN_K, H=PROPOSAL_H, T=CLOSED_LOOP_STEPS, net_H=PROPOSAL_H,
                features=P.UNICYCLE_FEATURES, label="unicycle",
                make=lambda rank: models.unicycle_batch(seed=4000 + rank, N=PROPOSAL_AGENTS,
                                                        K=PROPOSAL_PLAIN_K, H=PROPOSAL_H,
                                                        T=CLOSED_LOOP_STEPS),
                train=P.train_unicycle_proposal,
                data="plain MPPI K=16384, H=64, 4 seeds x 1024 agents x 300 steps",
                desc="128 unicycle agents per GPU (16 moving obstacles, sigma U[0.2,0.8])")


def net_roofline(per_agent: bool, flops: float, net_ms: float, rows: int, bf16_peak: float,
                 peaks: dict, mhz: float) -> dict:
    """The network pass of the proposal stage against its bound: the
    per-agent form (CUDA cores, one CTA per agent, BF16 weights streamed from
    L2) against the FP32 FMA rate, the tensor-core batch kernel against the
    measured BF16 peak."""
    achieved = flops / (net_ms / 1e3) / 1e12
    if per_agent:
        fma_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
        return {"kernel": "mppi_proposal_rows (per-agent network, CUDA cores)", "bound": "issue",
                "achieved": achieved, "peak": fma_peak, "unit": "TFLOP/s",
                "frac": achieved / fma_peak, "traffic": None,
                "note": f"{rows} agents, one CTA each; every CTA streams the 354 KB of BF16 "
                        "weights from L2 (latency-bound: four dependent layers per agent); "
                        f"peak = 148 SMs x 128 FP32 FMA/clk x 2 x {mhz:.0f} MHz; the dominant "
                        "kernel of the step is the rollout (issue-bound, see the batch workload)"}
    return {"kernel": "mlp_forward_cluster_kernel (proposal network forward)", "bound": "tensor",
            "achieved": achieved, "peak": bf16_peak, "unit": "TFLOP/s",
            "frac": achieved / bf16_peak, "traffic": None,
            "note": f"M = {rows} rows: 8-CTA clusters, latency-bound; the dominant kernel of the "
                    "step is the rollout (issue-bound, see the batch workload); peak = measured "
                    "bf16 burst" + ("" if peaks.get("bf16_tflops") else " (fallback)")}


def measure_proposal(ctx, args, name: str, steps: int, warmup: int) -> dict:
    """Proposal-MPPI against plain MPPI with more samples, on the same agents
    (proposal_spec).  value = control steps/s of the first proposal arm;
    every arm carries its rate, e2e, closed-loop cost and the ratios to the
    plain arm.  Setup (not timed): the network is trained on this GPU by the
    library's kernels on (features, u*) pairs from plain MPPI."""
    import torch  # noqa: F401  (CUDA context for the network's buffers)
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200 import models
    from mppi_metal_b200 import proposal as P
    spec = proposal_spec(name)

    t_setup = time.time()
    if args.proposal_weights and Path(args.proposal_weights).exists():
        net = P.ProposalNet.load(args.proposal_weights)
        training = {"loaded": args.proposal_weights}
    else:
        net, hist, pairs = spec["train"]()
        training = {"pairs": pairs, "epochs": len(hist), "final_loss": hist[-1],
                    "train_ms_per_step": net.last_train_ms(), "batch": 8192,
                    "data": spec["data"]}
    training["setup_s"] = round(time.time() - t_setup, 1)

    w = spec["make"](ctx.rank)
    N, T = w.num_agents, w.num_steps
    n, m, H = w.state_dim, w.control_dim, w.horizon

    def timed_arm(b):
        P._prepare(b, w)
        for _ in range(warmup):
            b.run(0)
            b.last_run_ms()
        times = []
        ctx.barrier()
        with ClockSampler(ctx.gpu) as clocks:
            for _ in range(steps):
                ctx.flush_l2()
                P._prepare(b, w)  # every timed loop starts from x0 and a zero nominal
                b.run(0)
                times.append(b.last_run_ms())
        ctx.barrier()
        r = b.fetch()
        cost = models.executed_cost(w, r["states"], r["controls"], r["terminal"])
        return ctx.max_over_ranks(sum(times)), cost, clocks.summary()

    plain = P.make_backend(w, spec["plain_K"])
    plain_ms, plain_cost, plain_clk = timed_arm(plain)
    plain_form = plain.launch_info()
    plain.close()
    plain_value = ctx.world * N * T * steps / (plain_ms / 1e3)

    # network forward: 2 * rows * (32*256 + 2*256*256 + 256*P) FLOPs
    out_pad = (spec["net_H"] * m + m + 15) // 16 * 16
    mlp_flops = 2 * N * (32 * 256 + 2 * 256 * 256 + 256 * out_pad)
    peaks = load_peaks()
    bf16_peak = peaks.get("bf16_tflops") or 1590.0
    h2d, d2h = e2e_bytes(w)
    arms = []
    for K, KS in spec["arms"]:
        prop = P.make_backend(w, K)
        prop.set_features(P.FEATURES_CALLABLE, spec["features"])
        prop.set_proposal(net, KS)
        prop_ms, prop_cost, clk = timed_arm(prop)
        kernels_per_step = prop.launch_info()["kernels_per_step"]  # network + rollout(+combine)
        form = prop.launch_info()
        rollout_ms, combine_ms = prop.time_passes(20)
        feat_ms, net_ms = prop.time_proposal(20)
        per_agent = prop.proposal_stage()[2]
        prop.set_proposal(None)
        prop.close()
        value = ctx.world * N * T * steps / (prop_ms / 1e3)

        # ---- e2e: public API (DriverOptions.proposal), host buffers ----------
        drv = make_driver(w, K, D.DriverOptions(proposal=net, proposal_samples=KS))
        ap = D.BatchAgentParams(cost_params=w.cost_params_packed,
                                cost_params_stride=w.cost_stride, sigma=w.agent_sigma)
        e2e_total, outs = timed_e2e(ctx, drv, w, ap, steps, warmup)
        e2e_cost = models.executed_cost(w, outs.states_out, outs.controls_out,
                                        outs.terminal_states_out)
        del drv
        arms.append({
            "samples": K, "proposal_samples": KS,
            "value": value, "unit": "control-steps/s", "ms_per_step": prop_ms / steps,
            "rollout_steps_per_s": value * K * H,
            "closed_loop_cost": {"mean": float(prop_cost.mean()), "agents": N,
                                 "vs_plain": float(prop_cost.mean() / plain_cost.mean())},
            "speedup_vs_plain": value / plain_value,
            "e2e": {"value": ctx.world * N * T * steps / e2e_total, "unit": "control-steps/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1e3 * e2e_total / steps,
                    "closed_loop_cost_mean": float(e2e_cost.mean())},
            "gpu_launches": (kernels_per_step * T + 1) * steps,
            "launch_geometry": form,
            "kernel_ms_per_pass": {"rollout": rollout_ms, "combine": combine_ms,
                                   "features_kernel": feat_ms, "network": net_ms},
            "roofline": net_roofline(per_agent, mlp_flops, net_ms, N, bf16_peak, peaks,
                                     clk.get("sm_mhz") or 1965.0),
            "clocks": clk,
        })
    first = arms[0]
    arm_txt = " and ".join(f"K={a['samples']} ({a['proposal_samples']} around the prediction)"
                           for a in arms)
    return {
        "metric": METRIC, "value": first["value"], "unit": "control-steps/s",
        "n_gpus": ctx.world, "steps": steps, "warmup": warmup,
        "ms_per_step": first["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 rollout, bf16 network (fp32 accumulate)",
        "data": "synthetic (seeded PCG64 workload generator, mppi_metal_b200/models.py)",
        "config": {
            "workload": (f"{name}: {spec['desc']}, H={H}, {T} closed-loop steps; "
                         f"proposal-MPPI {arm_txt} against plain MPPI K={spec['plain_K']}"),
            "agents_per_gpu": N, "samples": first["samples"],
            "proposal_samples": first["proposal_samples"],
            "plain_samples": spec["plain_K"], "horizon": H, "closed_loop_steps": T,
            "network": (f"MLP {spec['features']}->256->256->256->{spec['net_H'] * m + m}, "
                        f"GELU, bf16 weights, fp32 accumulate; predicts {spec['net_H']} steps"),
            "step": f"one simulate_batch closed loop ({T} control steps for every agent)",
            "l2": "flushed between timed iterations (256 MiB device write)",
            "parallelism": "agent-sharded replicas, no data-path collective",
        },
        "rollout_steps_per_s": first["rollout_steps_per_s"],
        "plain": {"control_steps_per_s": plain_value, "samples": spec["plain_K"],
                  "ms_per_step": plain_ms / steps, "launch_geometry": plain_form,
                  "closed_loop_cost_mean": float(plain_cost.mean()), "clocks": plain_clk},
        "closed_loop_cost": first["closed_loop_cost"],
        "speedup_vs_plain": first["speedup_vs_plain"],
        "arms": arms,
        "training": training,
        "e2e": first["e2e"],
        "gpu_launches": sum(a["gpu_launches"] for a in arms),
        "kernel_ms_per_pass": first["kernel_ms_per_pass"],
        "roofline": first["roofline"],
        "clocks": first["clocks"],
    }


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "kernels":
        return run_kernels_only(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
