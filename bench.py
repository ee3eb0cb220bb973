"""MPPI rollout throughput on B200 — one JSON line.

Workload (the batched configuration): 256 independent kinematic-unicycle
agents per GPU in one launch per pass, K = 4096 samples, horizon H = 50,
FP32, each agent with its own seeded start, goal, 16 moving circular
keep-out regions and per-dimension sigma U[0.2, 0.8]; 300 closed-loop
control steps.  One benchmark step = one such closed loop
(MPPIDriver::simulate_batch): 256 x 300 control steps of
rollout -> weights -> update -> propagate & shift.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value : rollout-steps/s over all ranks, inputs resident in HBM (device
        time, CUDA events on the library's stream, max over ranks)
e2e   : the same metric through the public C ABI call with host buffers
        (host->device inputs and device->host histories inside the timing)
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
    # workload: (warp-inst per rollout-step, DRAM bytes per launch)
    "batch": (496386048 / 52428800, 237568),          # 9.47
    "uneven": (178922783 / 16410677, 122880),         # 10.90
    "single": (247536 / 30720, 39680),                # 8.06
    "quadrotor/fp32": (6911910084 / 209715200, 153088),   # 32.96
    "quadrotor/mixed": (6401390457 / 209715200, 124416),  # 30.52
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
def run_b200(args):
    import torch
    from mppi_metal_b200 import dist
    R = dist.env()
    rank, world, local_rank = R.rank, R.world, R.local_rank
    torch.cuda.set_device(local_rank if world > 1 else 0)
    dist.init(R, "nccl", timeout_s=300)
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200 import models
    from mppi_metal_b200._lib import plugin_path
    from mppi_metal_b200.backend import Backend

    w = workload_for_rank(rank, args.workload, args.numeric)  # per-rank seed: disjoint agents
    N, T = w.num_agents, w.num_steps
    ks, hs = agent_shapes(w)
    rs_per_step = rollout_steps_per_control_step(w) * T  # per bench step (this rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        dist.barrier(R, "cuda")

    def max_over_ranks(x: float) -> float:
        return dist.max_over_ranks(R, x, "cuda")

    # ---- value: device-resident closed loop ---------------------------------
    b = Backend(w.plugin, w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam, w.sigma,
                w.u_min, w.u_max, sigma_inv=w.sigma_inv, cov_full=w.cov_full,
                control_cost=w.control_cost, model_params_size=len(w.model_params),
                cost_params_size=w.cost_stride, seed=w.seed, numeric_mode=w.numeric_mode)
    b.bind_params(w.model_params, w.cost_params[0])
    b.prepare(N, T, w.x0, cost_params=w.cost_params_packed, cost_stride=w.cost_stride,
              sigma=w.agent_sigma, sample_counts=ks, horizons=hs)
    for _ in range(args.warmup):
        b.run(0)
        b.last_run_ms()
    times = []
    barrier()
    with ClockSampler(physical_gpu_index(local_rank)) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            b.run(0)
            times.append(b.last_run_ms())
    barrier()
    total_ms = max_over_ranks(sum(times))
    value = world * rs_per_step * args.steps / (total_ms / 1e3)

    # ---- kernel-level timing for the roofline --------------------------------
    rollout_ms, combine_ms = b.time_passes(20)
    geom = b.launch_info()
    tuning = b.tuning_info()
    b.close()

    # ---- e2e: public API, host buffers ---------------------------------------
    form = D.CovarianceForm.kFull if w.cov_full else D.CovarianceForm.kDiagonal
    cfg = D.DriverConfig(w.state_dim, w.control_dim, w.horizon, w.sample_count, w.lam,
                         D.ControlNoiseConfig(form, w.sigma, w.sigma_inv, w.control_dim),
                         D.ControlBounds(w.u_min, w.u_max, w.control_dim),
                         D.NumericMode(w.numeric_mode))
    drv = D.MPPIDriver(cfg, D.DriverOptions(control_cost=w.control_cost))
    err = D.ErrorRef()
    spec = D.ModelPluginSpec(plugin_path(w.plugin),
                             D.CallableNames("mppi_dynamics", "mppi_stage_cost",
                                             "mppi_terminal_cost"),
                             D.ParamLayout(len(w.model_params), 4, w.cost_stride, 4),
                             D.RngConfig(w.seed))
    assert drv.initialize(spec, err), err.value
    assert drv.set_problem_params(D.ProblemParams(D.ByteView.of(w.model_params),
                                                  D.ByteView.of(w.cost_params[0])), err), err.value
    agent_params = D.BatchAgentParams(cost_params=w.cost_params_packed,
                                      cost_params_stride=w.cost_stride, sigma=w.agent_sigma,
                                      sample_counts=ks, horizons=hs)
    outs = D.BatchSimulationResults(np.zeros((T, N, w.state_dim), np.float32),
                                    np.zeros((T, N, w.control_dim), np.float32),
                                    np.zeros((T, N), np.float32),
                                    np.zeros((N, w.state_dim), np.float32), N, T)
    for _ in range(args.warmup):
        assert drv.reset(None, err)
        assert drv.simulate_batch(N, T, w.x0, outs, agent_params, err), err.value
    e2e_times = []
    barrier()
    for _ in range(args.steps):
        assert drv.reset(None, err)
        t0 = time.perf_counter()
        assert drv.simulate_batch(N, T, w.x0, outs, agent_params, err), err.value
        e2e_times.append(time.perf_counter() - t0)
    barrier()
    e2e_total = max_over_ranks(sum(e2e_times))
    # executed closed-loop cost of the last API call (from x0, step index 0)
    cost = models.executed_cost(w, outs.states_out, outs.controls_out,
                                outs.terminal_states_out)
    e2e_value = world * rs_per_step * args.steps / e2e_total
    HM = w.horizon * w.control_dim
    sig_len = w.control_dim * w.control_dim if w.cov_full else w.control_dim
    h2d = (N * w.state_dim + N * HM + 4) * 4 + N * ((w.cost_stride + 15) // 16 * 16) \
        + N * sig_len * 4
    if ks is not None:
        work_items = int(sum((int(k) + 127) // 128 for k in ks))
        h2d += 12 * N + 8 * work_items  # per-agent K / H / offsets and the work list
    d2h = (T * N * (w.state_dim + w.control_dim + 1) + N * w.state_dim) * 4

    # ---- CPU baseline (rank 0, N = 1 only) ------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "batch":
        lib = ROOT / "oracle" / "_ref" / "libmppi_ref_unicycle_obstacles.so"
        if lib.exists():
            nthreads = os.cpu_count() or 1
            agents, steps = choose_reference_sample(w, nthreads, target_s=5.0)
            dt, rs, c = reference_sample_run(w, agents, steps, nthreads)
            # the GPU's executed cost on the same agents over the same steps
            gpu_c = models.unicycle_executed_cost(
                outs.states_out[:steps, :agents], outs.controls_out[:steps, :agents],
                outs.states_out[steps, :agents], w.cost_params[:agents])
            dt1, rs1, _ = reference_sample_run(w, 2, 2, 1)
            cpu = {"value": rs / dt, "unit": "rollout-steps/s", "cores": nthreads,
                   "kind": "reference",
                   "sample": f"{agents} agents x {steps} closed-loop steps at full K={K_SAMPLES}, "
                             f"H={HORIZON} (reference kernels compiled for the CPU)",
                   "closed_loop_cost_sample": c,
                   "gpu_closed_loop_cost_same_sample": float(gpu_c.mean()),
                   "one_core": {"value": rs1 / dt1, "unit": "rollout-steps/s",
                                "sample": "2 agents x 2 closed-loop steps, one thread"}}

    if rank != 0:
        dist.finish(R)
        return 0

    rollout_units = rollout_steps_per_control_step(w)  # rollout-steps per rollout launch
    kname = "mppi_rollout_work_b128" if ks is not None else "mppi_rollout_b%d" % geom["block"]
    key = args.workload + ("/" + args.numeric if args.workload == "quadrotor" else "")
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
    line = {
        "metric": METRIC, "value": value, "unit": "rollout-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32" if w.numeric_mode == 0 else "fp32 (fp16 noise)",
        "data": "synthetic (seeded PCG64 workload generator, mppi_metal_b200/models.py)",
        "config": config_block(args.workload, w),
        "control_steps_per_s": value * N / rollout_steps_per_control_step(w),
        "closed_loop_cost": {"mean": float(cost.mean()), "agents": N,
                             "mean_first_agents": float(cost[:8].mean())},
        "e2e": {"value": e2e_value, "unit": "rollout-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e2e_total / args.steps},
        "gpu_launches": geom["kernels_per_step"] * T * args.steps,
        "launch_geometry": geom,
        "autotuner": tuning or None,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    print(json.dumps(line))
    dist.finish(R)
    return 0


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
                          K 256 (128 around the prediction) vs plain K 4096
    quadrotor_proposal : 32 quadrotors x 100 steps, H 100; proposal-MPPI K 4096
                          (1024 around the prediction, the network predicts 60
                          steps) vs plain K 65536"""
    from mppi_metal_b200 import models
    from mppi_metal_b200 import proposal as P
    if name == "quadrotor_proposal":
        return dict(agents=32, K=4096, samples=1024, plain_K=65536, H=100, T=100, net_H=60,
                    features=P.QUADROTOR_FEATURES, label="quadrotor",
                    make=lambda rank: models.quadrotor_batch(seed=4100 + rank, N=32, K=65536,
                                                             H=100, T=100),
                    train=P.train_quadrotor_proposal,
                    data="plain MPPI K=65536, H=100, 4 seeds x 256 agents x 100 steps",
                    desc="32 quadrotors per GPU (n=12, m=4, dt=0.01, 32 spherical obstacles)")
    return dict(agents=PROPOSAL_AGENTS, K=PROPOSAL_K, samples=PROPOSAL_SAMPLES,
                plain_K=PROPOSAL_PLAIN_K, H=PROPOSAL_H, T=CLOSED_LOOP_STEPS, net_H=PROPOSAL_H,
                features=P.UNICYCLE_FEATURES, label="unicycle",
                make=lambda rank: models.unicycle_batch(seed=4000 + rank, N=PROPOSAL_AGENTS,
                                                        K=PROPOSAL_PLAIN_K, H=PROPOSAL_H,
                                                        T=CLOSED_LOOP_STEPS),
                train=P.train_unicycle_proposal,
                data="plain MPPI K=16384, H=64, 4 seeds x 1024 agents x 300 steps",
                desc="128 unicycle agents per GPU (16 moving obstacles, sigma U[0.2,0.8])")


def run_proposal(args):
    """Proposal-MPPI against plain MPPI with 16x the samples, on the same
    agents (proposal_spec).  value = control steps/s of the proposal arm;
    the plain arm's rate and both closed-loop costs ride along.  Setup (not
    timed): the network is trained on this GPU by the library's kernels on
    (features, u*) pairs from plain MPPI."""
    import torch
    from mppi_metal_b200 import dist
    R = dist.env()
    rank, world, local_rank = R.rank, R.world, R.local_rank
    torch.cuda.set_device(local_rank if world > 1 else 0)
    dist.init(R, "nccl", timeout_s=900)
    from mppi_metal_b200 import driver as D
    from mppi_metal_b200 import models
    from mppi_metal_b200 import proposal as P
    from mppi_metal_b200._lib import plugin_path
    spec = proposal_spec(args.workload)

    def barrier():
        dist.barrier(R, "cuda")

    def max_over_ranks(x: float) -> float:
        return dist.max_over_ranks(R, x, "cuda")

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

    w = spec["make"](rank)
    N, T, K, KS = w.num_agents, w.num_steps, spec["K"], spec["samples"]
    n, m, H = w.state_dim, w.control_dim, w.horizon
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def timed_arm(b):
        P._prepare(b, w)
        for _ in range(args.warmup):
            b.run(0)
            b.last_run_ms()
        times = []
        barrier()
        with ClockSampler(physical_gpu_index(local_rank)) as clocks:
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                P._prepare(b, w)  # every timed loop starts from x0 and a zero nominal
                b.run(0)
                times.append(b.last_run_ms())
        barrier()
        r = b.fetch()
        cost = models.executed_cost(w, r["states"], r["controls"], r["terminal"])
        return max_over_ranks(sum(times)), cost, clocks.summary()

    plain = P.make_backend(w, spec["plain_K"])
    plain_ms, plain_cost, _ = timed_arm(plain)
    plain.close()
    prop = P.make_backend(w, K)
    prop.set_features(P.FEATURES_CALLABLE, spec["features"])
    prop.set_proposal(net, KS)
    prop_ms, prop_cost, clk = timed_arm(prop)
    kernels_per_step = prop.launch_info()["kernels_per_step"]  # network + rollout(+combine)
    rollout_ms, combine_ms = prop.time_passes(20)
    feat_ms, net_ms = prop.time_proposal(20)
    prop.set_proposal(None)
    prop.close()
    value = world * N * T * args.steps / (prop_ms / 1e3)
    plain_value = world * N * T * args.steps / (plain_ms / 1e3)

    # ---- e2e: public API (DriverOptions.proposal), host buffers --------------
    cfg = D.DriverConfig(n, m, H, K, w.lam,
                         D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, w.sigma, w.sigma_inv, m),
                         D.ControlBounds(w.u_min, w.u_max, m))
    drv = D.MPPIDriver(cfg, D.DriverOptions(proposal=net, proposal_samples=KS))
    err = D.ErrorRef()
    dspec = D.ModelPluginSpec(plugin_path(w.plugin),
                              D.CallableNames("mppi_dynamics", "mppi_stage_cost",
                                              "mppi_terminal_cost"),
                              D.ParamLayout(len(w.model_params), 4, w.cost_stride, 4),
                              D.RngConfig(w.seed))
    assert drv.initialize(dspec, err), err.value
    assert drv.set_problem_params(D.ProblemParams(D.ByteView.of(w.model_params),
                                                  D.ByteView.of(w.cost_params[0])), err), err.value
    ap = D.BatchAgentParams(cost_params=w.cost_params_packed, cost_params_stride=w.cost_stride,
                            sigma=w.agent_sigma)
    outs = D.BatchSimulationResults(np.zeros((T, N, n), np.float32),
                                    np.zeros((T, N, m), np.float32), np.zeros((T, N), np.float32),
                                    np.zeros((N, n), np.float32), N, T)
    for _ in range(args.warmup):
        assert drv.reset(None, err)
        assert drv.simulate_batch(N, T, w.x0, outs, ap, err), err.value
    e2e_times = []
    barrier()
    for _ in range(args.steps):
        assert drv.reset(None, err)
        t0 = time.perf_counter()
        assert drv.simulate_batch(N, T, w.x0, outs, ap, err), err.value
        e2e_times.append(time.perf_counter() - t0)
    barrier()
    e2e_total = max_over_ranks(sum(e2e_times))
    e2e_cost = models.executed_cost(w, outs.states_out, outs.controls_out,
                                    outs.terminal_states_out)
    sig_len = m if w.agent_sigma is not None else 0
    h2d = (N * n + N * H * m + 4) * 4 + N * ((w.cost_stride + 15) // 16 * 16) + N * sig_len * 4
    d2h = (T * N * (n + m + 1) + N * n) * 4

    if rank != 0:
        dist.finish(R)
        return 0
    # network forward: 2 * rows * (32*256 + 2*256*256 + 256*P) FLOPs
    out_pad = (spec["net_H"] * m + m + 15) // 16 * 16
    mlp_flops = 2 * N * (32 * 256 + 2 * 256 * 256 + 256 * out_pad)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    bf16_peak = peaks.get("bf16_tflops") or 1590.0
    line = {
        "metric": METRIC, "value": value, "unit": "control-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": prop_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 rollout, bf16 network (fp32 accumulate)",
        "data": "synthetic (seeded PCG64 workload generator, mppi_metal_b200/models.py)",
        "config": {
            "workload": (f"{args.workload}: {spec['desc']}, H={H}, {T} closed-loop steps; "
                         f"proposal-MPPI K={K} ({KS} samples around the network's prediction) "
                         f"against plain MPPI K={spec['plain_K']}"),
            "agents_per_gpu": N, "samples": K, "proposal_samples": KS,
            "plain_samples": spec["plain_K"], "horizon": H, "closed_loop_steps": T,
            "network": (f"MLP {spec['features']}->256->256->256->{spec['net_H'] * m + m}, GELU, "
                        f"bf16 weights, fp32 accumulate; predicts {spec['net_H']} steps"),
            "step": f"one simulate_batch closed loop ({T} control steps for every agent)",
            "l2": "flushed between timed iterations (256 MiB device write)",
            "parallelism": "agent-sharded replicas, no data-path collective",
        },
        "rollout_steps_per_s": value * K * H,
        "plain": {"control_steps_per_s": plain_value, "samples": spec["plain_K"],
                  "ms_per_step": plain_ms / args.steps,
                  "closed_loop_cost_mean": float(plain_cost.mean())},
        "closed_loop_cost": {"mean": float(prop_cost.mean()), "agents": N,
                             "vs_plain": float(prop_cost.mean() / plain_cost.mean())},
        "speedup_vs_plain": value / plain_value,
        "training": training,
        "e2e": {"value": world * N * T * args.steps / e2e_total, "unit": "control-steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": 1e3 * e2e_total / args.steps,
                "closed_loop_cost_mean": float(e2e_cost.mean())},
        "gpu_launches": (kernels_per_step * T + 1) * args.steps,
        "kernel_ms_per_pass": {"rollout": rollout_ms, "combine": combine_ms,
                               "features_kernel": feat_ms, "network": net_ms},
        "roofline": {"kernel": "mlp_forward_cluster_kernel (proposal network forward)",
                     "bound": "tensor",
                     "achieved": mlp_flops / (net_ms / 1e3) / 1e12, "peak": bf16_peak,
                     "unit": "TFLOP/s", "frac": mlp_flops / (net_ms / 1e3) / 1e12 / bf16_peak,
                     "traffic": None,
                     "note": f"M = {N} rows: one 8-CTA cluster, latency-bound; the dominant "
                             "kernel of the step is the rollout (issue-bound, see the batch "
                             "workload); peak = measured bf16 burst"
                             + ("" if peaks.get("bf16_tflops") else " (fallback)")},
        "clocks": clk,
    }
    print(json.dumps(line))
    dist.finish(R)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "kernels":
        return run_kernels_only(args)
    if args.workload in ("proposal", "quadrotor_proposal"):
        return run_proposal(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
