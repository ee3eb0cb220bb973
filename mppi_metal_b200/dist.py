"""Multi-GPU plumbing: one process per GPU, agents sharded across ranks.

MPPI agents are independent (the reference keys each agent's noise by its
index, shaders/mppi_rollout.metal:129-133), so ranks run disjoint agent sets
with no collective on the data path.  torch.distributed is used only for the
barrier around timed regions and the max-over-ranks of device times; the
backend is "nccl" on GPUs and "gloo" for CPU tests of this logic.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Rank:
    rank: int
    world: int
    local_rank: int

    @property
    def is_root(self) -> bool:
        return self.rank == 0


def env() -> Rank:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (defaults: 1 process)."""
    return Rank(int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
                int(os.environ.get("LOCAL_RANK", 0)))


def init(r: Rank, backend: str = "nccl", timeout_s: int = 300) -> None:
    """Joins the process group (no-op for one process).  A short timeout
    makes ranks that wait for a missing peer fail instead of hanging."""
    if r.world <= 1:
        return
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def finish(r: Rank) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def barrier(r: Rank, device=None) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()
    if device is not None and str(device).startswith("cuda"):
        import torch
        torch.cuda.synchronize()


def max_over_ranks(r: Rank, x: float, device="cpu") -> float:
    """The largest value of x over all ranks (every rank gets it)."""
    if r.world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agent_seed(base: int, r: Rank) -> int:
    """Weak scaling: every rank generates its own agents from its own seed,
    so agent sets are disjoint and per-rank work is fixed as world grows."""
    return base + r.rank


def shard(total: int, r: Rank) -> range:
    """Contiguous share of `total` agents for this rank (strong scaling):
    the first total % world ranks take one extra agent."""
    q, rem = divmod(total, r.world)
    start = r.rank * q + min(r.rank, rem)
    return range(start, start + q + (1 if r.rank < rem else 0))


def aggregate_rate(r: Rank, units_per_rank: float, seconds_this_rank: float,
                   device="cpu") -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time (every rank processes `units_per_rank`)."""
    return r.world * units_per_rank / max_over_ranks(r, seconds_this_rank, device)
