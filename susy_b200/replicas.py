"""Independent-lattice replicas over torch.distributed (one process per GPU).

The RHMC path of one lattice does not shard in this build: N GPUs run N
independent lattices (seeded per rank), with no collective in the data
path.  The process group only provides the barrier around the timed region
and the max-over-ranks time; any backend works (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank's replica: rank 0 keeps the base seed."""
    return base + 1000 * rank


def max_over_ranks(value: float, group=None) -> float:
    """Largest value across ranks (the job's wall time is the slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    dev = "cpu"
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def seconds_per_solve(max_ms: float, steps: int, world: int) -> float:
    """Whole-job seconds per solve: world replicas each did `steps` solves in
    the slowest rank's time max_ms."""
    return max_ms / 1e3 / (steps * world)
