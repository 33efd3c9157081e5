"""Multi-GPU runs of the step: independent replicas, one per rank.

The time step does not shard across GPUs here (one mesh per GPU), so N GPUs
run N independent replicas with no data-path collective.  The only
cross-rank operations are the barrier around the timed region and the
max-over-ranks of the measured times, which work on any torch.distributed
backend (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def barrier() -> None:
    d = _dist()
    if d is not None:
        d.barrier()


def max_over_ranks(x: float) -> float:
    d = _dist()
    if d is None:
        return float(x)
    import torch
    dev = "cuda" if d.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(work_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job throughput: every rank did work_per_rank units; the job took
    the slowest rank's time."""
    return world * work_per_rank / seconds_max
