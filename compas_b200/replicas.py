"""Host logic of running the level advance on several GPUs of one node as independent replicas.

The path shards by independent cases: every rank advances its own case (weak scaling; no collective on
the data path). The only collectives are the barriers around the timed region and the maximum of the
ranks' times, so the whole-job rate is the cells all ranks updated divided by the slowest rank's time.
Independent requests of a serving run are dealt to ranks round-robin. These functions take the process
group (torch.distributed, NCCL on GPUs, gloo in the CPU tests) and the device its reductions run on.
"""
from __future__ import annotations


def barrier(dist, sync=None) -> None:
    """Barrier over the ranks (no-op without a process group), then `sync()` if given."""
    if dist is not None:
        dist.barrier()
    if sync is not None:
        sync()


def max_over_ranks(x: float, dist, device="cpu") -> float:
    """Maximum of x over the ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank: int, stages_per_step: int, steps: int, seconds_max: float, world: int) -> float:
    """Cell-updates per second per RK stage of the whole job: every rank updated cells_per_rank cells in
    each of steps x stages_per_step stages; the job took the slowest rank's time."""
    if not seconds_max > 0.0:
        raise ValueError("the timed region must have a positive duration")
    return world * cells_per_rank * stages_per_step * steps / seconds_max


def deal_requests(requests, rank: int, world: int) -> list:
    """The requests rank `rank` of `world` serves: round-robin by request id, so every request is served
    by exactly one rank and the ranks' shares differ by at most one."""
    return [r for r in requests if r.rid % world == rank]


def gather(obj, dist) -> list:
    """obj of every rank, in rank order ([obj] without a process group)."""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


__all__ = ["barrier", "max_over_ranks", "whole_job_rate", "deal_requests", "gather"]
