"""Host-side logic of multi-GPU runs (one process per GPU, torch.distributed).

Field points, probes and tracks are independent, so a run with N ranks gives every rank its
own seeded block of points against the same replicated geometry and needs no data-path
collective; the only collectives are a barrier around the timed region and the max over
ranks of each rank's device time (the job is as slow as its slowest rank). The same code runs
over NCCL on GPUs and over gloo on CPU (tests/test_cpu_ranks.py).
"""

from __future__ import annotations

from . import geometry as G

POINT_SEED = 2024


def rank_points(n_per_rank: int, rank: int):
    """This rank's block of gap points: seeded per rank, so blocks differ and are reproducible."""
    return G.gap_points(n_per_rank, seed=POINT_SEED + rank)


def barrier(dist=None, device=None):
    """Synchronise the device (if any) and all ranks (if distributed)."""
    if device is not None:
        import torch

        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank scalar over all ranks (the job's time)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
