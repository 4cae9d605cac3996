"""Replicas over several processes (one per GPU): the multi-GPU form of this engine.

The explicit-dynamics path of one body is not split across GPUs here; independent bodies are
(ensemble specimens, benchmark replicas), so the ranks exchange nothing on the data path.
What the ranks share is bookkeeping: which specimens each rank owns, a barrier around timed
regions, and the maximum of the per-rank device times (whole-job throughput = the units of
all ranks / the slowest rank's time). The functions take a ``torch.distributed`` process
group of any backend (NCCL on GPUs, gloo on CPUs) or run single-process when it is None.
"""
from __future__ import annotations


def partition_specimens(sizes, world):
    """Specimen indices per rank, balancing the point (or bond) counts `sizes`: largest first
    onto the least loaded rank (longest-processing-time rule). Deterministic."""
    order = sorted(range(len(sizes)), key=lambda k: (-sizes[k], k))
    load = [0] * world
    owned = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owned[r].append(k)
        load[r] += sizes[k]
    return [sorted(o) for o in owned]


def _tensor(x, device):
    import torch
    return torch.tensor([float(x)], dtype=torch.float64, device=device)


def reduce_max(x, dist=None, device="cpu"):
    """Maximum of a per-rank scalar over the ranks (the timing rule of the benchmark)."""
    if dist is None:
        return float(x)
    t = _tensor(x, device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, dist=None, device="cpu"):
    if dist is None:
        return float(x)
    t = _tensor(x, device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def throughput(units, seconds, dist=None, device="cpu"):
    """Whole-job rate: the units processed by all ranks over the slowest rank's time."""
    return reduce_sum(units, dist, device) / reduce_max(seconds, dist, device)
