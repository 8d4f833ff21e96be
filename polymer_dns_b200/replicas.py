"""Replica bookkeeping for multi-GPU runs: one independent channel per rank, no data exchange.

The reference has no domain decomposition; its ensemble is a farm of independent processes
(LO_multi_run/setup.py:93-101).  Across ranks the only collectives are a barrier around the
timed region and the reduction of the timings: the whole-job time is the slowest rank's, and
the throughput counts every rank's steps.
"""
import torch


def reduce_max(dist, value, device):
    """Maximum of a per-rank float over the process group (every rank gets it)."""
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(dist, local_ms, steps_per_rank, world, device):
    """(max_ms over ranks, whole-job steps per second = world * steps / max time)."""
    ms = reduce_max(dist, local_ms, device)
    return ms, world * steps_per_rank / (ms / 1e3)


def checksum_all(dist, value, world, device):
    """Every rank's float (e.g. a field checksum), gathered on every rank."""
    if dist is None:
        return [float(value)]
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t)
    return [float(x.item()) for x in out]
