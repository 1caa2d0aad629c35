"""Replica sharding of samples across GPUs (one process per GPU, no data-path collective).

The reference runs one independent worker per GPU and gives worker w the samples with
sample_id % workers == w (source/production/worker.py:51).  The same rule is kept here; the
only cross-rank operation is the max of the elapsed times for reporting.
"""
from __future__ import annotations


def shard(records, rank, world):
    """Records of this rank (reference rule: sample_id % world == rank)."""
    if not 0 <= rank < world:
        raise ValueError("Invalid worker ID")
    return [r for r in records if r["sample_id"] % world == rank]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks of the default process group (identity when not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_ids(ids, device=None):
    """All ranks' sample ids (for checking that the shards partition the protocol)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [list(ids)]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(ids))
    return out
