"""Multi-GPU scoring by replicas: one process per GPU, frame pairs sharded round-robin.

Frame pairs are independent, so the only cross-rank traffic is host-side bookkeeping: the
per-pair scores are gathered once at the end and the timing is the maximum over ranks.  The
reference has no multi-GPU path at all (device selection only, src/VshipLib.cpp:201-218);
this mirrors how its users run one handler per GPU, without inventing a data-path collective.
"""
import numpy as np


def shard(n_items, rank, world):
    """Indices of the items rank `rank` of `world` scores (round-robin)."""
    return list(range(rank, n_items, world))


def gather_scores(local_scores, n_items, rank, world, group=None):
    """All ranks' scores in item order; local_scores are this rank's, in shard() order."""
    import torch.distributed as dist
    local = (rank, [float(s) for s in local_scores])
    if world == 1:
        parts = [local]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, local, group=group)
    out = np.full(n_items, np.nan)
    for r, vals in parts:
        idx = shard(n_items, r, world)
        out[idx] = vals
    return out


def max_over_ranks(seconds, world, device=None, group=None):
    """The slowest rank's time (the job's time)."""
    if world == 1:
        return float(seconds)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def score_pairs(pairs, score_fn, rank, world, group=None):
    """Scores pairs[i] with score_fn(pair) on the rank that owns i; returns every score on
    every rank."""
    mine = [score_fn(pairs[i]) for i in shard(len(pairs), rank, world)]
    return gather_scores(mine, len(pairs), rank, world, group)
