"""Splitting a batched parse across ranks (one process per GPU).

Pairs never cross windows, so whole windows are the unit: ``shard_windows`` assigns
them to ranks by greedy pair-count balance (largest first), and ``combine_bins`` sums
the ranks' per-bin (or per-block) float64 outputs with one all-reduce -- the only
exchange the path has, a few KB to MB.  Bootstrap blocks keep their global ids, so
per-block sums from different ranks land in disjoint rows and the all-reduce
concatenates them.
"""
from __future__ import annotations

import numpy as np


def window_pair_counts(positions, window_offsets, max_dist):
    """Pairs i < j with pos[j] - pos[i] <= max_dist inside each window."""
    pos = np.asarray(positions, dtype=np.float64)
    out = []
    for a, b in zip(window_offsets[:-1], window_offsets[1:]):
        p = pos[a:b]
        jm = np.searchsorted(p, p + max_dist, side="right")
        out.append(int(np.sum(np.maximum(0, jm - np.arange(len(p)) - 1))))
    return np.asarray(out, dtype=np.int64)


def shard_windows(pair_counts, world_size):
    """Rank of every window: longest-processing-time-first greedy balance."""
    counts = np.asarray(pair_counts, dtype=np.int64)
    load = np.zeros(world_size, dtype=np.int64)
    owner = np.empty(len(counts), dtype=np.int64)
    for w in np.argsort(-counts, kind="stable"):
        r = int(np.argmin(load))
        owner[w] = r
        load[r] += counts[w]
    return owner


def rank_slice(window_offsets, owner, rank):
    """SNP index array and local window offsets of the windows owned by ``rank``."""
    idx, offs = [], [0]
    for w, (a, b) in enumerate(zip(window_offsets[:-1], window_offsets[1:])):
        if owner[w] == rank:
            idx.append(np.arange(a, b))
            offs.append(offs[-1] + (b - a))
    snps = np.concatenate(idx) if idx else np.zeros(0, np.int64)
    return snps, np.asarray(offs, dtype=np.int64)


def combine_bins(local, group=None):
    """Sum a rank's float64 (or int64) output tensor over all ranks, in place."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(local, op=dist.ReduceOp.SUM, group=group)
    return local
