"""Splitting a parse across ranks (one process per GPU).

Two units, both with no exchange during the parse:

* whole windows (many windows, e.g. a batch of genome windows): ``shard_windows``
  assigns them to ranks by greedy pair-count balance (largest first);
* anchor ranges (one long window, e.g. a chromosome): ``split_anchors`` cuts the
  sequence of left SNPs into contiguous ranges of about equal pair count; a rank holds its
  anchors plus a read-only right halo -- the SNPs up to ``max_dist`` after its last anchor,
  which its pairs reach -- and parses that slab with ``anchor_end`` marking where its
  anchors stop (``ldk_parse_t.anchor_end``).  This is the unit of pg_gpu's own pair chunks
  (anchor blocks, ``ld_pipeline.py:57-122``), made contiguous so each rank reads one slab.

``combine_bins`` sums the ranks' per-bin (or per-block) float64 outputs with one
all-reduce -- the only exchange the path has, a few KB to MB.  Bootstrap blocks keep their
global ids, so per-block sums from different ranks land in the right rows.
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


def partner_ends(positions, window_offsets, max_dist):
    """jmax[i]: one past the last partner of SNP i (pos[j] - pos[i] <= max_dist, same window),
    the pair generator's range (ld_pipeline.py:57-122)."""
    pos = np.asarray(positions, dtype=np.float64)
    jmax = np.empty(len(pos), dtype=np.int64)
    for a, b in zip(window_offsets[:-1], window_offsets[1:]):
        jmax[a:b] = a + np.searchsorted(pos[a:b], pos[a:b] + max_dist, side="right")
    return jmax


def split_anchors(positions, window_offsets, max_dist, world_size, align=64):
    """Per rank, its segments ``(window, anchor_start, anchor_end, halo_end)`` in global SNP
    indices: contiguous anchor ranges of about equal pair count over the windows in order,
    cut at multiples of ``align`` SNPs from a window's start (the tensor-core kernel's row
    block, so a split does not change which SNPs share a row block).  A rank's pairs are
    those with their left SNP in ``[anchor_start, anchor_end)``; its partners end before
    ``halo_end``."""
    window_offsets = [int(x) for x in window_offsets]
    n = window_offsets[-1]
    jmax = partner_ends(positions, window_offsets, max_dist)
    per_snp = np.maximum(0, jmax - np.arange(n) - 1)
    cum = np.concatenate([[0], np.cumsum(per_snp)])
    total = int(cum[-1])
    starts = np.asarray(window_offsets[:-1], dtype=np.int64)
    cuts = [0]
    for r in range(1, world_size):
        c = int(np.searchsorted(cum, total * r / world_size, side="left"))
        w = max(0, int(np.searchsorted(starts, c, side="right")) - 1)  # window holding SNP c
        w0, w1 = window_offsets[w], window_offsets[w + 1]
        c = min(w1, w0 + int(round((c - w0) / align)) * align)
        cuts.append(max(cuts[-1], c))
    cuts.append(n)
    plans = []
    for r in range(world_size):
        lo, hi = cuts[r], cuts[r + 1]
        seg = []
        for w, (w0, w1) in enumerate(zip(window_offsets[:-1], window_offsets[1:])):
            a, e = max(lo, w0), min(hi, w1)
            if a < e:
                seg.append((w, a, e, max(e, int(jmax[e - 1]))))
        plans.append(seg)
    return plans


def slab_of(segments):
    """A rank's input slab: global SNP indices, local window offsets and local anchor ends
    (the ``window_offsets`` / ``anchor_end`` of its parse)."""
    idx, offs, ends = [], [0], []
    for _, a, e, h in segments:
        idx.append(np.arange(a, h))
        ends.append(offs[-1] + (e - a))
        offs.append(offs[-1] + (h - a))
    snps = np.concatenate(idx) if idx else np.zeros(0, np.int64)
    return snps, np.asarray(offs, dtype=np.int64), np.asarray(ends, dtype=np.int64)


def slab_workload(w, segments):
    """The workload one rank of an anchor split parses: its slab of ``w`` (a
    ``synth.Workload``) with local window offsets and ``anchor_end``; bootstrap blocks keep
    their global ids."""
    import dataclasses
    snps, offs, ends = slab_of(segments)
    return dataclasses.replace(
        w, data=np.ascontiguousarray(w.data[:, snps]), positions=w.positions[snps].copy(),
        window_offsets=offs, anchor_end=ends,
        snp_block=None if w.snp_block is None else w.snp_block[snps].copy())
