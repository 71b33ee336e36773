"""The multi-rank path on CPU (gloo, world size 2).  Two splits: whole windows sharded by
pair count (a batch of windows), and contiguous anchor ranges with a read-only right halo
(one long window: configurations 1 and 5).  Each rank parses only its own slab, one
all-reduce sums the per-bin / per-block outputs.  The per-rank compute here is the CPU
oracle standing in for the GPU parse (its ``anchor_end`` has the library's meaning); the
partition, the halo and the exchange are the code the GPU ranks run."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import ld_oracle as O
from pg_gpu_b200 import shard, synth


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_parse(w, rank, world, mode):
    """This rank's oracle bin sums over its own slab only, and its slab size."""
    wo = [0, w.n_var] if w.window_offsets is None else list(w.window_offsets)
    blk = w.snp_block
    if mode == "windows":
        counts = shard.window_pair_counts(w.positions, wo, w.max_dist)
        owner = shard.shard_windows(counts, world)
        snps, offs = shard.rank_slice(wo, owner, rank)
        ends = None
    else:
        snps, offs, ends = shard.slab_of(shard.split_anchors(w.positions, wo, w.max_dist, world)[rank])
    local = O.bin_sums(w.data[:, snps], w.positions[snps], w.pop_rows, w.edges, max_dist=w.max_dist,
                       window_offsets=offs, snp_block=None if blk is None else blk[snps],
                       n_blocks=w.n_blocks, anchor_end=ends)
    return local, len(snps)


def _worker(rank, world, port, cases, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        for cfg, scale, mode in cases:
            w = synth.make_config(cfg, scale=scale)
            local, slab = _rank_parse(w, rank, world, mode)
            sums = torch.from_numpy(local["sums"].copy())
            pairs = torch.from_numpy(local["pairs"].copy())
            shard.combine_bins(sums)
            shard.combine_bins(pairs)
            t = torch.tensor([float(rank + 1)], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            result_q.put(((cfg, mode), rank, sums.numpy(), pairs.numpy(), int(local["n_pairs"]), slab,
                          float(t.item())))
    finally:
        dist.destroy_process_group()


CASES = [(4, 0.002, "windows"), (4, 0.002, "anchors"), (1, 0.1, "anchors"), (5, 0.003, "anchors")]


def test_two_rank_splits_match_single_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, CASES, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world * len(CASES))]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for cfg, scale, mode in CASES:
        res = sorted((o for o in out if o[0] == (cfg, mode)), key=lambda o: o[1])
        w = synth.make_config(cfg, scale=scale)
        full = O.bin_sums(w.data, w.positions, w.pop_rows, w.edges, max_dist=w.max_dist,
                          window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks)
        for _, rank, sums, pairs, _, slab, tmax in res:
            np.testing.assert_array_equal(pairs, full["pairs"])
            np.testing.assert_allclose(sums, full["sums"], rtol=1e-12, atol=1e-15)
            assert tmax == float(world)  # max over ranks
        loads = [o[4] for o in res]
        assert sum(loads) == full["n_pairs"], (cfg, mode)  # every pair is owned by exactly one rank
        assert max(loads) <= 0.75 * sum(loads), (cfg, mode, loads)  # balanced enough to matter


def test_shard_windows_covers_each_window_once():
    rng = np.random.default_rng(0)
    counts = rng.integers(1, 10_000, size=57)
    for world in (1, 2, 3, 8):
        owner = shard.shard_windows(counts, world)
        assert owner.shape == counts.shape and owner.min() >= 0 and owner.max() < world
        loads = np.bincount(owner, weights=counts, minlength=world)
        assert loads.sum() == counts.sum()
        assert loads.max() - loads.min() <= counts.max()


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_anchors_partitions_pairs_with_halo(world):
    """Anchor ranges cover every SNP once, in order, cut at row-block multiples from a
    window start; each slab reaches every partner of its anchors and stays inside the
    window; the ranks' pair counts add up to the whole and are balanced to within the
    rounding of the cuts."""
    w = synth.make_config(5, scale=0.02)
    wo = [0, w.n_var]
    plans = shard.split_anchors(w.positions, wo, w.max_dist, world)
    jmax = shard.partner_ends(w.positions, wo, w.max_dist)
    covered = np.concatenate([np.arange(a, e) for p in plans for _, a, e, _ in p])
    np.testing.assert_array_equal(covered, np.arange(w.n_var))
    loads = []
    for p in plans:
        snps, offs, ends = shard.slab_of(p)
        for (_, a, e, h) in p:
            assert (a - wo[0]) % 64 == 0 or a == wo[0]
            assert h >= jmax[a:e].max() and h <= wo[-1]
        assert len(snps) == offs[-1] and np.all(ends <= offs[1:]) and np.all(ends >= offs[:-1])
        loads.append(sum(int(np.maximum(0, jmax[a:e] - np.arange(a, e) - 1).sum()) for _, a, e, _ in p))
    per_snp = np.maximum(0, jmax - np.arange(w.n_var) - 1)
    total = int(per_snp.sum())
    assert sum(loads) == total
    # each cut moves by at most half a row block (32 SNPs) from the balanced point
    assert max(loads) <= total / world + 2 * 33 * int(per_snp.max())
