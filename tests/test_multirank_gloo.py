"""The multi-rank path on CPU (gloo, world size 2): whole windows are sharded by pair
count, each rank parses its windows, one all-reduce sums the per-bin / per-block
outputs.  The per-rank compute here is the CPU oracle standing in for the GPU parse;
the sharding and the exchange are the code the GPU ranks run."""
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


def _worker(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        w = synth.make_config(4, scale=0.002)
        counts = shard.window_pair_counts(w.positions, w.window_offsets, w.max_dist)
        owner = shard.shard_windows(counts, world)
        snps, offs = shard.rank_slice(w.window_offsets, owner, rank)
        local = O.bin_sums(w.data[:, snps], w.positions[snps], w.pop_rows, w.edges, max_dist=w.max_dist,
                           window_offsets=offs, snp_block=w.snp_block[snps], n_blocks=w.n_blocks)
        sums = torch.from_numpy(local["sums"].copy())
        pairs = torch.from_numpy(local["pairs"].copy())
        shard.combine_bins(sums)
        shard.combine_bins(pairs)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        result_q.put((rank, sums.numpy(), pairs.numpy(), int(counts[owner == rank].sum()), float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_rank_window_sharding_matches_single_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    w = synth.make_config(4, scale=0.002)
    full = O.bin_sums(w.data, w.positions, w.pop_rows, w.edges, max_dist=w.max_dist,
                      window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks)
    for rank, sums, pairs, _, tmax in out:
        np.testing.assert_array_equal(pairs, full["pairs"])
        np.testing.assert_allclose(sums, full["sums"], rtol=1e-12, atol=1e-15)
        assert tmax == float(world)  # max over ranks
    loads = [o[3] for o in out]
    assert sum(loads) == full["n_pairs"]  # every generated pair is owned by exactly one rank
    assert max(loads) <= 0.75 * sum(loads)  # balanced enough to matter


def test_shard_windows_covers_each_window_once():
    rng = np.random.default_rng(0)
    counts = rng.integers(1, 10_000, size=57)
    for world in (1, 2, 3, 8):
        owner = shard.shard_windows(counts, world)
        assert owner.shape == counts.shape and owner.min() >= 0 and owner.max() < world
        loads = np.bincount(owner, weights=counts, minlength=world)
        assert loads.sum() == counts.sum()
        assert loads.max() - loads.min() <= counts.max()
