#!/usr/bin/env python
"""Throughput of the B200 two-locus LD parse: SNP pairs per second.

Workload (default): configuration 4, the batched windowed parse -- 200 windows of lognormal
SNP counts (median 2,000, 200..20,000), 3 populations of 50/120/300 haplotypes, 3%
missing, 16 log-spaced distance bins (10 bp .. 1 Mb), per-window per-bin FP64
DD/Dz/pi2 (45 statistics), 50-kb bootstrap blocks and 100 block-bootstrap replicates.
Seeded synthetic data (founder mosaics, see pg_gpu_b200/synth.py).

One step = the whole batched parse of that workload: pair ranges, indicator planes,
the fused INT8 tcgen05 count + estimator + bin kernel, per-window totals and bootstrap
replicates.  ``value`` has inputs resident in HBM; ``e2e`` copies the inputs from
pinned host memory and the results back every step.  ``--impl reference`` times pg_gpu's
path on the host cores instead: its own estimator kernels compiled for the host
(``oracle/_ref``, haplotype path with one, three or four populations) or the oracle's
restatement of it.

Multi-GPU (torchrun): weak scaling by default, each rank parses its own independently
seeded workload of the same shape; no data-path collective.  ``--split``: strong scaling of
one workload, cut into contiguous anchor ranges of equal pair count (``shard.split_anchors``);
each rank parses its slab (anchors plus the read-only right halo) and one NCCL all-reduce
per step sums the per-block bin outputs before the bootstrap replicates.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

METRIC = "LD SNP-pairs/s: INT8-TC+FP32 vs plain FP64 on same B200, rel err ≤1e-6"
UNIT = "SNP-pairs/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return dict(FALLBACK_PEAKS), "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, phys_index):
        self.phys = str(phys_index)
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != self.phys:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU side: the oracle (pg_gpu's algorithm restated in NumPy) on a bounded sample
# ---------------------------------------------------------------------------

CPU_WHAT = {
    "reference": "pg_gpu's own estimator kernels, compiled for the host from its source (oracle/_ref) and "
                 "driven by the oracle's restatement of its dispatch; counts and binning as its NumPy code",
    "port": "the oracle, a NumPy restatement of pg_gpu's path",
}


def cpu_kind(w):
    """"reference" where pg_gpu's own estimator kernels run on the host (oracle/_ref, built
    from its source; its kernel path: haplotypes with one, three or four populations),
    else "port" (the oracle's NumPy restatement)."""
    from oracle import ref_kernels
    return "reference" if (not w.genotypes and len(w.pop_rows) != 2 and ref_kernels.available()) else "port"


def _cpu_task(args):
    data, pos, pop_rows, edges, max_dist, n_anchor, genotypes, kind = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import ld_oracle as O
    stat_fn = None
    if kind == "reference":
        from oracle import ref_kernels
        stat_fn = ref_kernels.hap_stats
    t0 = time.perf_counter()
    r = O.bin_sums(data, pos, pop_rows, edges, genotypes=genotypes, max_dist=max_dist, anchor_end=[n_anchor],
                   stat_fn=stat_fn)
    return r["n_pairs"], time.perf_counter() - t0


def cpu_sample_tasks(w, workers, pairs_per_worker, seed=0):
    """One task per worker: all pairs of a run of consecutive anchor SNPs (every partner,
    so the whole distance range) starting at a SNP drawn in proportion to its pair count,
    i.e. pairs are sampled where the workload has them, over full-size windows.  A task is
    the anchors' slab: the anchors plus the partners after them."""
    from pg_gpu_b200 import shard
    offs = [0, w.n_var] if w.window_offsets is None else [int(x) for x in w.window_offsets]
    jmax = shard.partner_ends(w.positions, offs, w.max_dist)
    per = np.maximum(0, jmax - np.arange(w.n_var) - 1).astype(np.float64)
    win = np.zeros(w.n_var, np.int64)
    for k, (a, b) in enumerate(zip(offs[:-1], offs[1:])):
        win[a:b] = k
    rng = np.random.default_rng(seed)
    kind = cpu_kind(w)
    tasks = []
    for _ in range(workers):
        a = int(rng.choice(w.n_var, p=per / per.sum()))
        end = offs[win[a] + 1]
        e, got = a, 0
        while e < end and got < pairs_per_worker:
            got += int(per[e])
            e += 1
        h = max(e, int(jmax[e - 1]))
        tasks.append((np.ascontiguousarray(w.data[:, a:h]), w.positions[a:h].copy(), w.pop_rows, w.edges,
                      w.max_dist, e - a, bool(w.genotypes), kind))
    return tasks


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_pool(workers):
    import multiprocessing as mp
    pool = mp.get_context("spawn").Pool(workers)
    pool.map(_noop, range(workers))  # start every worker before timing
    return pool


def _noop(_):
    from oracle import ld_oracle  # noqa: F401
    return 0


def run_cpu_sample(w, seconds, workers=None, pool=None, seed=0):
    """Time the oracle on ~``seconds`` of CPU work per worker; pairs/s over all workers (a
    rate measured on a sample: the full workload's CPU time is extrapolated from it)."""
    workers = workers or cpu_cores()
    probe = cpu_sample_tasks(w, 1, 20_000, seed=10_000 + seed)[0]
    n, dt = _cpu_task(probe)
    rate = n / max(dt, 1e-9)
    per_worker = max(20_000, int(rate * seconds))
    tasks = cpu_sample_tasks(w, workers, per_worker, seed=seed)
    own = pool is None
    if own:
        pool = cpu_pool(workers)
    t0 = time.perf_counter()
    res = pool.map(_cpu_task, tasks)
    wall = time.perf_counter() - t0
    if own:
        pool.close()
        pool.join()
    pairs = sum(r[0] for r in res)
    return {"value": pairs / wall, "pairs": pairs, "wall_s": wall, "workers": workers,
            "per_worker_pairs": per_worker, "kind": tasks[0][-1]}


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------

def make_workload(cfg, scale, rank):
    from pg_gpu_b200 import synth
    seed = {1: 1, 2: 2, 3: 3, 4: 4, 5: 5}[cfg] + 1000 * rank
    return synth.make_config(cfg, scale=scale, seed=seed)


def bench_workload(args, rank):
    """The configuration's workload, its rows regrouped into ``--pops`` populations if asked."""
    w = make_workload(args.config, args.scale, rank)
    if args.pops:
        import dataclasses
        rows = np.concatenate([np.asarray(r) for r in w.pop_rows])
        w = dataclasses.replace(w, pop_rows=[np.asarray(x) for x in np.array_split(rows, args.pops)],
                                name=f"{w.name}, rows regrouped into {args.pops} populations")
    return w


def algorithmic_int_ops_per_pair(w):
    """Count-stage INT ops per pair (MAC = 2): haplotypes, four 0/1 dot products of
    length n per population (h.h, h.v, v.h, v.v), i.e. 8n; genotypes, the 3 x 3 Gram of
    {g = 1, g = 2, valid}, i.e. 18n per population."""
    return sum((18 if w.genotypes else 8) * len(r) for r in w.pop_rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=4)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--method", choices=["tc", "plain"], default="tc")
    ap.add_argument("--plain-steps", type=int, default=2, help="steps of the plain FP64 kernel for the ratio")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="call ldk_parse per step instead of a graph replay")
    ap.add_argument("--no-autotune", action="store_true", help="default tile width, no tuning")
    ap.add_argument("--packed", action="store_true",
                    help="inputs stored two bits per entry (parse.pack_codes): a quarter of the bytes to copy")
    ap.add_argument("--pops", type=int, default=0,
                    help="regroup the workload's sampled rows into this many populations of equal size")
    ap.add_argument("--split", action="store_true",
                    help="strong scaling: one workload split into anchor ranges over the ranks")
    ap.add_argument("--all-pairs", action="store_true",
                    help="time the all-pairs LD kernel (ldk_ld_matrix) instead of the binned parse")
    ap.add_argument("--snps", type=int, default=24576, help="--all-pairs: SNPs in the set")
    ap.add_argument("--haplotypes", type=int, default=200, help="--all-pairs: haplotypes")
    ap.add_argument("--estimator", choices=["r2", "sigma_d2", "r2_counts", "diploid_r2", "rogers_huff_r",
                                            "sigma_d2_geno"], default="r2")
    ap.add_argument("--reduce-only", action="store_true", help="--all-pairs: ZnS sums only, no matrix")
    args = ap.parse_args()

    ws, rank, local = dist_env()
    if args.all_pairs:
        return run_all_pairs(args)
    if args.impl == "reference":
        return run_reference(args, ws, rank)

    import torch
    import torch.distributed as dist

    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    from pg_gpu_b200 import _lib, parse, synth

    lib = _lib.load()
    w = bench_workload(args, 0 if args.split else rank)
    n_pairs = synth.count_pairs(w)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = run_cpu_sample(w, args.cpu_seconds)
    whole_pairs = n_pairs
    if args.split:  # this rank's slab: anchors plus the right halo
        from pg_gpu_b200 import shard
        wo = [0, w.n_var] if w.window_offsets is None else list(w.window_offsets)
        seg = shard.split_anchors(w.positions, wo, w.max_dist, ws, align=_lib.tc_row_blocks(w.genotypes)[0])[rank]
        w = shard.slab_workload(w, seg)
        n_pairs = synth.count_pairs(w)
    split_comm = args.split and ws > 1

    def combine(out):
        """Sum the ranks' per-block outputs (the split's one collective)."""
        if split_comm:
            for t in (out.sums, out.r2_sums, out.pairs, out.r2_counts):
                dist.all_reduce(t, op=dist.ReduceOp.SUM)

    if not args.no_autotune:
        _lib.autotune(True)
    x_in = parse.pack_codes(w.data) if args.packed else w.data  # the input as the host stores it
    parser = parse.Parser(x_in, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes, method=args.method,
                          packed=args.packed,
                          max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                          n_blocks=w.n_blocks, anchor_end=w.anchor_end, device=dev)
    reps_w = torch.as_tensor(w.replicate_weights if w.replicate_weights is not None
                             else np.ones((1, w.n_blocks), np.int32), dtype=torch.int32, device=dev)
    if w.window_of_block is not None:
        win_ind = np.zeros((len(w.window_offsets) - 1, w.n_blocks), np.int32)
        win_ind[w.window_of_block, np.arange(w.n_blocks)] = 1
    else:
        win_ind = np.ones((1, w.n_blocks), np.int32)
    win_w = torch.as_tensor(win_ind, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    # kernel time of the dominant kernel (CUDA events around it inside ldk_parse), outside
    # the timed steps; the first call also tunes the tile width (recorded below)
    lib.ldk_profile(1)
    prof_ms = []
    for _ in range(3):
        parser.run()
        prof_ms.append(lib.ldk_profile_last_kernel_ms())
    prof_ms = prof_ms[1:]

    # One step = parse + bootstrap replicates + per-window totals.  Default: the whole step
    # captured once as a CUDA graph and replayed (the inputs are re-read in place).
    if args.no_graph:
        def step():
            r = parser.run()
            combine(r)
            reps = parse.block_combine(r.sums, reps_w)
            wins = parse.block_combine(r.sums, win_w)
            return r, reps, wins
    elif split_comm:  # the parse replayed as a graph; the all-reduce and replicates after it
        graph, _ = parser.graph()

        def step():
            graph.replay()
            combine(parser.out)
            return parser.out, parse.block_combine(parser.out.sums, reps_w), parse.block_combine(parser.out.sums, win_w)
    else:
        graph, (g_reps, g_wins) = parser.graph(
            after=lambda out: (parse.block_combine(out.sums, reps_w), parse.block_combine(out.sums, win_w)))

        def step():
            graph.replay()
            return parser.out, g_reps, g_wins

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    phys = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    phys_index = phys[dev.index] if phys and phys[0] not in ("",) and dev.index < len(phys) else dev.index
    kernel_ms = []
    with ClockSampler(phys_index) as clk:
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            r, reps, wins = step()
        e1.record(stream)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
    elapsed_ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    t_max = elapsed_ms
    if ws > 1:
        t = torch.tensor([elapsed_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    total_pairs = (whole_pairs if args.split else n_pairs * ws) * args.steps
    value = total_pairs / (t_max / 1e3)
    ms_per_step = t_max / args.steps
    if not args.no_graph:
        parser.status()  # device status word of the last replay (raises on a device error)
    k_ms = statistics.mean(prof_ms) if prof_ms else None

    # ---- end to end through the public API: pinned host inputs in, results out.  With
    # graphs, parse.Pipeline double-buffers the steps: each step's inputs are copied in
    # (pinned host -> device) while the previous step parses, and its results copied out
    # while the next one parses; the timed region spans the first copy in to the last copy
    # out.  Without graphs the steps run in series on one stream.
    X_h = torch.from_numpy(np.ascontiguousarray(x_in).view(np.int8)).pin_memory()
    pos_h = torch.from_numpy(np.ascontiguousarray(w.positions)).pin_memory()
    blk_h = torch.from_numpy(np.ascontiguousarray(w.snp_block if w.snp_block is not None
                                                  else np.zeros(w.n_var, np.int32))).pin_memory()
    rw_h = reps_w.cpu().pin_memory()

    def host_outputs():
        return [torch.empty(parser.out.sums.shape, dtype=torch.float64).pin_memory(),
                torch.empty(parser.out.pairs.shape, dtype=torch.int64).pin_memory(),
                torch.empty((reps_w.shape[0],) + tuple(parser.out.sums.shape[1:]), dtype=torch.float64).pin_memory(),
                torch.empty((win_w.shape[0],) + tuple(parser.out.sums.shape[1:]), dtype=torch.float64).pin_memory()]

    h_in = {"X": X_h, "pos": pos_h, "reps_w": rw_h}
    if parser.block is not None:
        h_in["block"] = blk_h
    h2d = sum(t.numel() * t.element_size() for t in h_in.values())
    if args.no_graph or split_comm:  # steps in series on one stream
        outs_h = [host_outputs()]

        def e2e_step(k):
            parser.X.copy_(X_h, non_blocking=True)
            parser.pos.copy_(pos_h, non_blocking=True)
            if parser.block is not None:
                parser.block.copy_(blk_h, non_blocking=True)
            reps_w.copy_(rw_h, non_blocking=True)
            r, reps, wins = step()
            for h, d in zip(outs_h[0], (r.sums, r.pairs, reps, wins)):
                h.copy_(d, non_blocking=True)

        def e2e_done():
            pass
    else:
        def make_slot():
            p = parse.Parser(x_in, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes, method=args.method,
                             packed=args.packed,
                             max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                             n_blocks=w.n_blocks, anchor_end=w.anchor_end, device=dev)
            rw = torch.empty_like(reps_w)
            rw.copy_(reps_w)
            ins = {"X": p.X, "pos": p.pos, "block": p.block, "reps_w": rw}
            return p, ins, (lambda out: (parse.block_combine(out.sums, rw), parse.block_combine(out.sums, win_w)))

        pipe = parse.Pipeline(make_slot, slots=2)
        outs_h = [host_outputs() for _ in range(2)]

        def e2e_step(k):
            pipe.submit(h_in, outs_h[k % 2])

        def e2e_done():
            pipe.drain()
    d2h = sum(t.numel() * t.element_size() for t in outs_h[0])
    for k in range(2):  # warm-up: both slots once
        e2e_step(k)
    e2e_done()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for k in range(args.steps):
        e2e_step(k)
    e2e_done()
    f1.record(stream)
    torch.cuda.synchronize()
    if not (args.no_graph or split_comm):
        pipe.status()
        # the last step's results, copied out through the pipeline, match the resident run
        last = outs_h[(args.steps - 1) % 2]
        if not (np.array_equal(last[1].numpy(), parser.out.pairs.cpu().numpy())
                and np.allclose(last[0].numpy(), parser.out.sums.cpu().numpy(), rtol=1e-9, atol=0)):
            raise RuntimeError("end-to-end pipeline results differ from the resident parse")
    e2e_ms = f0.elapsed_time(f1)
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = total_pairs / (e2e_ms / 1e3)

    # ---- the plain FP64 kernel on the same workload, and parity of the fast path against it
    plain = None
    parity = None
    if args.method != "plain" and args.plain_steps > 0:
        fast = {k: v.copy() for k, v in parser.out.numpy().items()}
        pp = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes, method="plain",
                          max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                          n_blocks=w.n_blocks, anchor_end=w.anchor_end, device=dev)
        pp.run()
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        pk = []
        for _ in range(args.plain_steps):
            pp.run()
            pk.append(lib.ldk_profile_last_kernel_ms())
        g1.record(stream)
        torch.cuda.synchronize()
        pms = g0.elapsed_time(g1) / args.plain_steps
        if ws > 1:
            t = torch.tensor([pms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pms = float(t.item())
        combine(pp.out)  # a split compares the combined outputs
        ref = pp.out.numpy()
        tot_f, tot_p = fast["sums"].sum(axis=0), ref["sums"].sum(axis=0)
        parity = {
            "pairs_bit_exact": bool(np.array_equal(fast["pairs"], ref["pairs"])
                                    and np.array_equal(fast["r2_counts"], ref["r2_counts"])),
            "max_rel_err_per_bin": float(np.max(np.abs(tot_f - tot_p) / np.maximum(np.abs(tot_p), 1e-300))),
            "max_rel_err_per_block_bin": float(np.max(np.abs(fast["sums"] - ref["sums"])
                                                      / np.maximum(np.abs(ref["sums"]), 1e-300))),
            "reference": "plain FP64 kernel, same workload",
        }
        plain = {"value": (whole_pairs if args.split else n_pairs * ws) / (pms / 1e3), "ms_per_step": pms,
                 "kernel_ms": statistics.mean(pk) if pk else None}
        del pp

    # ---- the tuning table's choice for this shape (tile width, row-block order)
    tuned_entry = None
    if not args.no_autotune and args.method == "tc":
        with tempfile.TemporaryDirectory() as td:
            tp = os.path.join(td, "tune.json")
            if _lib.autotune_save(tp) > 0:
                ents = json.load(open(tp))["entries"]
                mine = [e for e in ents if e["pops"] == len(w.pop_rows) and e["genotypes"] == int(w.genotypes)
                        and e["bins"] == len(w.edges) - 1]
                tuned_entry = mine[0] if len(mine) == 1 else None

    # ---- roofline of the dominant kernel
    pk_d, pk_kind = peaks()
    probe_i8, probe_f64 = _lib.probe_peaks()
    int8_peak = probe_i8 / 1e12
    ops = algorithmic_int_ops_per_pair(w) * n_pairs
    achieved = ops / (k_ms / 1e3) / 1e12 if k_ms else None
    traffic = None
    tfile = os.path.join(REPO, "profiles", "k_parse_tc_c4_traffic.json")
    if os.path.exists(tfile) and args.config == 4 and args.method == "tc":
        with open(tfile) as f:
            tj = json.load(f)
        # captured on this full-size workload: bytes per launch as measured
        traffic = tj["dram_bytes_per_launch"] if tj.get("pairs") == n_pairs else None
    fp64 = None
    ifile = os.path.join(REPO, "profiles", "k_parse_tc_c4_fp64.json")
    if os.path.exists(ifile) and args.config == 4 and args.method == "tc" and k_ms:
        with open(ifile) as f:
            fj = json.load(f)
        per_pair = fj["fp64_thread_inst_per_pair"]
        rate = per_pair * n_pairs / (k_ms / 1e3)
        fp64 = {"inst_per_pair": per_pair, "inst_per_pair_source": "ncu, " + fj["workload"],
                "achieved_inst_per_s": rate, "peak_fma_per_s": probe_f64, "frac": rate / probe_f64,
                "peak_source": "ldk_probe_peaks in this run (8 FP64 FMA chains per thread, 16 warps per SM)"}
    roofline = {"bound": "tensor", "kernel": "k_parse_tc", "achieved": achieved, "peak": int8_peak,
                "unit": "TOP/s (INT8, MAC=2)", "frac": (achieved / int8_peak) if achieved else None,
                "peak_source": "measured in this run: ldk_probe_peaks, back-to-back tcgen05 kind::i8 "
                               "128x256x32 MMAs on every SM",
                "peak_bf16x2_derived": 2.0 * pk_d["bf16_tflops"],
                "traffic": traffic, "kernel_ms": k_ms, "fp64": fp64,
                "note": "count stage algorithmic ops = 8 (haplotypes) or 18 (genotypes) x sum(n_pop) per pair; the fused kernel is bound by "
                        "its FP64 estimator epilogue (see fp64), not by the tensor pipe"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if args.split else "weak", "vs_baseline": None,
            "dtype": {"tc": "u8 counts / s32 accumulate / f64 estimators",
                      "plain": "i8 byte counts / f64 estimators"}[args.method],
            "data": "synthetic (seeded founder mosaics; no public dataset offline)",
            "config": {"workload": w.name, "config_index": args.config, "scale": args.scale,
                       "snps": int(w.n_var), "pairs_per_step_per_gpu": int(n_pairs),
                       "populations": [len(r) for r in w.pop_rows], "bins": int(len(w.edges) - 1),
                       "statistics": int(parse.n_stats(len(w.pop_rows))), "windows":
                       int(len(w.window_offsets) - 1) if w.window_offsets is not None else 1,
                       "bootstrap_blocks": int(w.n_blocks),
                       "bootstrap_replicates": int(reps_w.shape[0]),
                       "method": args.method,
                       "input": "2-bit packed codes (LDK_X_PACKED2)" if args.packed else "int8 codes",
                       "parallelism": (f"strong x{ws}: anchor ranges with right halo, one all-reduce of the "
                                       f"per-block bin outputs per step") if args.split
                       else f"weak x{ws}, no data-path collective",
                       "whole_workload_pairs": int(whole_pairs),
                       "tile_partners": int(parser.tile_width()),
                       "tile_source": "autotuned (ldk_autotune)" if not args.no_autotune else "default",
                       "tuned": tuned_entry,
                       "l2": "inputs larger than L2 (haplotypes %d MB, indicator planes %d MB)" % (
                           w.data.nbytes >> 20, (w.n_var * 2 * parser_ktot(w)) >> 20)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "roofline": roofline,
            # per step: k_jmax, k_prep_planes, k_split_items, k_parse_tc, k_fx_finish,
            # 2 x k_block_combine, and on
            # the genotype path (1-3 populations) k_fill_gtab; plain: k_jmax, k_parse_plain,
            # k_fx_finish, 2 x combine (a workspace reciprocal table, k_fill_rtab, serves only
            # populations whose table does not fit in shared memory: none of configurations 1-5)
            "gpu_launches": int(args.steps * (5 if parser.method == "plain" else
                                              7 + int(bool(w.genotypes) and len(w.pop_rows) <= 3))),
            "launch": "CUDA graph replay (memsets, k_jmax, planes, work items + parse kernel, k_fx_finish, "
                      "2 x k_block_combine"
                      + (", genotype reciprocal table" if w.genotypes and parser.method != "plain" else "") + ")"
                      if not args.no_graph else "ldk_parse per step",
            "clocks": clocks,
        }
        if plain:
            line["plain_fp64"] = plain
            line["speedup_vs_plain_fp64"] = value / plain["value"]
        if parity:
            line["parity"] = parity
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["workers"], "kind": cpu["kind"],
                                    "extrapolated": True,
                                    "sample": f"{CPU_WHAT[cpu['kind']]}: per worker all pairs "
                                              f"of ~{cpu['per_worker_pairs']} consecutive-anchor pairs (every "
                                              f"distance) at a pair-weighted random SNP of the full workload, "
                                              f"{cpu['workers']} spawn workers, {cpu['wall_s']:.1f} s wall; the "
                                              f"rate extrapolates the full workload's CPU time"}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def run_all_pairs(args):
    """All-pairs LD of one SNP set (pairwise r^2 / sigma_D^2 / count r^2 for every pair,
    the matrix written to HBM unless --reduce-only): one JSON line, roofline against HBM
    (matrix bytes written) or, reduce-only, against the INT8 tensor peak."""
    import torch
    from pg_gpu_b200 import _lib, ld_matrix, synth
    lib = _lib.load()
    rng = np.random.default_rng(6)
    m, n = args.snps, args.haplotypes
    est = ld_matrix.ESTIMATORS[args.estimator]
    geno = est >= 3
    # genotype estimators: dosages of paired haplotypes (complete data where the estimator needs it)
    hap, _pos = synth.haplotype_region(rng, [2 * n if geno else n], m, m * 100,
                                       0.0 if args.estimator in ("rogers_huff_r", "sigma_d2_geno") else 0.01)
    if geno:
        g = (np.maximum(hap[0::2], 0) + np.maximum(hap[1::2], 0)).astype(np.int8)
        g[(hap[0::2] < 0) | (hap[1::2] < 0)] = -1
        hap = g
    X = torch.as_tensor(np.ascontiguousarray(hap), device="cuda")
    R = torch.arange(n, dtype=torch.int32, device="cuda")
    M = None if args.reduce_only else torch.empty((m, m), dtype=torch.float64, device="cuda")
    S = torch.zeros(2, dtype=torch.float64, device="cuda")
    wsb = torch.empty(int(lib.ldk_ld_matrix_workspace_size(m, n)), dtype=torch.uint8, device="cuda")

    def step():
        _lib.check(lib.ldk_ld_matrix(_lib.ptr(X), m, m, _lib.ptr(R), n, est, _lib.ptr(M), m, _lib.ptr(S),
                                     _lib.ptr(wsb), wsb.numel(), _lib.stream_handle()))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    pairs = m * (m - 1) // 2
    pk_d, pk_kind = peaks()
    probe_i8, _ = _lib.probe_peaks()
    if M is not None:
        bytes_ = m * m * 8
        roof = {"bound": "hbm", "achieved": bytes_ / (ms / 1e3) / 1e9, "peak": pk_d["hbm_gbs"], "unit": "GB/s",
                "peak_source": f"{pk_kind} copy bandwidth", "algorithmic_bytes": bytes_}
    else:
        ops = (18 if geno else 8) * n * pairs
        roof = {"bound": "tensor", "achieved": ops / (ms / 1e3) / 1e12, "peak": probe_i8 / 1e12,
                "unit": "TOP/s (INT8, MAC=2)", "peak_source": "measured in this run: ldk_probe_peaks"}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["traffic"] = None
    print(json.dumps({
        "metric": "all-pairs LD SNP-pairs/s", "value": pairs / (ms / 1e3), "unit": "SNP-pairs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8 counts / s32 accumulate / f64 values",
        "data": "synthetic (seeded founder mosaics, 1% missing)",
        "config": {"workload": f"all-pairs {args.estimator}, {m} SNPs x {n} {'individuals' if geno else 'haplotypes'}",
                   "matrix": M is not None, "pairs": pairs, "l2": "matrix larger than L2" if M is not None else
                   "reduction only"},
        "roofline": roof, "gpu_launches": int(args.steps * ((M is not None) + (est == 0) + geno + 3)),
        "clocks": clk.summary()}),
        flush=True)


def parser_ktot(w):
    k = sum((len(r) + 31) // 32 * 32 for r in w.pop_rows)
    return (k + 127) // 128 * 128


def run_reference(args, ws, rank):
    """pg_gpu's path on the CPU -- its own estimator kernels compiled for the host where they
    cover the workload, else the oracle's restatement -- all host cores, bounded samples."""
    if ws > 1 and rank != 0:
        return
    w = bench_workload(args, 0)
    cores = cpu_cores()
    # each step a bounded sample (~4 s of every core), so that K + W steps end in a few minutes
    per_step = max(2.0, min(args.cpu_seconds, 200.0 / max(1, args.steps + args.warmup)) / 4.0)
    pool = cpu_pool(cores)
    for k in range(max(0, min(args.warmup, 1))):
        run_cpu_sample(w, 1.0, cores, pool, seed=100 + k)
    vals, pairs, wall = [], 0, 0.0
    kind = cpu_kind(w)
    for k in range(args.steps):
        r = run_cpu_sample(w, per_step, cores, pool, seed=k)
        vals.append(r["value"])
        pairs += r["pairs"]
        wall += r["wall_s"]
    pool.close()
    pool.join()
    value = pairs / wall
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded founder mosaics)",
            "config": {"workload": w.name, "config_index": args.config, "scale": args.scale},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "extrapolated": True,
                             "sample": f"{CPU_WHAT[kind]}; per step and worker all "
                                       f"pairs of a run of consecutive anchors at a pair-weighted random SNP "
                                       f"of the full workload (every distance), {cores} workers, "
                                       f"~{per_step:.0f} s per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
