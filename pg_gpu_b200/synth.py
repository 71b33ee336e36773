"""Seeded synthetic LD workloads (no public dataset is available offline).

Haplotypes are mosaics of 20 founders: per SNP the founders' derived-allele count k in
1..19 is drawn with P(k) ~ 1/k (neutral SFS) and k random founders carry allele 1; each
haplotype starts on a random founder and switches at Poisson breakpoints (rate per bp)
to a random founder, so LD decays with distance.  With several populations the
founders are shared and each population resamples every founder allele as
Bernoulli(p'), p' ~ Beta(p(1-F)/F, (1-p)(1-F)/F) (drift F).  Missing entries are
i.i.d. Bernoulli(rate), stored as -1.  Sites not polymorphic in the union of the
populations are dropped (the reference's biallelic filter).

``make_config(k, scale)`` builds configuration k in 1..5 at full size (scale = 1) or
scaled down for tests.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

N_FOUNDERS = 20


@dataclass
class Workload:
    name: str
    data: np.ndarray              # (n_rows, n_var) int8: haplotypes or genotypes
    positions: np.ndarray         # (n_var,) float64
    pop_rows: list                # row indices per population
    edges: np.ndarray             # bin edges
    max_dist: float
    genotypes: bool = False
    window_offsets: np.ndarray | None = None
    snp_block: np.ndarray | None = None
    n_blocks: int = 1
    replicate_weights: np.ndarray | None = None  # (n_rep, n_blocks) bootstrap multiplicities
    window_of_block: np.ndarray | None = None
    meta: dict = field(default_factory=dict)
    anchor_end: np.ndarray | None = None  # per window: left SNPs end here (a rank's slab of a split)

    @property
    def n_var(self):
        return self.data.shape[1]


def _sfs_counts(rng, m):
    k = np.arange(1, N_FOUNDERS)
    p = (1.0 / k) / np.sum(1.0 / k)
    return rng.choice(k, size=m, p=p)


def _founders(rng, m):
    """(N_FOUNDERS, m) founder alleles with a 1/k derived-count spectrum."""
    kk = _sfs_counts(rng, m)
    keys = rng.random((N_FOUNDERS, m))
    ranks = np.argsort(np.argsort(keys, axis=0), axis=0)
    return (ranks < kk[None, :]).astype(np.int8)


def _drift(rng, founders, F):
    p = founders.mean(axis=0)
    a = np.maximum(p * (1 - F) / F, 1e-6)
    b = np.maximum((1 - p) * (1 - F) / F, 1e-6)
    pp = rng.beta(a, b)
    return (rng.random(founders.shape) < pp[None, :]).astype(np.int8)


def _mosaic(rng, founders, positions, span, n_hap, switch_rate):
    m = len(positions)
    out = np.empty((n_hap, m), dtype=np.int8)
    cols = np.arange(m)
    for h in range(n_hap):
        nbreak = rng.poisson(switch_rate * span)
        breaks = np.sort(rng.uniform(0, span, nbreak))
        seg = rng.integers(0, N_FOUNDERS, nbreak + 1)
        f = seg[np.searchsorted(breaks, positions - positions[0], side="right")]
        out[h] = founders[f, cols]
    return out


def _positions(rng, m, span, start=0):
    pos = np.unique(rng.choice(int(span), size=min(int(m * 1.02) + 8, int(span)), replace=False))
    if len(pos) > m:
        pos = np.sort(rng.choice(pos, size=m, replace=False))
    return (pos + start).astype(np.int64)


def haplotype_region(rng, sizes, m, span, missing, F=0.05, switch_rate=1e-5, start=0):
    """One region: (n_hap_total, m) int8 haplotypes, positions; populations stacked."""
    pos = _positions(rng, m, span, start)
    fo = _founders(rng, len(pos))
    mats = []
    for n in sizes:
        fp = _drift(rng, fo, F) if len(sizes) > 1 else fo
        mats.append(_mosaic(rng, fp, pos.astype(np.float64), span, n, switch_rate))
    hap = np.concatenate(mats, axis=0)
    if missing:
        hap[rng.random(hap.shape) < missing] = -1
    return hap, pos


def _poly_keep_hap(hap):
    return (np.sum(hap == 0, axis=0) > 0) & (np.sum(hap == 1, axis=0) > 0)


def _poly_keep_geno(g):
    v = g >= 0
    alt = np.where(v, g, 0).astype(np.int64).sum(axis=0)
    nv = v.sum(axis=0)
    return (alt > 0) & (alt < 2 * nv) & (nv >= 2)


def _rows(sizes):
    off = np.concatenate([[0], np.cumsum(sizes)])
    return [np.arange(off[p], off[p + 1], dtype=np.int32) for p in range(len(sizes))]


def config1(scale=1.0, seed=1):
    """1 pop x 100 haplotypes, 5,000 SNPs on 1 Mb, no missing, bins [0,1e3,1e4,1e5,1e6]."""
    rng = np.random.default_rng(seed)
    m = max(50, int(5000 * scale))
    hap, pos = haplotype_region(rng, [100], m, 1_000_000, 0.0)
    keep = _poly_keep_hap(hap)
    return Workload("C1: 1 pop x 100 hap, 5k SNPs / 1 Mb", hap[:, keep].copy(), pos[keep].astype(np.float64),
                    _rows([100]), np.array([0.0, 1e3, 1e4, 1e5, 1e6]), 1e6)


def config2(scale=1.0, seed=2):
    """2 pops (100, 140), 50,000 SNPs on 5 Mb, 5% missing, 16 log bins 10 bp .. 1 Mb."""
    rng = np.random.default_rng(seed)
    m = max(80, int(50_000 * scale))
    span = max(20_000, int(5_000_000 * scale))
    hap, pos = haplotype_region(rng, [100, 140], m, span, 0.05)
    keep = _poly_keep_hap(hap)
    return Workload("C2: 2 pops (100, 140), 50k SNPs / 5 Mb, 5% missing", hap[:, keep].copy(),
                    pos[keep].astype(np.float64), _rows([100, 140]), np.logspace(1, 6, 17), 1e6)


def config3(scale=1.0, seed=3):
    """500 diploids (sums of two mosaic haplotypes), 100,000 SNPs on 10 Mb, 2% missing,
    cutoff 200 kb, 20 linear bins on [0, 2e5]."""
    rng = np.random.default_rng(seed)
    m = max(80, int(100_000 * scale))
    span = max(40_000, int(10_000_000 * scale))
    n_ind = max(20, int(500 * min(1.0, scale * 10)))
    hap, pos = haplotype_region(rng, [2 * n_ind], m, span, 0.0)
    geno = (hap[0::2] + hap[1::2]).astype(np.int8)
    geno[rng.random(geno.shape) < 0.02] = -1
    keep = _poly_keep_geno(geno)
    return Workload(f"C3: {n_ind} diploids, 100k SNPs / 10 Mb, 2% missing", geno[:, keep].copy(),
                    pos[keep].astype(np.float64), _rows([n_ind]), np.linspace(0, 2e5, 21), 2e5, genotypes=True)


def config4(scale=1.0, seed=4, n_windows=200, n_rep=100, block_bp=50_000):
    """200 windows (lognormal SNP counts, median 2,000, clipped to [200, 20,000], 0.01 SNP/bp),
    3 pops (50, 120, 300), 3% missing, 16 log bins 10 bp .. 1 Mb, 50-kb bootstrap blocks,
    100 replicates."""
    rng = np.random.default_rng(seed)
    nw = max(2, int(round(n_windows * min(1.0, scale * 20)))) if scale < 1 else n_windows
    sizes_snps = np.clip(np.exp(rng.normal(np.log(2000), np.log(10) / 3, nw)), 200, 20_000).astype(int)
    if scale < 1:
        sizes_snps = np.maximum(40, (sizes_snps * scale * 10).astype(int))
    pops = [50, 120, 300]
    mats, poss, offs, blocks, wob = [], [], [0], [], []
    nblk = 0
    for w, m in enumerate(sizes_snps):
        span = int(m * 100)
        hap, pos = haplotype_region(rng, pops, int(m), span, 0.03, start=0)
        keep = _poly_keep_hap(hap)
        hap, pos = hap[:, keep], pos[keep]
        mats.append(hap)
        poss.append(pos.astype(np.float64))
        offs.append(offs[-1] + hap.shape[1])
        b = ((pos - pos[0]) // block_bp).astype(np.int32)
        blocks.append(b + nblk)
        wob += [w] * (int(b.max()) + 1 if len(b) else 0)
        nblk += int(b.max()) + 1 if len(b) else 0
    data = np.concatenate(mats, axis=1)
    positions = np.concatenate(poss)
    snp_block = np.concatenate(blocks).astype(np.int32)
    rep = np.zeros((n_rep, nblk), dtype=np.int32)
    for r in range(n_rep):
        idx = rng.integers(0, nblk, size=nblk)
        rep[r] = np.bincount(idx, minlength=nblk)
    return Workload(f"C4: {nw} windows x 3 pops (50/120/300), 3% missing, {n_rep} bootstrap reps",
                    data, positions, _rows(pops), np.logspace(1, 6, 17), 1e6,
                    window_offsets=np.asarray(offs, dtype=np.int64), snp_block=snp_block, n_blocks=nblk,
                    replicate_weights=rep, window_of_block=np.asarray(wob, dtype=np.int32),
                    meta={"window_snps": np.diff(offs).tolist()})


def config5(scale=1.0, seed=5):
    """1 pop x 2,000 haplotypes, 1,000,000 SNPs on 50 Mb, 1% missing, cutoff 100 kb,
    32 log bins over [10, 1e5]."""
    rng = np.random.default_rng(seed)
    m = max(100, int(1_000_000 * scale))
    span = max(50_000, int(50_000_000 * scale))
    n = 2000 if scale >= 0.01 else max(64, int(2000 * scale * 100))
    hap, pos = haplotype_region(rng, [n], m, span, 0.01)
    keep = _poly_keep_hap(hap)
    return Workload(f"C5: 1 pop x {n} hap, 1e6 SNPs / 50 Mb, 1% missing", hap[:, keep].copy(),
                    pos[keep].astype(np.float64), _rows([n]), np.logspace(1, 5, 33), 1e5)


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}


def make_config(k: int, scale: float = 1.0, **kw) -> Workload:
    return CONFIGS[k](scale=scale, **kw)


def count_pairs(w: Workload) -> int:
    """Pairs i < j within a window with pos[j] - pos[i] <= max_dist."""
    offs = w.window_offsets if w.window_offsets is not None else np.array([0, w.n_var])
    tot = 0
    for k, (a, b) in enumerate(zip(offs[:-1], offs[1:])):
        p = w.positions[a:b]
        jm = np.searchsorted(p, p + w.max_dist, side="right")
        per = np.maximum(0, jm - np.arange(len(p)) - 1)
        if w.anchor_end is not None:
            per = per[:max(0, int(w.anchor_end[k]) - a)]
        tot += int(np.sum(per))
    return tot
