"""Drop-in for ``pg_gpu.moments_ld.compute_ld_statistics`` (``pg_gpu/moments_ld.py:40-203``),
itself moments.LD.Parsing.compute_ld_statistics' signature, on libldk.

The bin loop of ``_compute_ld_sums`` (:309-341) is one ``ldk_parse`` call; bins are
right-open with ``d == bins[-1]`` dropped; with ``r_bins`` the genetic map is
interpolated on the host (:211-223) and the physical cutoff bounded (:226-245).  The
returned dict has moments' layout: ``bins``, ``sums`` = [bin_0 .. bin_{B-1}, H], ``stats``
= (ld_names, het_names), ``pops``.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .genotype_matrix import GenotypeMatrix
from .haplotype_matrix import HaplotypeMatrix
from .ld_pipeline import het_names, ld_names


def _interpolate_genetic_distances(positions, rec_map_file):
    """Per-variant map positions in Morgans from a (pos, cM) map (moments_ld.py:211-223)."""
    map_pos, map_vals = [], []
    with open(rec_map_file) as f:
        for line in f:
            parts = line.strip().split()
            if len(parts) >= 2:
                try:
                    map_pos.append(float(parts[0]))
                    map_vals.append(float(parts[1]) / 100.0)
                except ValueError:
                    continue
    return np.interp(positions, np.array(map_pos), np.array(map_vals))


def _max_bp_for_r_dist(positions, gen_dists, max_r):
    """Conservative bp cutoff for a genetic-distance cutoff (moments_ld.py:226-245)."""
    chrom_len = float(positions[-1] - positions[0])
    if len(positions) < 2:
        return chrom_len
    bp = np.diff(positions).astype(np.float64)
    rd = np.diff(gen_dists)
    valid = bp > 0
    if not np.any(valid):
        return chrom_len
    rates = rd[valid] / bp[valid]
    min_rate = np.min(rates[rates > 0]) if np.any(rates > 0) else max_r / chrom_len
    return min(max_r / min_rate * 1.1, chrom_len)


def _to_np(x):
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)


def _compute_ld_sums(mat, pops, bins, gen_dists, max_bp_dist, use_genotypes=False, method=None):
    """(n_bins, n_ld) float64 sums (moments_ld.py:248-343)."""
    torch = _lib.require_cuda()
    from .parse import ld_parse
    if use_genotypes:
        mat.transfer_to_gpu()
        union = sorted(set(int(i) for p in pops for i in mat.sample_sets[p]))
        keep = mat.biallelic_keep(rows=union).nonzero().flatten()
        data = mat.genotypes.index_select(1, keep).contiguous()
        pos = mat.positions.index_select(0, keep)
        gd = None if gen_dists is None else np.asarray(gen_dists)[keep.cpu().numpy()]
        method = method or "auto"
    else:
        mat.transfer_to_gpu()
        data, pos, gd = mat.haplotypes, mat.positions, gen_dists
        method = method or "auto"
    rows = [np.asarray(mat.sample_sets[p]) for p in pops]
    res = ld_parse(data, pos.to(torch.float64), rows, bins, genotypes=use_genotypes, method=method,
                   max_dist=float(max_bp_dist), coords=gd).numpy()
    return res["sums"][0]


def _compute_heterozygosity(mat, pops, use_genotypes=False):
    """H_i_j sums over sites (moments_ld.py:346-388), on the GPU."""
    torch = _lib.require_cuda()
    alt, ref, nh = [], [], []
    for p in pops:
        idx = torch.as_tensor(list(mat.sample_sets[p]), device="cuda")
        if use_genotypes:
            g = mat.genotypes.index_select(0, idx)
            v = g >= 0
            a = torch.where(v, g, torch.zeros_like(g)).to(torch.int64).sum(0).to(torch.float64)
            n = 2.0 * v.sum(0).to(torch.float64)
        else:
            h = mat.haplotypes.index_select(0, idx)
            a = h.clamp(min=0).to(torch.int64).sum(0).to(torch.float64)
            n = torch.full_like(a, float(len(mat.sample_sets[p])))
        alt.append(a)
        ref.append(n - a)
        nh.append(n)
    out = {}
    for i in range(len(pops)):
        for j in range(i, len(pops)):
            if i == j:
                v = (2.0 * ref[i] * alt[i] / (nh[i] * (nh[i] - 1))).sum()
            else:
                v = ((ref[i] * alt[j] + alt[i] * ref[j]) / (nh[i] * nh[j])).sum()
            out[f"H_{i}_{j}"] = float(v.item())
    return out


def compute_ld_statistics(vcf_file=None, rec_map_file=None, pop_file=None, pops=None, r_bins=None, bp_bins=None,
                          use_genotypes=False, report=True, ac_filter=True, haplotype_matrix=None,
                          genotype_matrix=None, accessible_bed=None, method=None):
    """moments-format LD statistics for 1-4 populations (moments_ld.py:40-203).

    ``method``: "auto" (the default: "tc", or "plain" for shapes the tensor-core kernel
    cannot stage), "tc" (tensor-core counts, FP64 estimators) or "plain" (byte-counting
    FP64 kernel).  ``accessible_bed`` is not supported
    (masking is ingest, outside this library)."""
    if pops is None:
        pops = ["pop0", "pop1"]
    if not 1 <= len(pops) <= 4:
        raise ValueError("1-4 populations supported")
    if r_bins is None and bp_bins is None:
        raise ValueError("Either r_bins or bp_bins must be provided")
    if accessible_bed is not None:
        raise NotImplementedError("accessibility masks are outside the LD parse; filter the matrix first")
    if use_genotypes:
        if genotype_matrix is not None:
            mat = genotype_matrix
        elif haplotype_matrix is not None:
            mat = GenotypeMatrix.from_haplotype_matrix(haplotype_matrix)
        else:
            if vcf_file is None:
                raise ValueError("vcf_file or genotype_matrix required")
            if pop_file is None:
                raise ValueError("pop_file is required when loading from VCF")
            mat = GenotypeMatrix.from_vcf(vcf_file)
            mat.load_pop_file(pop_file, pops=pops)
            if ac_filter:
                mat = mat.apply_biallelic_filter()
        if report:
            print(f"  {mat.num_individuals} individuals, {mat.num_variants:,} variants")
    else:
        if haplotype_matrix is not None:
            mat = haplotype_matrix
        else:
            if vcf_file is None:
                raise ValueError("vcf_file or haplotype_matrix is required")
            if pop_file is None:
                raise ValueError("pop_file is required when loading from VCF")
            mat = HaplotypeMatrix.from_vcf(vcf_file)
            mat.load_pop_file(pop_file, pops=pops)
            if ac_filter:
                mat = mat.apply_biallelic_filter()
        if report:
            print(f"  {mat.num_haplotypes} hap, {mat.num_variants:,} variants")
    mat.transfer_to_gpu()
    pos_cpu = _to_np(mat.positions)
    if r_bins is not None:
        if rec_map_file is None:
            raise ValueError("rec_map_file required with r_bins")
        bins = np.asarray(r_bins, dtype=np.float64)
        gen = _interpolate_genetic_distances(pos_cpu, rec_map_file)
        max_bp = _max_bp_for_r_dist(pos_cpu, gen, float(bins[-1]))
    else:
        bins = np.asarray(bp_bins, dtype=np.float64)
        gen = None
        max_bp = float(bins[-1])
    n_bins = len(bins) - 1
    if report:
        print(f"  Computing LD ({n_bins} bins, {len(pops)} pops) ...")
    ld_sums = _compute_ld_sums(mat, pops, bins, gen, max_bp, use_genotypes=use_genotypes, method=method)
    het = _compute_heterozygosity(mat, pops, use_genotypes=use_genotypes)
    hn = het_names(len(pops))
    return {"bins": [(float(bins[i]), float(bins[i + 1])) for i in range(n_bins)],
            "sums": [ld_sums[i] for i in range(n_bins)] + [np.array([het[h] for h in hn])],
            "stats": (ld_names(len(pops)), hn), "pops": pops}
