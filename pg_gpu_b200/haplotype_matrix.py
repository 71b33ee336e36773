"""``HaplotypeMatrix`` with pg_gpu's LD methods (``pg_gpu/haplotype_matrix.py``), on libldk.

Only what the two-locus LD parse needs: the (n_haplotypes, n_variants) int8 matrix in
{0, 1, -1}, positions, population sample sets, the biallelic filter, a plain-text VCF
reader for phased biallelic calls, and ``compute_ld_statistics_gpu_single_pop`` /
``_two_pops`` / ``compute_ld_statistics`` (any 1..4 populations) with the reference's
return conventions.  Data may live on the host (numpy) or the GPU (torch).
"""
from __future__ import annotations

import gzip
from collections import OrderedDict

import numpy as np

from . import _lib
from .ld_pipeline import ld_names


def _open_text(path):
    return gzip.open(path, "rt") if str(path).endswith(".gz") else open(path)


def read_vcf(path):
    """Phased text VCF -> (haplotypes (2*n_samples, n_var) int8 with the first alleles of all
    samples then the second alleles (haplotype_matrix.py:326-329), positions int64,
    sample names).  Missing alleles ('.') become -1; ALT alleles beyond the first keep
    their index (>= 2) so that the biallelic filter drops the site."""
    pos, rows, samples = [], [], None
    with _open_text(path) as f:
        for line in f:
            if line.startswith("##"):
                continue
            parts = line.rstrip("\n").split("\t")
            if line.startswith("#"):
                samples = parts[9:]
                continue
            pos.append(int(parts[1]))
            first, second = [], []
            for gt in parts[9:]:
                g = gt.split(":")[0].replace("/", "|").split("|")
                a = g[0]
                b = g[1] if len(g) > 1 else g[0]
                first.append(-1 if a == "." else int(a))
                second.append(-1 if b == "." else int(b))
            rows.append(first + second)
    if samples is None:
        raise ValueError(f"{path}: no #CHROM header")
    hap = np.asarray(rows, dtype=np.int8).T.copy() if rows else np.zeros((2 * len(samples), 0), np.int8)
    return hap, np.asarray(pos, dtype=np.int64), samples


def read_pop_file(pop_file):
    """sample -> population (tab/space separated; a header line starting 'sample' skipped)."""
    pop_map = {}
    with open(pop_file) as f:
        for line in f:
            parts = line.strip().split()
            if len(parts) >= 2 and parts[0] != "sample":
                pop_map[parts[0]] = parts[1]
    return pop_map


class HaplotypeMatrix:
    def __init__(self, genotypes, positions, chrom_start=None, chrom_end=None, sample_sets=None, samples=None):
        self.haplotypes = genotypes
        self.positions = positions
        self.samples = samples
        self._sample_sets = dict(sample_sets) if sample_sets else None
        pos = self._np(positions)
        self.chrom_start = chrom_start if chrom_start is not None else (int(pos[0]) if len(pos) else 0)
        self.chrom_end = chrom_end if chrom_end is not None else (int(pos[-1]) if len(pos) else 0)

    # -- basics -------------------------------------------------------------
    @staticmethod
    def _np(x):
        return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)

    @property
    def device(self):
        return "GPU" if hasattr(self.haplotypes, "is_cuda") and self.haplotypes.is_cuda else "CPU"

    @property
    def num_haplotypes(self):
        return int(self.haplotypes.shape[0])

    @property
    def num_variants(self):
        return int(self.haplotypes.shape[1])

    @property
    def sample_sets(self):
        if self._sample_sets is None:
            return {"all": list(range(self.num_haplotypes))}
        return self._sample_sets

    @sample_sets.setter
    def sample_sets(self, value):
        self._sample_sets = dict(value) if value is not None else None

    def transfer_to_gpu(self):
        torch = _lib.require_cuda()
        if self.device != "GPU":
            self.haplotypes = torch.as_tensor(np.ascontiguousarray(self.haplotypes), dtype=torch.int8, device="cuda")
            self.positions = torch.as_tensor(np.asarray(self.positions), device="cuda")
        return self

    def transfer_to_cpu(self):
        self.haplotypes = self._np(self.haplotypes)
        self.positions = self._np(self.positions)
        return self

    @classmethod
    def from_vcf(cls, path):
        hap, pos, samples = read_vcf(path)
        return cls(hap, pos, samples=samples)

    def load_pop_file(self, pop_file, pops=None):
        """Sample sets from a population file; haplotypes i and i + n_samples of sample i
        (haplotype_matrix.py:475-512)."""
        if self.samples is None:
            raise ValueError("No sample names stored. Use from_vcf() to load data.")
        pop_map = read_pop_file(pop_file)
        if pops is None:
            pops = sorted(set(pop_map.values()))
        n = len(self.samples)
        sets = {p: [] for p in pops}
        for i, name in enumerate(self.samples):
            p = pop_map.get(name)
            if p in sets:
                sets[p] += [i, i + n]
        self.sample_sets = sets

    def apply_biallelic_filter(self):
        """Keep sites with both alleles 0 and 1 present and no allele >= 2
        (haplotype_matrix.py:724-789)."""
        h = self.haplotypes
        if self.device == "GPU":
            keep = ((h == 0).any(0) & (h == 1).any(0) & ~(h >= 2).any(0)).nonzero().flatten()
            hap, pos = h.index_select(1, keep).contiguous(), self.positions.index_select(0, keep)
        else:
            keep = np.flatnonzero((h == 0).any(0) & (h == 1).any(0) & ~(h >= 2).any(0))
            hap, pos = h[:, keep], np.asarray(self.positions)[keep]
        return HaplotypeMatrix(hap, pos, sample_sets=self._sample_sets, samples=self.samples)

    # -- LD -------------------------------------------------------------------
    def _parse(self, bp_bins, pop_rows, method):
        from .parse import ld_parse
        self.transfer_to_gpu()
        edges = np.asarray(bp_bins, dtype=np.float64)
        return ld_parse(self.haplotypes, self.positions.double(), pop_rows, edges, method=method,
                        max_dist=float(edges[-1])).numpy()

    @staticmethod
    def _bin_dict(bp_bins, names, res, raw, as_tuple):
        edges = np.asarray(bp_bins, dtype=np.float64)
        out = {}
        sums, pairs = res["sums"][0], res["pairs"][0]
        for b in range(len(edges) - 1):
            key = (float(edges[b]), float(edges[b + 1]))
            if raw:
                vals = sums[b]
            else:
                vals = sums[b] / pairs[b] if pairs[b] > 0 else np.zeros_like(sums[b])
            vals = [float(v) for v in vals]
            out[key] = tuple(vals) if as_tuple else OrderedDict(zip(names, vals))
        return out

    def pairwise_r2(self, estimator="r2"):
        """(n_variants, n_variants) float64 pairwise r^2 on the GPU
        (haplotype_matrix.py:1138-1175); ``estimator='sigma_d2'`` gives the unbiased
        sigma_D^2 matrix instead, ``'rogers_huff'`` the Rogers-Huff r^2 of paired
        haplotypes (NaN set to 0)."""
        from .ld_matrix import dosages, ld_matrix
        if estimator == "rogers_huff":  # haplotype_matrix.py:1159-1165: squared, NaN -> 0, diagonal 0
            r = ld_matrix(dosages(self), estimator="rogers_huff_r")[0]
            r2 = r * r
            r2 = r2.nan_to_num(nan=0.0)
            r2.fill_diagonal_(0.0)
            return r2
        if estimator not in ("r2", "sigma_d2"):
            raise ValueError(f"Unknown estimator: {estimator!r} (expected 'r2', 'rogers_huff' or 'sigma_d2')")
        self.transfer_to_gpu()
        return ld_matrix(self.haplotypes, estimator=estimator)[0]

    def windowed_r_squared(self, bp_bins, percentile=50, pop=None, estimator="r2"):
        """Percentiles of r^2 per genomic distance bin and pair counts
        (haplotype_matrix.py:1235-1317), over the rows of ``pop`` (default: all)."""
        from .ld_matrix import windowed_r_squared
        if estimator != "r2":
            raise NotImplementedError("only the 'r2' estimator is provided")
        self.transfer_to_gpu()
        rows = None if pop is None else self.sample_sets[pop]
        return windowed_r_squared(self.haplotypes, self._np(self.positions), bp_bins, percentile, rows=rows)

    def compute_ld_statistics_gpu_single_pop(self, bp_bins, raw=False, ac_filter=True, chunk_size="auto",
                                             method="auto"):
        """{(lo, hi): (DD, Dz, pi2)} over all haplotypes, sums if ``raw`` else means
        (haplotype_matrix.py:1592-1716).  ``chunk_size`` is accepted for compatibility: the
        parse is one library call."""
        m = self.apply_biallelic_filter() if ac_filter else self
        res = m._parse(bp_bins, [np.arange(m.num_haplotypes)], method)
        return self._bin_dict(bp_bins, ld_names(1), res, raw, as_tuple=True)

    def compute_ld_statistics_gpu_two_pops(self, bp_bins, pop1, pop2, raw=False, ac_filter=True,
                                           chunk_size="auto", method="auto"):
        """{(lo, hi): OrderedDict of the 15 two-population statistics}
        (haplotype_matrix.py:1719-1866)."""
        m = self.apply_biallelic_filter() if ac_filter else self
        sets = m.sample_sets
        res = m._parse(bp_bins, [sets[pop1], sets[pop2]], method)
        return self._bin_dict(bp_bins, ld_names(2), res, raw, as_tuple=False)

    def compute_ld_statistics(self, bp_bins, pops=None, raw=True, ac_filter=True, method="auto"):
        """{(lo, hi): OrderedDict of the moments statistics} for 1..4 named populations."""
        m = self.apply_biallelic_filter() if ac_filter else self
        sets = m.sample_sets
        pops = list(sets) if pops is None else list(pops)
        res = m._parse(bp_bins, [sets[p] for p in pops], method)
        return self._bin_dict(bp_bins, ld_names(len(pops)), res, raw, as_tuple=False)
