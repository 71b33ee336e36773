"""``GenotypeMatrix`` for the unphased genotype LD path (``pg_gpu/genotype_matrix.py``).

(n_individuals, n_variants) int8 in {0, 1, 2, -1}, positions, sample sets; built from a
``HaplotypeMatrix`` by summing consecutive haplotype pairs (genotype_matrix.py:255-305).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .haplotype_matrix import read_pop_file, read_vcf


class GenotypeMatrix:
    def __init__(self, genotypes, positions, chrom_start=None, chrom_end=None, sample_sets=None, samples=None):
        self.genotypes = genotypes
        self.positions = positions
        self.samples = samples
        self._sample_sets = dict(sample_sets) if sample_sets else None
        pos = positions.detach().cpu().numpy() if hasattr(positions, "detach") else np.asarray(positions)
        self.chrom_start = chrom_start if chrom_start is not None else (int(pos[0]) if len(pos) else 0)
        self.chrom_end = chrom_end if chrom_end is not None else (int(pos[-1]) if len(pos) else 0)

    @property
    def device(self):
        return "GPU" if hasattr(self.genotypes, "is_cuda") and self.genotypes.is_cuda else "CPU"

    @property
    def num_individuals(self):
        return int(self.genotypes.shape[0])

    @property
    def num_variants(self):
        return int(self.genotypes.shape[1])

    @property
    def sample_sets(self):
        if self._sample_sets is None:
            return {"all": list(range(self.num_individuals))}
        return self._sample_sets

    @sample_sets.setter
    def sample_sets(self, value):
        self._sample_sets = dict(value) if value is not None else None

    def transfer_to_gpu(self):
        torch = _lib.require_cuda()
        if self.device != "GPU":
            self.genotypes = torch.as_tensor(np.ascontiguousarray(self.genotypes), dtype=torch.int8, device="cuda")
            self.positions = torch.as_tensor(np.asarray(self.positions), device="cuda")
        return self

    @classmethod
    def from_haplotype_matrix(cls, hm):
        """Individual k = haplotypes 2k and 2k+1; -1 if either is missing."""
        hap = hm.haplotypes
        if hap.shape[0] % 2:
            raise ValueError(f"Need even number of haplotypes for diploid conversion, got {hap.shape[0]}")
        if hasattr(hap, "is_cuda"):
            h1, h2 = hap[0::2], hap[1::2]
            g = (h1.clamp(min=0) + h2.clamp(min=0)).to(hap.dtype)
            g[(h1 < 0) | (h2 < 0)] = -1
        else:
            h1, h2 = hap[0::2], hap[1::2]
            g = (np.maximum(h1, 0) + np.maximum(h2, 0)).astype(np.int8)
            g[(h1 < 0) | (h2 < 0)] = -1
        sets = None
        if hm._sample_sets is not None:
            sets = {name: sorted(set(int(i) // 2 for i in idx)) for name, idx in hm._sample_sets.items()}
        return cls(g, hm.positions, hm.chrom_start, hm.chrom_end, sample_sets=sets)

    @classmethod
    def from_vcf(cls, path):
        hap, pos, samples = read_vcf(path)
        n = len(samples)
        a, b = hap[:n], hap[n:]
        g = (np.maximum(a, 0) + np.maximum(b, 0)).astype(np.int8)
        g[(a < 0) | (b < 0)] = -1
        return cls(g, pos, samples=samples)

    def load_pop_file(self, pop_file, pops=None):
        if self.samples is None:
            raise ValueError("No sample names stored. Use from_vcf() to load data.")
        pop_map = read_pop_file(pop_file)
        if pops is None:
            pops = sorted(set(pop_map.values()))
        sets = {p: [] for p in pops}
        for i, name in enumerate(self.samples):
            if pop_map.get(name) in sets:
                sets[pop_map[name]].append(i)
        self.sample_sets = sets

    def biallelic_keep(self, rows=None):
        """Boolean keep mask: alt count strictly between 0 and 2 x valid, >= 2 valid
        (genotype_matrix.py:506-539; over the given rows as in moments_ld.py:256-278)."""
        g = self.genotypes
        if rows is not None:
            g = g[list(rows)] if not hasattr(g, "is_cuda") else g.index_select(
                0, _lib.require_cuda().as_tensor(list(rows), device=g.device))
        if hasattr(g, "is_cuda"):
            v = g >= 0
            alt = g.clamp(min=0).to(_lib.require_cuda().int64).sum(0)
            nv = v.sum(0)
            return (alt > 0) & (alt < 2 * nv) & (nv >= 2)
        v = g >= 0
        alt = np.maximum(g, 0).astype(np.int64).sum(0)
        nv = v.sum(0)
        return (alt > 0) & (alt < 2 * nv) & (nv >= 2)

    def apply_biallelic_filter(self):
        keep = self.biallelic_keep()
        if hasattr(keep, "is_cuda"):
            idx = keep.nonzero().flatten()
            return GenotypeMatrix(self.genotypes.index_select(1, idx).contiguous(), self.positions.index_select(0, idx),
                                  self.chrom_start, self.chrom_end, sample_sets=self._sample_sets, samples=self.samples)
        return GenotypeMatrix(self.genotypes[:, keep], np.asarray(self.positions)[keep], self.chrom_start,
                              self.chrom_end, sample_sets=self._sample_sets, samples=self.samples)
