"""Generate the golden fixtures in this folder from the reference itself.

Runs only where the pg_gpu checkout is present (``--reference``, else the checkout that
``oracle/build_ref.py`` reads: ``PG_GPU_REFERENCE`` or its default); the fixtures it writes
are committed and are all the tests need elsewhere.

* ``im_example.npz`` -- the reference's IM example (``examples/data/im-parsing-example.vcf``
  + ``im_pop.txt``) read into the HaplotypeMatrix layout (``haplotype_matrix.py:326-329``,
  populations as rows i and i + n_samples, ``:509-510``) together with moments' own output
  cached by the reference (``tests/cache/moments_ld_test_im_4bins_deme0-deme1.pkl``).
* ``ref_ldm.npz`` -- the reference's all-pairs LD functions (pairwise r^2, sigma_D^2
  matrix, ZnS, Omega, windowed r^2 percentiles) on seeded haplotypes.
* ``ref_*.npz`` / ``ref_names.json`` -- outputs of the reference's own functions
  (``ld_pipeline``, ``ld_statistics``, ``haplotype_kernels``, ``genotype_kernels``,
  ``ld_statistics_genotype``), run on the CPU via ``oracle/ref_shim.py`` with the
  kernel bodies compiled for the host by ``oracle/build_ref.py``, on seeded inputs.

Usage: ``python tests/golden/make_golden.py [--reference PATH]``.
"""
from __future__ import annotations

import argparse
import json
import os
import pickle
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import build_ref, ref_shim  # noqa: E402


def read_vcf_haplotypes(path):
    """Phased biallelic text VCF -> (hap (2*ns, n_var) int8, pos int64, samples)."""
    pos, rows, samples = [], [], None
    with open(path) as f:
        for line in f:
            if line.startswith("##"):
                continue
            parts = line.rstrip("\n").split("\t")
            if line.startswith("#"):
                samples = parts[9:]
                continue
            pos.append(int(parts[1]))
            a, b = [], []
            for gt in parts[9:]:
                g = gt.split(":")[0].replace("/", "|").split("|")
                a.append(-1 if g[0] == "." else int(g[0]))
                b.append(-1 if g[1] == "." else int(g[1]))
            rows.append(a + b)
    hap = np.asarray(rows, dtype=np.int8).T.copy()
    return hap, np.asarray(pos, dtype=np.int64), samples


def make_im_example(reference):
    vcf = os.path.join(reference, "examples/data/im-parsing-example.vcf")
    popf = os.path.join(reference, "examples/data/im_pop.txt")
    pkl = os.path.join(reference, "tests/cache/moments_ld_test_im_4bins_deme0-deme1.pkl")
    hap, pos, samples = read_vcf_haplotypes(vcf)
    ns = len(samples)
    pop_of = {}
    with open(popf) as f:
        next(f)
        for line in f:
            s, p = line.split()
            pop_of[s] = p
    pops = ["deme0", "deme1"]
    rows = {p: [] for p in pops}
    for i, s in enumerate(samples):
        if pop_of.get(s) in rows:
            rows[pop_of[s]] += [i, i + ns]
    with open(pkl, "rb") as f:
        mom = pickle.load(f)
    edges = [mom["bins"][0][0]] + [b[1] for b in mom["bins"]]
    np.savez_compressed(
        os.path.join(HERE, "im_example.npz"),
        hap=hap, pos=pos,
        rows0=np.asarray(rows["deme0"], np.int32), rows1=np.asarray(rows["deme1"], np.int32),
        edges=np.asarray(edges, np.float64),
        ld_sums=np.asarray(mom["sums"][:-1], np.float64),
        het_sums=np.asarray(mom["sums"][-1], np.float64),
        ld_names=np.asarray(mom["stats"][0]), het_names=np.asarray(mom["stats"][1]))


def _random_hap(rng, n_hap, n_var, missing):
    h = (rng.random((n_hap, n_var)) < rng.uniform(0.05, 0.95, n_var)).astype(np.int8)
    if missing:
        h[rng.random(h.shape) < missing] = -1
    return h


def _random_geno(rng, n_ind, n_var, missing):
    p = rng.uniform(0.05, 0.95, n_var)
    g = ((rng.random((n_ind, n_var)) < p).astype(np.int8)
         + (rng.random((n_ind, n_var)) < p).astype(np.int8))
    if missing:
        g[rng.random(g.shape) < missing] = -1
    return g


def make_reference_fixtures(reference):
    mods = ref_shim.import_reference_modules(
        reference, ["ld_pipeline", "ld_statistics", "haplotype_kernels",
                    "genotype_kernels", "ld_statistics_genotype"])
    lp, ls = mods["ld_pipeline"], mods["ld_statistics"]
    hk, gk, lsg = mods["haplotype_kernels"], mods["genotype_kernels"], mods["ld_statistics_genotype"]

    names = {P: {"ld": lp.ld_names(P), "het": lp.het_names(P),
                 "specs": [[n, [[w, k, list(q)] for (w, k, q) in calls]]
                           for n, calls in lp.generate_stat_specs(P)]} for P in (1, 2, 3, 4)}
    with open(os.path.join(HERE, "ref_names.json"), "w") as f:
        json.dump(names, f)

    rng = np.random.default_rng(20261203)
    # ---- haplotype: matrices, pair lists, counts, statistics for P = 1..4 ----
    hap_out = {}
    for P in (1, 2, 3, 4):
        sizes = [int(x) for x in rng.choice([5, 8, 13, 20, 33], P)]
        n_var = 40
        miss = [0.0 if (P == 1) else 0.06 * (q % 2) for q in range(P)]
        mats = [_random_hap(rng, s, n_var, m) for s, m in zip(sizes, miss)]
        hap = np.concatenate(mats, axis=0)
        offs = np.cumsum([0] + sizes)
        ii, jj = np.triu_indices(n_var, 1)
        ii, jj = ii.astype(np.int32), jj.astype(np.int32)
        counts, nvalid = [], []
        for q in range(P):
            rows = list(range(offs[q], offs[q + 1]))
            c, nv = lp.compute_counts_for_pairs(hap, ii, jj, rows)
            counts.append(np.asarray(c))
            nvalid.append(None if nv is None else np.asarray(nv))
        cf = [c.astype(np.float64) for c in counts]
        nvf = [None if v is None else v.astype(np.float64) for v in nvalid]
        stats = hk.compute_multi_pop_statistics_batch_hap(cf, nvf, ls, lp.generate_stat_specs(P))
        hap_out[f"P{P}_hap"] = hap
        hap_out[f"P{P}_offs"] = offs
        hap_out[f"P{P}_ii"] = ii
        hap_out[f"P{P}_jj"] = jj
        for q in range(P):
            hap_out[f"P{P}_counts{q}"] = counts[q]
            hap_out[f"P{P}_nvalid{q}"] = (np.full(len(ii), -1, np.int64) if nvalid[q] is None
                                         else nvalid[q])
        hap_out[f"P{P}_stats"] = np.asarray(stats)
        if P == 2:
            hap_out["P2_twopop_stats"] = np.asarray(lp.compute_two_pop_statistics_batch(
                cf[0], cf[1], nvf[0], nvf[1], ls))
        if P == 1:
            hap_out["P1_r"] = np.asarray(ls.r(cf[0], nvf[0]))
            hap_out["P1_r2"] = np.asarray(ls.r_squared(cf[0], nvf[0]))
            hap_out["P1_dprime"] = np.asarray(ls.d_prime(cf[0], nvf[0]))
    # r^2 edge cases (tests/test_haplotype_kernels_rsq.py:92-126 and test_ld_r_squared.py)
    edge = np.array([[0, 0, 50, 50], [50, 0, 0, 50], [0, 50, 50, 0], [3, 1, 2, 4],
                     [0, 0, 0, 7], [1, 0, 0, 0]], dtype=np.float64)
    hap_out["edge_counts"] = edge
    hap_out["edge_r"] = np.asarray(ls.r(edge))
    hap_out["edge_r2"] = np.asarray(ls.r_squared(edge))
    hap_out["edge_dprime"] = np.asarray(ls.d_prime(edge))
    hap_out["edge_stats1"] = np.asarray(hk.compute_multi_pop_statistics_batch_hap(
        [edge], [None], ls, lp.generate_stat_specs(1)))
    np.savez_compressed(os.path.join(HERE, "ref_hap.npz"), **hap_out)

    # ---- genotype: counts kernel, statistics for P = 1..4, polynomial module ----
    geno_out = {}
    for P in (1, 2, 3, 4):
        sizes = [int(x) for x in rng.choice([6, 9, 14, 25], P)]
        n_var = 30
        miss = [0.05 * ((q + 1) % 2) for q in range(P)]
        mats = [_random_geno(rng, s, n_var, m) for s, m in zip(sizes, miss)]
        geno = np.concatenate(mats, axis=0)
        offs = np.cumsum([0] + sizes)
        ii, jj = np.triu_indices(n_var, 1)
        ii, jj = ii.astype(np.int32), jj.astype(np.int32)
        counts, nvalid = [], []
        for q in range(P):
            rows = np.arange(offs[q], offs[q + 1], dtype=np.int32)
            c, nv = lp.compute_genotype_counts_for_pairs(geno, ii, jj, rows)
            counts.append(np.asarray(c))
            nvalid.append(None if nv is None else np.asarray(nv))
        stats = gk.compute_multi_pop_statistics_batch_geno(counts, nvalid, None,
                                                           lp.generate_stat_specs(P))
        geno_out[f"P{P}_geno"] = geno
        geno_out[f"P{P}_offs"] = offs
        geno_out[f"P{P}_ii"] = ii
        geno_out[f"P{P}_jj"] = jj
        for q in range(P):
            geno_out[f"P{P}_counts{q}"] = counts[q]
            geno_out[f"P{P}_nvalid{q}"] = (np.full(len(ii), -1, np.int64) if nvalid[q] is None
                                          else nvalid[q])
        geno_out[f"P{P}_stats"] = np.asarray(stats)
        if P == 1:
            pd = gk._PopDataGeno(counts[0], nvalid[0])
            geno_out["P1_poly_dd"] = np.asarray(lsg.dd_geno_single(pd))
            geno_out["P1_poly_dz"] = np.asarray(lsg.dz_geno_single(pd))
            geno_out["P1_poly_pi2"] = np.asarray(lsg.pi2_geno_single(pd))
    np.savez_compressed(os.path.join(HERE, "ref_geno.npz"), **geno_out)


def make_ldm_fixtures(reference):
    """``ref_ldm.npz``: the reference's all-pairs LD functions -- HaplotypeMatrix.pairwise_r2,
    ld_statistics._build_sigma_d2_matrix, zns, omega, HaplotypeMatrix.windowed_r_squared --
    on seeded haplotypes with missing calls and monomorphic sites.  haplotype_matrix.py
    imports scikit-allel / tskit / zarr at module level; stand-in modules satisfy those
    imports (none of the functions used here touches them), and the NumPy-backed cupy
    stand-in gets a ``.get()`` on reduction results."""
    import types

    class _Stub(types.ModuleType):
        def __getattr__(self, k):
            return type(k, (), {})

    for name in ("allel", "tskit", "zarr", "msprime", "moments"):
        sys.modules.setdefault(name, _Stub(name))
    mods = ref_shim.import_reference_modules(reference, ["ld_statistics", "haplotype_matrix"])

    class _A(np.ndarray):
        def get(self):
            return np.asarray(self)

    cpm = sys.modules["cupy"]
    for fn in ("sum", "max", "trace", "digitize"):
        f = getattr(np, fn)
        setattr(cpm, fn, (lambda f: lambda *a, **k: np.asarray(f(*a, **k)).view(_A))(f))
    L = mods["ld_statistics"]
    rs = L.r_squared
    L.r_squared = lambda *a, **k: np.asarray(rs(*a, **k)).view(_A)
    HM = mods["haplotype_matrix"].HaplotypeMatrix

    rng = np.random.default_rng(77)
    n_hap, m = 64, 90
    founders = (rng.random((5, m)) < rng.uniform(0.05, 0.7, m)).astype(np.int8)
    hap = founders[rng.integers(0, 5, n_hap)]
    hap = np.where(rng.random(hap.shape) < 0.04, 1 - hap, hap).astype(np.int8)
    hap[:, 7] = 0                                  # monomorphic
    hap[:, 30] = 1                                 # monomorphic (derived everywhere)
    hap[rng.random(hap.shape) < 0.05] = -1         # missing calls
    pos = np.sort(rng.choice(200_000, m, replace=False)).astype(np.int64)
    out = {"hap": hap, "pos": pos}
    hm = HM(hap.copy(), pos.copy())
    out["pairwise_r2"] = np.asarray(hm.pairwise_r2())
    out["sigma_d2_seg"] = np.asarray(L._build_sigma_d2_matrix(HM(hap.copy(), pos.copy())))
    for md in ("include", "exclude"):
        for est in ("r2", "sigma_d2"):
            out[f"zns_{est}_{md}"] = np.float64(L.zns(HM(hap.copy(), pos.copy()), missing_data=md, estimator=est))
            out[f"omega_{est}_{md}"] = np.float64(L.omega(HM(hap.copy(), pos.copy()), missing_data=md,
                                                          estimator=est))
    for k, (bins, pct) in enumerate((([0, 1000, 5000, 20000, 200000], [10, 50, 95]), ([0, 50000, 200000], 50))):
        res, cnt = HM(hap.copy(), pos.copy()).windowed_r_squared(np.array(bins), percentile=pct)
        out[f"win{k}_bins"] = np.array(bins, dtype=np.float64)
        out[f"win{k}_pct"] = np.atleast_1d(pct).astype(np.float64)
        out[f"win{k}_res"] = np.asarray(res)
        out[f"win{k}_cnt"] = np.asarray(cnt)
    # genotype path: Rogers-Huff r and sigma_D^2 (no missing calls), dosage r^2, ZnS and
    # Omega of a GenotypeMatrix (with missing calls)
    mods_g = ref_shim.import_reference_modules(
        reference, ["ld_statistics", "genotype_matrix", "ld_statistics_genotype", "ld_pipeline", "genotype_kernels"])
    Lg = mods_g["ld_statistics"]
    for fn in ("sum", "max", "trace", "digitize"):
        f = getattr(np, fn)
        setattr(sys.modules["cupy"], fn, (lambda f: lambda *a, **k: np.asarray(f(*a, **k)).view(_A))(f))
    GM = mods_g["genotype_matrix"].GenotypeMatrix
    geno = (hap[0::2].clip(0) + hap[1::2].clip(0)).astype(np.int8)   # 32 diploids, no missing
    gpos = pos.copy()
    out["geno"] = geno
    out["rogers_huff_r"] = np.asarray(Lg.rogers_huff_r(GM(geno.copy(), gpos.copy())))
    out["sigma_d2_geno"] = np.asarray(mods_g["ld_statistics_genotype"].sigma_d2_geno(GM(geno.copy(), gpos.copy())))
    geno_m = geno.copy()
    geno_m[np.random.default_rng(78).random(geno_m.shape) < 0.04] = -1
    out["geno_missing"] = geno_m
    out["diploid_r2"] = np.asarray(Lg._r2_matrix_diploid(GM(geno_m.copy(), gpos.copy())))
    out["zns_diploid"] = np.float64(Lg.zns(GM(geno_m.copy(), gpos.copy())))
    out["omega_diploid"] = np.float64(Lg.omega(GM(geno_m.copy(), gpos.copy())))
    np.savez_compressed(os.path.join(HERE, "ref_ldm.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=build_ref.DEFAULT_REFERENCE)
    args = ap.parse_args()
    build_ref.build(args.reference)
    make_im_example(args.reference)
    make_reference_fixtures(args.reference)
    make_ldm_fixtures(args.reference)
    for f in sorted(os.listdir(HERE)):
        if f.endswith((".npz", ".json")):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
