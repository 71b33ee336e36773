"""Pin the CPU oracle against the reference's golden vectors (no GPU).

* moments' own output on the reference's IM example (2 pops x 20 haplotypes, 2599 SNPs,
  3 bins) -- the reference's tests/cache pickle, rtol 1e-10 (measured 2.9e-12);
* the reference's functions run on the host (``tests/golden/make_golden.py``):
  counts bit-exact, statistics within 1e-13 relative.
"""
import json
import os

import numpy as np
import pytest

from oracle import ld_oracle as O


def _rel(a, b, floor=1e-14):
    d = np.abs(a - b)
    r = np.abs(b)
    return np.max(np.where(r > floor, d / np.where(r > floor, r, 1), d)) if d.size else 0.0


@pytest.fixture(scope="module")
def ref_hap(golden_dir):
    return np.load(os.path.join(golden_dir, "ref_hap.npz"))


@pytest.fixture(scope="module")
def ref_geno(golden_dir):
    return np.load(os.path.join(golden_dir, "ref_geno.npz"))


def test_names_and_specs_match_reference(golden_dir):
    with open(os.path.join(golden_dir, "ref_names.json")) as f:
        ref = json.load(f)
    for P in (1, 2, 3, 4):
        r = ref[str(P)]
        assert O.ld_names(P) == r["ld"]
        assert O.het_names(P) == r["het"]
        mine = [[n, [[w, k, list(q)] for (w, k, q) in calls]] for n, calls in O.stat_specs(P)]
        assert mine == r["specs"]
    assert [len(O.ld_names(P)) for P in (1, 2, 3, 4)] == [3, 15, 45, 105]


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_hap_counts_and_stats(ref_hap, P):
    g = ref_hap
    hap, offs, ii, jj = g[f"P{P}_hap"], g[f"P{P}_offs"], g[f"P{P}_ii"], g[f"P{P}_jj"]
    cl, nl = [], []
    for q in range(P):
        c, nv = O.hap_counts(hap, ii, jj, list(range(offs[q], offs[q + 1])))
        np.testing.assert_array_equal(c, g[f"P{P}_counts{q}"])
        rnv = g[f"P{P}_nvalid{q}"]
        if nv is None:
            assert (rnv == -1).all()
        else:
            np.testing.assert_array_equal(nv, rnv)
        cl.append(c)
        nl.append(nv)
    st = O.hap_stats(cl, nl)
    assert _rel(st, g[f"P{P}_stats"]) < 1e-13
    if P == 2:
        assert _rel(st, g["P2_twopop_stats"]) < 1e-13


def test_hap_r_family_and_edges(ref_hap):
    g = ref_hap
    hap, offs, ii, jj = g["P1_hap"], g["P1_offs"], g["P1_ii"], g["P1_jj"]
    c, nv = O.hap_counts(hap, ii, jj, list(range(offs[0], offs[1])))
    for name, fn in (("P1_r", O.hap_r), ("P1_r2", O.hap_r_squared), ("P1_dprime", O.hap_d_prime)):
        np.testing.assert_allclose(fn(c, nv), g[name], rtol=1e-14, atol=1e-15, equal_nan=True)
    e = g["edge_counts"]
    np.testing.assert_allclose(O.hap_r_squared(e), g["edge_r2"], rtol=1e-14, equal_nan=True)
    # known answers: perfect LD -> 1, monomorphic -> NaN, n < 4 -> 0
    assert np.isnan(O.hap_r_squared(e)[0]) and O.hap_r_squared(e)[1] == 1.0
    np.testing.assert_array_equal(O.hap_stats([e]), g["edge_stats1"])
    assert np.all(O.hap_stats([e])[5] == 0.0)


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_geno_counts_and_stats(ref_geno, P):
    g = ref_geno
    geno, offs, ii, jj = g[f"P{P}_geno"], g[f"P{P}_offs"], g[f"P{P}_ii"], g[f"P{P}_jj"]
    cl, nl = [], []
    for q in range(P):
        c, nv = O.geno_counts(geno, ii, jj, list(range(offs[q], offs[q + 1])))
        np.testing.assert_array_equal(c, g[f"P{P}_counts{q}"])
        rnv = g[f"P{P}_nvalid{q}"]
        if nv is None:
            assert (rnv == -1).all()
        else:
            np.testing.assert_array_equal(nv, rnv)
        cl.append(c)
        nl.append(nv)
    st = O.geno_stats(cl, nl)
    ref = g[f"P{P}_stats"]
    assert np.array_equal(np.isfinite(st), np.isfinite(ref))
    f = np.isfinite(ref)
    assert _rel(st[f], ref[f]) < 1e-13
    if P == 1:
        for k, col in (("P1_poly_dd", 0), ("P1_poly_dz", 1), ("P1_poly_pi2", 2)):
            assert _rel(st[:, col], g[k]) < 1e-12


def test_moments_golden_im_example(golden_dir):
    im = np.load(os.path.join(golden_dir, "im_example.npz"))
    hap, pos = im["hap"], im["pos"]
    keep = O.biallelic_keep(hap)
    hap, pos = hap[:, keep], pos[keep]
    assert hap.shape == (40, 2599)
    rows = [im["rows0"], im["rows1"]]
    res = O.bin_sums(hap, pos, rows, im["edges"])
    assert res["n_pairs"] == 640143
    assert _rel(res["sums"][0], im["ld_sums"]) < 1e-10
    H = O.heterozygosity(hap, rows)
    np.testing.assert_allclose([H[k] for k in O.het_names(2)], im["het_sums"], rtol=1e-12)
    assert list(im["ld_names"]) == O.ld_names(2)


def _naive_pairs(pos, max_dist):
    return {(i, j) for i in range(len(pos)) for j in range(i + 1, len(pos))
            if pos[j] - pos[i] <= max_dist}


@pytest.mark.parametrize("n", [2, 10, 50])
@pytest.mark.parametrize("f", [0.1, 0.5, 1.0, 10.0])
def test_pairs_match_naive(n, f):
    """Pair-set oracle of the reference's tests/test_ld_pair_iteration.py:21-59."""
    rng = np.random.default_rng(n * 997 + int(f * 1000))
    pos = np.unique(np.sort(rng.integers(0, 10 * n, size=n)))
    if len(pos) < 2:
        pytest.skip("collapsed")
    md = max(1, int((pos[-1] - pos[0]) * f))
    ii, jj = O.pairs_within_distance(pos, md)
    assert set(zip(ii.tolist(), jj.tolist())) == _naive_pairs(pos, md)
    assert np.all(ii < jj)


def test_pairs_edge_cases():
    assert len(O.pairs_within_distance(np.empty(0), 100)[0]) == 0
    assert len(O.pairs_within_distance(np.array([42]), 100)[0]) == 0
    assert len(O.pairs_within_distance(np.arange(10), 0)[0]) == 0
    n = 25
    ii, _ = O.pairs_within_distance(np.arange(n) * 10, 10 ** 9)
    assert len(ii) == n * (n - 1) // 2


def test_bin_semantics_right_open():
    edges = [10.0, 100.0, 1000.0]
    d = np.array([5.0, 10.0, 99.9, 100.0, 999.0, 1000.0, 2000.0])
    np.testing.assert_array_equal(O.bin_index(d, edges), [-1, 0, 0, 1, 1, 2, 2])


def test_all_pairs_ld_oracle_matches_reference(golden_dir):
    """pairwise r^2, sigma_D^2 matrix, ZnS, Omega and windowed r^2 percentiles of the
    oracle against the reference's own functions (tests/golden/ref_ldm.npz)."""
    g = np.load(os.path.join(golden_dir, "ref_ldm.npz"))
    hap, pos = g["hap"], g["pos"]
    np.testing.assert_allclose(O.pairwise_r2_matrix(hap), g["pairwise_r2"], rtol=1e-12, atol=1e-15)
    seg = O.segregating(hap)
    np.testing.assert_allclose(O.sigma_d2_matrix(hap[:, seg])[0], g["sigma_d2_seg"], rtol=1e-12, atol=1e-15)
    for md in ("include", "exclude"):
        for est in ("r2", "sigma_d2"):
            np.testing.assert_allclose(O.zns(hap, est, md), g[f"zns_{est}_{md}"], rtol=1e-12, atol=1e-15)
            np.testing.assert_allclose(O.omega(hap, est, md), g[f"omega_{est}_{md}"], rtol=1e-12, atol=1e-15)
    for k in range(2):
        pct = g[f"win{k}_pct"]
        res, cnt = O.windowed_r2(hap, pos, g[f"win{k}_bins"], pct if len(pct) > 1 else pct[0])
        np.testing.assert_array_equal(cnt, g[f"win{k}_cnt"])
        np.testing.assert_allclose(res, g[f"win{k}_res"], rtol=1e-12, equal_nan=True)


def test_all_pairs_genotype_oracle_matches_reference(golden_dir):
    """Rogers-Huff r, sigma_D^2 of genotype pairs, dosage r^2 with missing calls, and ZnS /
    Omega of a GenotypeMatrix, against the reference's own functions."""
    g = np.load(os.path.join(golden_dir, "ref_ldm.npz"))
    np.testing.assert_allclose(O.rogers_huff_r(g["geno"]), g["rogers_huff_r"], rtol=1e-12, equal_nan=True)
    np.testing.assert_allclose(O.sigma_d2_geno(g["geno"]), g["sigma_d2_geno"], rtol=1e-12, equal_nan=True)
    np.testing.assert_allclose(O.diploid_r2_matrix(g["geno_missing"]), g["diploid_r2"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(O.zns_diploid(g["geno_missing"]), g["zns_diploid"], rtol=1e-12)
    np.testing.assert_allclose(O.omega_diploid(g["geno_missing"]), g["omega_diploid"], rtol=1e-12)


@pytest.mark.parametrize("P", [1, 3, 4])
def test_reference_kernel_driver_reproduces_golden(ref_hap, P):
    """oracle.ref_kernels (pg_gpu's own estimator kernels, host-compiled in oracle/_ref,
    driven by a restatement of its dispatch) gives the statistics the reference itself
    produced (golden fixture made by running pg_gpu's Python), on the golden counts with
    missing data.  Runs where oracle/_ref has been built."""
    from oracle import ref_kernels
    if not ref_kernels.available():
        pytest.skip("oracle/_ref not built")
    g = ref_hap
    counts = [g[f"P{P}_counts{p}"] for p in range(P)]
    nvalid = [None if (g[f"P{P}_nvalid{p}"] == -1).all() else g[f"P{P}_nvalid{p}"] for p in range(P)]
    got = ref_kernels.hap_stats(counts, nvalid)
    np.testing.assert_allclose(got, g[f"P{P}_stats"], rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(got, O.hap_stats(counts, nvalid), rtol=1e-12, atol=1e-15)
