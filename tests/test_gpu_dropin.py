"""The pg_gpu call surface on the GPU: moments_ld.compute_ld_statistics,
HaplotypeMatrix.compute_ld_statistics_gpu_*, ld_pipeline and ld_statistics, checked
against moments' golden output, the reference's own function outputs and the oracle
(the same checks as pg_gpu's tests/test_ld_validation_full.py, test_moments_ld.py,
test_ld_pair_iteration.py, test_two_pop_stats.py, test_haplotype_kernels_rsq.py)."""
import os

import numpy as np
import pytest

from oracle import ld_oracle as O
from pg_gpu_b200 import genotype_matrix, haplotype_matrix, ld_pipeline, ld_statistics, moments_ld, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


@pytest.fixture(scope="module")
def im(golden_dir):
    d = np.load(os.path.join(golden_dir, "im_example.npz"))
    hm = haplotype_matrix.HaplotypeMatrix(d["hap"], d["pos"],
                                          sample_sets={"deme0": list(d["rows0"]), "deme1": list(d["rows1"])})
    return d, hm


@pytest.mark.parametrize("method,tol", [("tc", 1e-6), ("plain", 1e-10)])
def test_moments_ld_compute_ld_statistics_matches_moments(im, method, tol):
    d, hm = im
    out = moments_ld.compute_ld_statistics(haplotype_matrix=hm.apply_biallelic_filter(), pops=["deme0", "deme1"],
                                           bp_bins=d["edges"], report=False, method=method)
    assert out["stats"][0] == list(d["ld_names"]) and out["stats"][1] == list(d["het_names"])
    assert out["bins"] == [(float(a), float(b)) for a, b in zip(d["edges"][:-1], d["edges"][1:])]
    assert rel(np.array(out["sums"][:-1]), d["ld_sums"]) < tol
    np.testing.assert_allclose(out["sums"][-1], d["het_sums"], rtol=1e-12)


def test_two_pops_method_matches_moments_cache(im):
    """pg_gpu tests/test_ld_validation_full.py with raw=True, at 1e-6 instead of 1e-2."""
    d, hm = im
    res = hm.compute_ld_statistics_gpu_two_pops(d["edges"], "deme0", "deme1", raw=True)
    for b, key in enumerate(res):
        got = np.array(list(res[key].values()))
        assert list(res[key].keys()) == list(d["ld_names"])
        assert rel(got, d["ld_sums"][b]) < 1e-6


def test_single_pop_means(im):
    d, hm = im
    f = hm.apply_biallelic_filter()
    res = f.compute_ld_statistics_gpu_single_pop(d["edges"], raw=False)
    want = O.bin_sums(np.asarray(f.haplotypes), np.asarray(f.positions, np.float64),
                      [np.arange(f.num_haplotypes)], d["edges"])
    for b, key in enumerate(res):
        assert rel(res[key], want["sums"][0, b] / want["pairs"][0, b]) < 1e-6


def _collect(pos, max_dist, chunk):
    ii, jj = [], []
    for ci, cj in ld_pipeline.iter_pairs_within_distance(pos, max_dist, chunk):
        ii.append(ci.cpu().numpy())
        jj.append(cj.cpu().numpy())
    if not ii:
        return np.empty(0, np.int32), np.empty(0, np.int32)
    return np.concatenate(ii), np.concatenate(jj)


@pytest.mark.parametrize("n", [2, 10, 50])
@pytest.mark.parametrize("f", [0.1, 0.5, 1.0, 10.0])
def test_iter_pairs_matches_naive(n, f):
    """pg_gpu tests/test_ld_pair_iteration.py:32-59."""
    rng = np.random.default_rng(n * 997 + int(f * 1000))
    pos = np.unique(np.sort(rng.integers(0, 10 * n, size=n)))
    if len(pos) < 2:
        pytest.skip("collapsed")
    md = max(1, int((pos[-1] - pos[0]) * f))
    ii, jj = _collect(pos, md, 7)
    naive = {(i, j) for i in range(len(pos)) for j in range(i + 1, len(pos)) if pos[j] - pos[i] <= md}
    assert set(zip(ii.tolist(), jj.tolist())) == naive


def test_iter_pairs_chunk_independence_and_edges():
    rng = np.random.default_rng(12345)
    pos = np.unique(np.sort(rng.integers(0, 100_000, size=500)))
    ref = _collect(pos, 5000, 1)
    for cs in (100, 10_000, 1_000_000):
        got = _collect(pos, 5000, cs)
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
    assert list(ld_pipeline.iter_pairs_within_distance(np.empty(0), 100, 10)) == []
    assert list(ld_pipeline.iter_pairs_within_distance(np.array([42]), 100, 10)) == []
    assert _collect(np.arange(10), 0, 4)[0].size == 0
    assert _collect(np.arange(25) * 10, 10 ** 9, 7)[0].size == 25 * 24 // 2


def test_counts_and_batch_statistics(golden_dir):
    g = np.load(os.path.join(golden_dir, "ref_hap.npz"))
    hap, offs, ii, jj = g["P2_hap"], g["P2_offs"], g["P2_ii"], g["P2_jj"]
    cl, nl = [], []
    for q in range(2):
        c, nv = ld_pipeline.compute_counts_for_pairs(hap, ii, jj, list(range(offs[q], offs[q + 1])))
        np.testing.assert_array_equal(c.cpu().numpy(), g[f"P2_counts{q}"])
        assert (nv is None) == bool((g[f"P2_nvalid{q}"] < 0).all())
        cl.append(c)
        nl.append(nv)
    st = ld_pipeline.compute_two_pop_statistics_batch(cl[0], cl[1], nl[0], nl[1]).cpu().numpy()
    assert rel(st, g["P2_twopop_stats"], 1e-3) < 1e-12
    for P in (1, 3, 4):
        cs = [g[f"P{P}_counts{q}"] for q in range(P)]
        nvs = [None if (g[f"P{P}_nvalid{q}"] < 0).all() else g[f"P{P}_nvalid{q}"] for q in range(P)]
        got = ld_pipeline.compute_multi_pop_statistics_batch_hap(cs, nvs, None,
                                                                 ld_pipeline.generate_stat_specs(P)).cpu().numpy()
        assert rel(got, g[f"P{P}_stats"], 1e-3) < 1e-12


def test_ld_statistics_api_reproduces_two_pop_batch(golden_dir):
    """The 15 statistics assembled from ld_statistics.dd/dz/pi2 exactly as
    compute_two_pop_statistics_batch does (ld_pipeline.py:293-322)."""
    g = np.load(os.path.join(golden_dir, "ref_hap.npz"))
    c1, c2 = g["P2_counts0"].astype(np.float64), g["P2_counts1"].astype(np.float64)
    n1 = None if (g["P2_nvalid0"] < 0).all() else g["P2_nvalid0"].astype(np.float64)
    n2 = None if (g["P2_nvalid1"] < 0).all() else g["P2_nvalid1"].astype(np.float64)
    cb = np.concatenate([c1, c2], axis=1)
    nb = (n1 if n1 is not None else c1.sum(1), n2 if n2 is not None else c2.sum(1))
    L = ld_statistics
    cols = [L.dd(c1, n_valid=n1), L.dd(cb, (0, 1), nb), L.dd(c2, n_valid=n2),
            L.dz(c1, n_valid=n1), 0.5 * (L.dz(cb, (0, 0, 1), nb) + L.dz(cb, (0, 1, 0), nb)),
            L.dz(cb, (0, 1, 1), nb), L.dz(cb, (1, 0, 0), nb),
            0.5 * (L.dz(cb, (1, 0, 1), nb) + L.dz(cb, (1, 1, 0), nb)), L.dz(c2, n_valid=n2),
            L.pi2(c1, n_valid=n1), L.pi2(cb, (0, 0, 0, 1), nb), L.pi2(cb, (0, 0, 1, 1), nb),
            L.pi2(cb, (0, 1, 0, 1), nb), L.pi2(cb, (0, 1, 1, 1), nb), L.pi2(c2, n_valid=n2)]
    got = torch.stack(cols, 1).cpu().numpy()
    assert rel(got, g["P2_twopop_stats"], 1e-3) < 1e-12


def test_r_squared_known_answers():
    """pg_gpu tests/test_haplotype_kernels_rsq.py:92-126."""
    e = np.array([[0, 0, 50, 50], [50, 0, 0, 50], [0, 50, 50, 0]], np.float64)
    assert np.isnan(ld_statistics.r_squared(e[:1]).cpu().numpy()).all()
    np.testing.assert_allclose(ld_statistics.r(e[1:]).cpu().numpy(), [1.0, -1.0], atol=1e-12)
    np.testing.assert_allclose(ld_statistics.r_squared(e[1:]).cpu().numpy(), [1.0, 1.0], atol=1e-12)
    np.testing.assert_allclose(ld_statistics.d_prime(e[1:]).cpu().numpy(), [1.0, -1.0], atol=1e-12)


def test_genotype_path_matches_oracle():
    w = synth.make_config(3, scale=0.002)
    gm = genotype_matrix.GenotypeMatrix(w.data, w.positions.astype(np.int64), sample_sets={"p": list(w.pop_rows[0])})
    out = moments_ld.compute_ld_statistics(genotype_matrix=gm, pops=["p"], bp_bins=w.edges, use_genotypes=True,
                                           report=False)
    keep = O.geno_biallelic_keep(w.data, w.pop_rows[0])
    want = O.bin_sums(w.data[:, keep], w.positions[keep], w.pop_rows, w.edges, genotypes=True)
    assert rel(np.array(out["sums"][:-1]), want["sums"][0]) < 1e-12
    H = O.heterozygosity(w.data, w.pop_rows, genotypes=True)
    np.testing.assert_allclose(out["sums"][-1], [H["H_0_0"]], rtol=1e-12)


def test_genetic_map_bins_match_oracle(tmp_path):
    w = synth.make_config(2, scale=0.004)
    m = tmp_path / "map.txt"
    span = float(w.positions[-1])
    m.write_text(f"pos\tcM\n0\t0.0\n{span / 2}\t0.4\n{span + 1}\t1.5\n")
    hm = haplotype_matrix.HaplotypeMatrix(w.data, w.positions.astype(np.int64),
                                          sample_sets={"a": list(w.pop_rows[0]), "b": list(w.pop_rows[1])})
    r_bins = np.array([0.0, 1e-4, 1e-3, 3e-3])
    out = moments_ld.compute_ld_statistics(haplotype_matrix=hm, rec_map_file=str(m), pops=["a", "b"],
                                           r_bins=r_bins, report=False)
    gen = moments_ld._interpolate_genetic_distances(w.positions, str(m))
    max_bp = moments_ld._max_bp_for_r_dist(w.positions, gen, r_bins[-1])
    want = O.bin_sums(w.data, w.positions, w.pop_rows, r_bins, max_dist=max_bp, coords=gen)
    assert want["pairs"].sum() > 0
    assert rel(np.array(out["sums"][:-1]), want["sums"][0]) < 1e-6
