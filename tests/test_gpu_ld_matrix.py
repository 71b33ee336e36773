"""All-pairs LD (``ldk_ld_matrix`` and the functions on it) against the reference's own
outputs (tests/golden/ref_ldm.npz: pairwise_r2, sigma_D^2 matrix, ZnS, Omega, windowed
r^2 percentiles) and against the oracle on larger seeded inputs."""
import os

import numpy as np
import pytest

from oracle import ld_oracle as O
from pg_gpu_b200 import _lib, haplotype_matrix, ld_matrix, ld_statistics

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def g(golden_dir):
    return np.load(os.path.join(golden_dir, "ref_ldm.npz"))


def test_pairwise_matrices_match_reference(g):
    hm = haplotype_matrix.HaplotypeMatrix(g["hap"], g["pos"])
    np.testing.assert_allclose(hm.pairwise_r2().cpu().numpy(), g["pairwise_r2"], rtol=1e-12, atol=1e-15)
    seg = O.segregating(g["hap"])
    sd, _ = ld_matrix.ld_matrix(g["hap"][:, seg], estimator="sigma_d2")
    np.testing.assert_allclose(sd.cpu().numpy(), g["sigma_d2_seg"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("md", ["include", "exclude"])
@pytest.mark.parametrize("est", ["r2", "sigma_d2"])
def test_zns_omega_match_reference(g, md, est):
    hm = haplotype_matrix.HaplotypeMatrix(g["hap"], g["pos"])
    np.testing.assert_allclose(ld_statistics.zns(hm, md, est), g[f"zns_{est}_{md}"], rtol=1e-11)
    np.testing.assert_allclose(ld_statistics.omega(hm, md, est), g[f"omega_{est}_{md}"], rtol=1e-11)


def test_windowed_r_squared_matches_reference(g):
    hm = haplotype_matrix.HaplotypeMatrix(g["hap"], g["pos"])
    for k in range(2):
        pct = g[f"win{k}_pct"]
        res, cnt = hm.windowed_r_squared(g[f"win{k}_bins"], pct if len(pct) > 1 else pct[0])
        np.testing.assert_array_equal(cnt, g[f"win{k}_cnt"])
        np.testing.assert_allclose(res, g[f"win{k}_res"], rtol=1e-12, equal_nan=True)


@pytest.mark.parametrize("n_hap,m", [(200, 300), (37, 129), (130, 64), (9, 2)])
def test_all_estimators_match_oracle(n_hap, m):
    """Tile edges (m not a multiple of the 64-row block or the 128-partner tile), an odd
    sample count, a row subset, missing calls and monomorphic sites."""
    rng = np.random.default_rng(n_hap * 1000 + m)
    hap = (rng.random((n_hap, m)) < rng.uniform(0.02, 0.6, m)).astype(np.int8)
    hap[:, :: max(1, m // 7)] = 0
    hap[rng.random(hap.shape) < 0.04] = -1
    rows = np.sort(rng.choice(n_hap, size=max(2, n_hap - 3), replace=False))
    sub = hap[rows]
    want = {"r2": O.pairwise_r2_matrix(sub), "sigma_d2": O.sigma_d2_matrix(sub)[0],
            "r2_counts": O.r2_counts_matrix(sub)}
    for est, w in want.items():
        M, S = ld_matrix.ld_matrix(hap, rows=rows, estimator=est, reduce=True)
        got = M.cpu().numpy()
        np.testing.assert_allclose(got, w, rtol=1e-12, atol=1e-15, equal_nan=True)
        iu = np.triu_indices(m, k=1)
        up = w[iu]
        if est == "sigma_d2":
            n_joint = ((sub >= 0).astype(np.int64).T @ (sub >= 0).astype(np.int64))[iu]
            want_sum, want_cnt = up.sum(), (n_joint >= 4).sum()
        elif est == "r2_counts":
            want_sum, want_cnt = np.nansum(up), np.isfinite(up).sum()
        else:
            want_sum, want_cnt = up.sum(), len(up)
        total, count = S.tolist()
        assert count == want_cnt
        np.testing.assert_allclose(total, want_sum, rtol=1e-11, atol=1e-14)


def test_reduce_only_and_errors():
    rng = np.random.default_rng(4)
    hap = (rng.random((50, 70)) < 0.3).astype(np.int8)
    _, S = ld_matrix.ld_matrix(hap, estimator="sigma_d2", matrix=False, reduce=True)
    sd, valid = O.sigma_d2_matrix(hap)
    np.testing.assert_allclose(S.cpu().numpy(), [np.triu(sd, 1).sum(), np.triu(valid, 1).sum()], rtol=1e-11)
    lib = _lib.load()
    assert lib.ldk_ld_matrix(None, 0, 5, None, 1, 0, None, 0, None, None, 0, None) == _lib.LDK_ERR_ARG
    assert lib.ldk_ld_matrix(None, 10, 10, None, 3, 7, None, 10, None, None, 0, None) == _lib.LDK_ERR_ARG


def test_genotype_all_pairs_match_reference(g):
    from pg_gpu_b200 import genotype_matrix, ld_statistics_genotype
    gm = genotype_matrix.GenotypeMatrix(g["geno"], g["pos"])
    np.testing.assert_allclose(ld_statistics.rogers_huff_r(gm).cpu().numpy(), g["rogers_huff_r"], rtol=1e-12,
                               atol=1e-15, equal_nan=True)
    np.testing.assert_allclose(ld_statistics_genotype.sigma_d2_geno(gm).cpu().numpy(), g["sigma_d2_geno"],
                               rtol=1e-12, atol=1e-15, equal_nan=True)
    gmm = genotype_matrix.GenotypeMatrix(g["geno_missing"], g["pos"])
    np.testing.assert_allclose(ld_matrix.diploid_r2_matrix(g["geno_missing"]).cpu().numpy(), g["diploid_r2"],
                               rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(ld_statistics.zns(gmm), g["zns_diploid"], rtol=1e-11)
    np.testing.assert_allclose(ld_statistics.omega(gmm), g["omega_diploid"], rtol=1e-11)
    with pytest.raises(ValueError, match="missing"):
        ld_statistics.rogers_huff_r(gmm)


@pytest.mark.parametrize("n_ind,m", [(150, 300), (33, 129), (5, 40)])
def test_genotype_estimators_match_oracle(n_ind, m):
    rng = np.random.default_rng(n_ind * 7 + m)
    geno = (rng.random((n_ind, m)) < rng.uniform(0.05, 0.6, m)).astype(np.int8) + \
        (rng.random((n_ind, m)) < rng.uniform(0.05, 0.6, m)).astype(np.int8)
    geno[:, 3] = 1  # constant site
    iu = np.triu_indices(m, k=1)
    M, _ = ld_matrix.ld_matrix(geno, estimator="rogers_huff_r")
    np.testing.assert_allclose(M.cpu().numpy()[iu], O.rogers_huff_r(geno), rtol=1e-11, atol=1e-14, equal_nan=True)
    M, _ = ld_matrix.ld_matrix(geno, estimator="sigma_d2_geno")
    np.testing.assert_allclose(M.cpu().numpy()[iu], O.sigma_d2_geno(geno), rtol=1e-11, atol=1e-14, equal_nan=True)
    gm = geno.copy()
    gm[rng.random(gm.shape) < 0.05] = -1
    M, S = ld_matrix.ld_matrix(gm, estimator="diploid_r2", reduce=True)
    want = O.diploid_r2_matrix(gm)
    np.testing.assert_allclose(M.cpu().numpy(), want, rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(S.cpu().numpy(), [np.triu(want, 1).sum(), m * (m - 1) / 2], rtol=1e-10)
    # complete-data estimators reject missing calls through the device status
    with pytest.raises(_lib.LdkError):
        ld_matrix.ld_matrix(gm, estimator="rogers_huff_r")


def test_haplotype_rogers_huff_pairwise():
    rng = np.random.default_rng(12)
    hap = (rng.random((40, 50)) < 0.4).astype(np.int8)
    hm = haplotype_matrix.HaplotypeMatrix(hap, np.arange(50) * 10)
    r = O.rogers_huff_r(hap[0::2] + hap[1::2])
    want = np.zeros((50, 50))
    iu = np.triu_indices(50, k=1)
    want[iu] = np.nan_to_num(r ** 2)
    want = want + want.T
    np.testing.assert_allclose(hm.pairwise_r2("rogers_huff").cpu().numpy(), want, rtol=1e-11, atol=1e-14)
