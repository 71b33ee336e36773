"""GPU parity: libldk (through its C ABI) against the float64 oracle and the reference's
golden vectors.  Tolerances: counts and pair tallies bit-exact; plain FP64 path 1e-12
relative (1e-15 absolute) per value / per bin; tensor-core path (INT8 Gram counts, FP64
estimators and bin sums) 1e-6 relative per bin."""
import ctypes
import os

import numpy as np
import pytest

from oracle import ld_oracle as O
from pg_gpu_b200 import _lib, parse, synth
from pg_gpu_b200.csrc import gen_estimators as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

PLAIN_RTOL = 1e-12
TC_RTOL = 1e-6


def rel_err(got, want, floor):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    d = np.abs(got - want)
    scale = np.maximum(np.abs(want), floor)
    return float(np.max(d / scale)) if d.size else 0.0


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.fixture(scope="module")
def ref_hap(golden_dir):
    return np.load(os.path.join(golden_dir, "ref_hap.npz"))


@pytest.fixture(scope="module")
def ref_geno(golden_dir):
    return np.load(os.path.join(golden_dir, "ref_geno.npz"))


def _stream():
    return _lib.stream_handle()


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_counts_hap_bit_exact(ref_hap, P):
    lib = _lib.load()
    g = ref_hap
    hap, offs = g[f"P{P}_hap"], g[f"P{P}_offs"]
    ii, jj = g[f"P{P}_ii"], g[f"P{P}_jj"]
    X, I, J = dev(hap, torch.int8), dev(ii, torch.int32), dev(jj, torch.int32)
    n = len(ii)
    for q in range(P):
        rows = dev(np.arange(offs[q], offs[q + 1]), torch.int32)
        counts = torch.empty((n, 4), dtype=torch.int32, device="cuda")
        nv = torch.empty(n, dtype=torch.int32, device="cuda")
        _lib.check(lib.ldk_counts_hap(_lib.ptr(X), hap.shape[1], hap.shape[1], _lib.ptr(rows), rows.numel(),
                                      _lib.ptr(I), _lib.ptr(J), n, _lib.ptr(counts), _lib.ptr(nv), _stream()))
        np.testing.assert_array_equal(counts.cpu().numpy(), g[f"P{P}_counts{q}"])
        ref_nv = g[f"P{P}_nvalid{q}"]
        if (ref_nv >= 0).all():
            np.testing.assert_array_equal(nv.cpu().numpy(), ref_nv)


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_counts_geno_bit_exact(ref_geno, P):
    lib = _lib.load()
    g = ref_geno
    geno, offs = g[f"P{P}_geno"], g[f"P{P}_offs"]
    ii, jj = g[f"P{P}_ii"], g[f"P{P}_jj"]
    X, I, J = dev(geno, torch.int8), dev(ii, torch.int32), dev(jj, torch.int32)
    n = len(ii)
    for q in range(P):
        rows = dev(np.arange(offs[q], offs[q + 1]), torch.int32)
        counts = torch.empty((n, 9), dtype=torch.int32, device="cuda")
        nv = torch.empty(n, dtype=torch.int32, device="cuda")
        _lib.check(lib.ldk_counts_geno(_lib.ptr(X), geno.shape[1], geno.shape[1], _lib.ptr(rows), rows.numel(),
                                       _lib.ptr(I), _lib.ptr(J), n, _lib.ptr(counts), _lib.ptr(nv), _stream()))
        np.testing.assert_array_equal(counts.cpu().numpy(), g[f"P{P}_counts{q}"])


def _stats(genotypes, counts_list, nvalid_list):
    lib = _lib.load()
    P = len(counts_list)
    n = counts_list[0].shape[0]
    C = dev(np.stack(counts_list), torch.int32)
    NV = None
    if any(v is not None for v in nvalid_list):
        NV = dev(np.stack([v if v is not None else c.sum(axis=1) for v, c in zip(nvalid_list, counts_list)]),
                 torch.int32)
    out = torch.empty((n, parse.n_stats(P)), dtype=torch.float64, device="cuda")
    _lib.check(lib.ldk_stats(int(genotypes), P, _lib.ptr(C), _lib.ptr(NV), n, _lib.ptr(out), _stream()))
    return out.cpu().numpy()


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_stats_hap_golden(ref_hap, P):
    g = ref_hap
    cl = [g[f"P{P}_counts{q}"] for q in range(P)]
    nl = [None if (g[f"P{P}_nvalid{q}"] < 0).all() else g[f"P{P}_nvalid{q}"] for q in range(P)]
    got = _stats(False, cl, nl)
    assert rel_err(got, g[f"P{P}_stats"], 1e-3) < PLAIN_RTOL
    if P == 2:
        assert rel_err(got, g["P2_twopop_stats"], 1e-3) < PLAIN_RTOL


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_stats_geno_golden(ref_geno, P):
    g = ref_geno
    cl = [g[f"P{P}_counts{q}"] for q in range(P)]
    nl = [None if (g[f"P{P}_nvalid{q}"] < 0).all() else g[f"P{P}_nvalid{q}"] for q in range(P)]
    got = _stats(True, cl, nl)
    ref = g[f"P{P}_stats"]
    assert np.array_equal(np.isfinite(got), np.isfinite(ref))
    f = np.isfinite(ref)
    assert rel_err(got[f], ref[f], 1e-3) < PLAIN_RTOL


def test_raw_calls_every_case():
    """ldk_raw_hap for every canonical case against the oracle's raw call."""
    lib = _lib.load()
    rng = np.random.default_rng(7)
    P = 4
    n = 500
    counts = [rng.multinomial(rng.integers(3, 60), [0.3, 0.2, 0.2, 0.3], size=n) for _ in range(P)]
    for c in counts:
        c[:5] = [[0, 0, 0, 3], [1, 0, 0, 0], [0, 0, 0, 0], [2, 0, 0, 2], [0, 1, 1, 0]]
    pops = [O.HapPop(c) for c in counts]
    C = dev(np.concatenate(counts, axis=1).astype(np.float64), torch.float64)
    examples = {"dd1": ("dd", (1, 1)), "dd2": ("dd", (0, 2)), "dz_iii": ("dz", (2, 2, 2)),
                "dz_iij": ("dz", (1, 1, 3)), "dz_iji": ("dz", (0, 2, 0)), "dz_ijj": ("dz", (3, 1, 1)),
                "dz_ijk": ("dz", (0, 1, 2)), "pi2_same": ("pi2", (3, 3, 3, 3)),
                "pi2_iikk": ("pi2", (0, 0, 2, 2)), "pi2_iikl": ("pi2", (1, 1, 0, 3)),
                "pi2_ijkk": ("pi2", (0, 2, 3, 3)), "pi2_alldiff": ("pi2", (0, 1, 2, 3)),
                "pi2_triple": ("pi2", (2, 1, 2, 2)), "pi2_ijij": ("pi2", (1, 3, 1, 3)),
                "pi2_shared": ("pi2", (0, 1, 0, 2))}
    for cid, case in enumerate(G.RAW_CASES):
        kind, q = examples[case]
        ccase, args = G.canonical(kind, q)
        assert ccase == case
        a = (ctypes.c_int32 * 4)(*(list(args) + [0] * (4 - len(args))))
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        _lib.check(lib.ldk_raw_hap(cid, a, P, _lib.ptr(C), None, n, _lib.ptr(out), _stream()))
        want = O.hap_raw(kind, q, pops)
        assert rel_err(out.cpu().numpy(), want, 1e-3) < PLAIN_RTOL, case


def test_r_family_golden(ref_hap):
    lib = _lib.load()
    g = ref_hap
    hap, offs, ii, jj = g["P1_hap"], g["P1_offs"], g["P1_ii"], g["P1_jj"]
    c, nv = O.hap_counts(hap, ii, jj, list(range(offs[0], offs[1])))
    C = dev(c.astype(np.float64), torch.float64)
    for which, key in ((0, "P1_r"), (1, "P1_r2"), (2, "P1_dprime")):
        out = torch.empty(len(c), dtype=torch.float64, device="cuda")
        _lib.check(lib.ldk_r_family(which, _lib.ptr(C), None, len(c), _lib.ptr(out), _stream()))
        np.testing.assert_allclose(out.cpu().numpy(), g[key], rtol=1e-12, atol=1e-15, equal_nan=True)
    e = g["edge_counts"]
    out = torch.empty(len(e), dtype=torch.float64, device="cuda")
    _lib.check(lib.ldk_r_family(1, _lib.ptr(dev(e, torch.float64)), None, len(e), _lib.ptr(out), _stream()))
    np.testing.assert_allclose(out.cpu().numpy(), g["edge_r2"], rtol=1e-12, equal_nan=True)


# ---------------------------------------------------------------------------
# the binned parse
# ---------------------------------------------------------------------------

SCALES = {1: 0.1, 2: 0.004, 3: 0.003, 4: 0.004, 5: 0.0015}


@pytest.fixture(scope="module")
def workloads():
    return {k: synth.make_config(k, scale=s) for k, s in SCALES.items()}


@pytest.fixture(scope="module")
def oracle_results(workloads):
    out = {}
    for k, w in workloads.items():
        out[k] = O.bin_sums(w.data, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes,
                            max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                            n_blocks=w.n_blocks)
    return out


def run_parse(w, method):
    r = parse.ld_parse(w.data, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes, method=method,
                       max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                       n_blocks=w.n_blocks)
    return r.numpy()


def check_parse(got, want, rtol):
    np.testing.assert_array_equal(got["pairs"], want["pairs"])
    np.testing.assert_array_equal(got["r2_counts"], want["r2_count"])
    assert want["pairs"].sum() > 0
    # per-bin relative error against the FP64 oracle, scaled by the bin's magnitude
    floor = 1e-300
    assert rel_err(got["sums"], want["sums"], floor) < rtol
    assert rel_err(got["r2_sums"], want["r2_sum"], floor) < rtol


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_parse_plain_matches_oracle(workloads, oracle_results, k):
    check_parse(run_parse(workloads[k], "plain"), oracle_results[k], PLAIN_RTOL)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_parse_tc_matches_oracle(workloads, oracle_results, k):
    check_parse(run_parse(workloads[k], "tc"), oracle_results[k], TC_RTOL)


def test_im_example_against_moments(golden_dir):
    im = np.load(os.path.join(golden_dir, "im_example.npz"))
    hap, pos = im["hap"], im["pos"].astype(np.float64)
    keep = O.biallelic_keep(hap)
    hap, pos = hap[:, keep], pos[keep]
    rows = [im["rows0"], im["rows1"]]
    for method, tol in (("plain", 1e-10), ("tc", TC_RTOL)):
        r = parse.ld_parse(hap, pos, rows, im["edges"], method=method).numpy()
        assert rel_err(r["sums"][0], im["ld_sums"], 1e-300) < tol, method


def test_parse_edge_cases():
    rng = np.random.default_rng(3)
    hap = rng.integers(0, 2, size=(12, 40)).astype(np.int8)
    pos = np.arange(40, dtype=np.float64) * 10.0
    rows = [np.arange(12)]
    for method in ("plain", "tc"):
        # max_dist 0 with unique positions: no pairs
        r = parse.ld_parse(hap, pos, rows, [0.0, 5.0], method=method, max_dist=0.0).numpy()
        assert r["pairs"].sum() == 0 and np.all(r["sums"] == 0)
        # a single SNP: nothing to do
        r = parse.ld_parse(hap[:, :1], pos[:1], rows, [0.0, 5.0], method=method).numpy()
        assert r["pairs"].sum() == 0
        # distance exactly on the last edge is generated but dropped; below the first edge dropped
        r = parse.ld_parse(hap, pos, rows, [15.0, 30.0], method=method).numpy()
        want = O.bin_sums(hap, pos, rows, [15.0, 30.0])
        np.testing.assert_array_equal(r["pairs"], want["pairs"])
        assert want["n_pairs"] > want["pairs"].sum()
        # empty and one-SNP windows
        wo = np.array([0, 0, 1, 17, 17, 40])
        r = parse.ld_parse(hap, pos, rows, [0.0, 100.0, 1000.0], method=method, window_offsets=wo).numpy()
        want = O.bin_sums(hap, pos, rows, [0.0, 100.0, 1000.0], window_offsets=wo)
        np.testing.assert_array_equal(r["pairs"], want["pairs"])
        assert rel_err(r["sums"], want["sums"], 1e-300) < (PLAIN_RTOL if method == "plain" else TC_RTOL)


@pytest.mark.parametrize("genotypes", [False, True])
def test_work_items_dense_cluster_and_isolated_snps(genotypes):
    """Work items on a mixed layout: a dense cluster whose row blocks have many partner tiles
    (each cut into several items), then SNPs spaced beyond the cutoff (row blocks without
    partners get no item), then a second cluster; pairs bit-exact and sums within tolerance
    of the oracle."""
    rng = np.random.default_rng(21)
    n1, n2, n3 = 1300, 700, 500
    pos = np.concatenate([np.sort(rng.choice(50_000, n1, replace=False)).astype(np.float64),
                          1e6 + np.arange(n2) * 70_000.0,
                          6e7 + np.sort(rng.choice(40_000, n3, replace=False)).astype(np.float64)])
    m = len(pos)
    if genotypes:
        data, rows = _genotypes(rng, 90, m, 0.02), [np.arange(90)]
    else:
        data = (rng.random((120, m)) < rng.uniform(0.05, 0.5, m)).astype(np.int8)
        data[rng.random(data.shape) < 0.03] = -1
        rows = [np.arange(120)]
    edges = [0.0, 100.0, 1_000.0, 10_000.0, 60_000.0]
    got = parse.ld_parse(data, pos, rows, edges, genotypes=genotypes, method="tc", max_dist=60_000.0).numpy()
    want = O.bin_sums(data, pos, rows, edges, genotypes=genotypes, max_dist=60_000.0)
    check_parse(got, want, TC_RTOL)


def test_work_items_many_row_blocks():
    """More row blocks than the work-item split handles in one round of its block scan
    (1,132 > 1,024): 1,100 windows of 64 SNPs (one tile each) and, at a random place in the
    window order, one window of 2,000 SNPs whose row blocks are cut into several items."""
    rng = np.random.default_rng(23)
    sizes = [64] * 1100 + [2000]
    sizes = [sizes[k] for k in rng.permutation(len(sizes))]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    pos = np.concatenate([2e6 * k + np.sort(rng.choice(10**6, s, replace=False)).astype(np.float64)
                          for k, s in enumerate(sizes)])
    m = len(pos)
    data = (rng.random((80, m)) < rng.uniform(0.05, 0.5, m)).astype(np.int8)
    data[rng.random(data.shape) < 0.03] = -1
    rows, edges = [np.arange(80)], [0.0, 1e3, 1e4, 1e5, 1e6]
    got = parse.ld_parse(data, pos, rows, edges, method="tc", window_offsets=offs).numpy()
    want = O.bin_sums(data, pos, rows, edges, window_offsets=offs)
    check_parse(got, want, TC_RTOL)


def _genotypes(rng, n_ind, n_var, missing):
    """Genotypes as sums of two correlated haplotypes (a few founders), with missing calls."""
    founders = (rng.random((6, n_var)) < rng.uniform(0.05, 0.6, n_var)).astype(np.int8)
    h = founders[rng.integers(0, 6, size=(2 * n_ind,))]
    flip = rng.random(h.shape) < 0.05
    h = np.where(flip, 1 - h, h).astype(np.int8)
    g = (h[0::2] + h[1::2]).astype(np.int8)
    g[rng.random(g.shape) < missing] = -1
    return g


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_parse_tc_genotypes_windows_blocks(P):
    """Genotype path on tensor cores: 128-SNP row blocks, several populations of unequal
    size, windows of 0, 1, 3 and many SNPs, bootstrap blocks up to four per row block."""
    rng = np.random.default_rng(100 + P)
    sizes = [17, 40, 9, 33][:P]
    n_var = 700
    g = _genotypes(rng, sum(sizes), n_var, 0.03)
    pos = np.cumsum(rng.integers(1, 40, size=n_var)).astype(np.float64)
    offs = np.cumsum([0] + sizes)
    rows = [np.arange(offs[p], offs[p + 1]) for p in range(P)]
    wo = np.array([0, 0, 1, 4, 300, n_var])
    blocks = np.minimum(pos // 1500, 1e9).astype(np.int32)
    nblk = int(blocks.max()) + 1
    edges = np.array([0.0, 50.0, 200.0, 800.0, 3000.0])
    want = O.bin_sums(g, pos, rows, edges, genotypes=True, max_dist=2500.0, window_offsets=wo,
                      snp_block=blocks, n_blocks=nblk)
    assert want["pairs"].sum() > 0
    for method, tol in (("plain", PLAIN_RTOL), ("tc", TC_RTOL)):
        r = parse.ld_parse(g, pos, rows, edges, genotypes=True, method=method, max_dist=2500.0,
                           window_offsets=wo, snp_block=blocks, n_blocks=nblk).numpy()
        check_parse(r, want, tol)


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_parse_tc_haplotypes_windows_blocks(P):
    """Haplotype path on tensor cores for one to four populations of unequal size (four
    only appear here: the benchmark configurations have at most three), 64-SNP row blocks,
    windows of 0, 1, 3 and many SNPs, bootstrap blocks, missing calls."""
    rng = np.random.default_rng(200 + P)
    sizes = [23, 61, 14, 40][:P]
    n_var = 900
    hap, _ = synth.haplotype_region(rng, sizes, n_var, n_var * 30, 0.04)
    pos = np.cumsum(rng.integers(1, 40, size=n_var)).astype(np.float64)
    offs = np.cumsum([0] + sizes)
    rows = [np.arange(offs[p], offs[p + 1]) for p in range(P)]
    wo = np.array([0, 0, 1, 4, 500, n_var])
    # bootstrap blocks of ~150 SNPs: a 64-SNP row block of the haplotype path may span two
    blocks = (pos // 3000).astype(np.int32)
    nblk = int(blocks.max()) + 1
    edges = np.array([0.0, 40.0, 150.0, 600.0, 2500.0])
    want = O.bin_sums(hap, pos, rows, edges, max_dist=2000.0, window_offsets=wo, snp_block=blocks,
                      n_blocks=nblk)
    assert want["pairs"].sum() > 0
    # plain: 1e-11 here -- 105 four-population statistics of a 14-haplotype population
    # round a little further from the oracle's (2e-12 seen) than the 1e-12 used elsewhere
    for method, tol in (("plain", 10 * PLAIN_RTOL), ("tc", TC_RTOL)):
        r = parse.ld_parse(hap, pos, rows, edges, method=method, max_dist=2000.0, window_offsets=wo,
                           snp_block=blocks, n_blocks=nblk).numpy()
        check_parse(r, want, tol)


def test_parse_tc_genotype_edge_cases():
    rng = np.random.default_rng(7)
    g = _genotypes(rng, 25, 300, 0.0)
    g[:, 5] = 0          # monomorphic site: r^2 undefined, statistics still counted
    g[:, 6] = -1         # a site missing everywhere: n_valid 0
    pos = np.arange(300, dtype=np.float64) * 7.0
    rows = [np.arange(25)]
    for edges, md in (([0.0, 5.0], 0.0), ([14.0, 70.0, 700.0], None), ([0.0, 10.0, 2100.0], None)):
        want = O.bin_sums(g, pos, rows, edges, genotypes=True, max_dist=md)
        r = parse.ld_parse(g, pos, rows, edges, genotypes=True, method="tc", max_dist=md).numpy()
        np.testing.assert_array_equal(r["pairs"], want["pairs"])
        np.testing.assert_array_equal(r["r2_counts"], want["r2_count"])
        assert rel_err(r["sums"], want["sums"], 1e-300) < TC_RTOL


def test_parse_reports_errors():
    hap = np.zeros((4, 10), np.int8)
    hap[0] = 1
    pos = np.arange(10, dtype=np.float64)
    with pytest.raises(_lib.LdkError, match="unsorted"):
        parse.ld_parse(hap, pos[::-1].copy(), [np.arange(4)], [0.0, 5.0], method="plain")
    with pytest.raises(_lib.LdkError, match="snp_block"):
        parse.ld_parse(hap, pos, [np.arange(4)], [0.0, 5.0], method="plain",
                       snp_block=np.full(10, 3, np.int32), n_blocks=2)
    with pytest.raises(_lib.LdkError, match="edges"):
        parse.ld_parse(hap, pos, [np.arange(4)], [5.0, 1.0], method="plain")


@pytest.mark.parametrize("n_rep,n_blocks,nb,ns", [(7, 30, 4, 15), (100, 1203, 16, 46), (200, 1203, 16, 46)])
def test_block_combine_bootstrap(n_rep, n_blocks, nb, ns):
    """Replicate sums from per-block sums: multinomial-like weights (many zeros), replicate
    counts that do not fill the kernel's groups of eight, and one-hot window weights (the
    per-window totals, n_rep = 200)."""
    rng = np.random.default_rng(11 + n_rep)
    bs = rng.normal(size=(n_blocks, nb, ns))
    if n_rep == 200:
        w = np.zeros((n_rep, n_blocks), np.int32)
        w[rng.integers(0, n_rep, size=n_blocks), np.arange(n_blocks)] = 1
    else:
        w = rng.integers(0, 3, size=(n_rep, n_blocks)).astype(np.int32)
    got = parse.block_combine(dev(bs, torch.float64), w).cpu().numpy()
    np.testing.assert_allclose(got, np.tensordot(w, bs, axes=(1, 0)), rtol=1e-12, atol=1e-12)


def test_probe_peaks_plausible():
    """The roofline denominators measured on this device: INT8 tensor ops/s between
    1 and 10 POP/s (B200 nominal dense 4.5) and FP64 FMA/s between 5 and 30 T/s
    (nominal 18.5 T FMA/s); a second call agrees with the first within 20%."""
    i8, f64 = _lib.probe_peaks()
    assert 1e15 < i8 < 1e16, i8
    assert 5e12 < f64 < 3e13, f64
    i8b, f64b = _lib.probe_peaks()
    assert abs(i8b - i8) < 0.2 * i8 and abs(f64b - f64) < 0.2 * f64


@pytest.mark.parametrize("method", ["tc", "plain"])
def test_parse_graph_replay_matches_run(method):
    """Setup once, capture the enqueue in a CUDA graph, replay: the same bits as ldk_parse;
    after the input matrix changes in place, a replay gives the same bits as a fresh parse
    of the new data.  The bin sums are order-independent (fixed-point integer
    accumulation), so runs, replays and separate parsers agree exactly although their row
    blocks finish in different orders."""
    w = synth.make_config(4, scale=0.003)
    p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method=method, max_dist=w.max_dist,
                     window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks)
    want = {k: v.copy() for k, v in p.run().numpy().items()}
    g, reps = p.graph(after=lambda out: parse.block_combine(out.sums, torch.ones((1, w.n_blocks), dtype=torch.int32,
                                                                                   device="cuda")))
    for _ in range(2):
        g.replay()
        p.status()
        got = p.out.numpy()
        for k in ("pairs", "r2_counts", "sums", "r2_sums"):
            np.testing.assert_array_equal(got[k], want[k])
        np.testing.assert_allclose(reps.cpu().numpy()[0], want["sums"].sum(axis=0), rtol=1e-11, atol=1e-12)
    data2 = w.data.copy()
    perm = np.random.default_rng(9).permutation(data2.shape[0])
    data2[:, ::7] = data2[perm][:, ::7]  # re-pairs the haplotypes at every 7th SNP: new LD
    p.X.copy_(torch.as_tensor(data2, device="cuda"))
    g.replay()
    p.status()
    ref = parse.ld_parse(data2, w.positions, w.pop_rows, w.edges, method=method, max_dist=w.max_dist,
                         window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks).numpy()
    got = p.out.numpy()
    for k in ("pairs", "r2_counts", "sums", "r2_sums"):
        np.testing.assert_array_equal(got[k], ref[k])
    assert rel_err(got["sums"], want["sums"], 1e-300) > 1e-6  # the replay saw the new data


@pytest.mark.parametrize("cfg,stretch", [(1, 3.0), (3, 20.0)])
def test_graph_replay_after_positions_change(cfg, stretch):
    """The tensor-core work items (runs of a row block's partner tiles) are split on the
    device from each run's own pair ranges.  Captured once, then replayed after the SNP
    positions are stretched in place (SNPs lose the partners that move beyond the cutoff,
    so the split differs from the captured run's), a replay counts every pair once:
    bit-equal to a fresh parse of the new positions and within the tolerance of the oracle
    (haplotypes and genotypes)."""
    w = synth.make_config(cfg, scale={1: 0.3, 3: 0.01}[cfg])
    kw = dict(genotypes=w.genotypes, method="tc", max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)
    p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
    before = {k: v.copy() for k, v in p.run().numpy().items()}
    g, _ = p.graph()
    pos2 = w.positions[0] + (w.positions - w.positions[0]) * stretch
    p.pos.copy_(torch.as_tensor(pos2, device="cuda"))
    g.replay()
    p.status()
    got = p.out.numpy()
    fresh = parse.ld_parse(w.data, pos2, w.pop_rows, w.edges, **kw).numpy()
    for k in ("pairs", "r2_counts", "sums", "r2_sums"):
        np.testing.assert_array_equal(got[k], fresh[k])
    want = O.bin_sums(w.data, pos2, w.pop_rows, w.edges, max_dist=w.max_dist, window_offsets=w.window_offsets,
                      snp_block=w.snp_block, n_blocks=w.n_blocks, genotypes=bool(w.genotypes))
    check_parse(got, want, TC_RTOL)
    assert got["pairs"].sum() != before["pairs"].sum()


@pytest.mark.parametrize("genotypes", [False, True])
def test_autotune_picks_a_candidate_and_keeps_results(genotypes):
    """With tuning on, the first parse of a shape times the tile candidates and keeps one;
    its results and those of later calls (tuned width) match the default-width parse, and
    the first call's own parse (after the candidates) does the full work again."""
    w = synth.make_config(3 if genotypes else 2, scale=0.1)
    kw = dict(genotypes=w.genotypes, method="tc", max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)
    ref = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
    want = {k: v.copy() for k, v in ref.run().numpy().items()}
    try:
        _lib.autotune(True)
        p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
        lib = _lib.load()
        lib.ldk_profile(1)
        kernel_ms = []
        for _ in range(2):
            got = p.run().numpy()
            kernel_ms.append(lib.ldk_profile_last_kernel_ms())
            np.testing.assert_array_equal(got["pairs"], want["pairs"])
            assert rel_err(got["sums"], want["sums"], 1e-300) < 1e-11
        assert p.tile_width() in ({12, 24} if genotypes else {48, 24})
        # a parse launched on the candidates' spent row-block counter would finish at once
        assert kernel_ms[0] > 0.3 * kernel_ms[1], kernel_ms
    finally:
        _lib.load().ldk_profile(0)
        _lib.autotune(False)


@pytest.mark.parametrize("cfg,method", [(4, "tc"), (4, "plain"), (3, "tc"), (5, "tc"), (2, "tc"), (1, "tc")])
def test_parse_is_bit_reproducible(cfg, method):
    """Repeated parses of one input give identical bits in every output, on the haplotype
    and genotype paths and both kernels, although CTAs claim row blocks (warps claim row
    chunks) dynamically and finish in a different order each run; ldk_parse_reproducible
    says so for these shapes."""
    w = synth.make_config(cfg, scale={1: 0.5, 2: 0.01, 3: 0.02, 4: 0.003, 5: 0.002}[cfg])
    kw = dict(genotypes=w.genotypes, method=method, max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)
    p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
    assert p.reproducible()
    first = {k: v.copy() for k, v in p.run().numpy().items()}
    assert first["pairs"].sum() > 0
    for _ in range(3):
        again = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw).run().numpy()
        for k in ("pairs", "r2_counts", "sums", "r2_sums"):
            np.testing.assert_array_equal(again[k], first[k])
