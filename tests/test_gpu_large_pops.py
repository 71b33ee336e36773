"""Large populations on the tensor-core path.  The per-n_valid reciprocal table (32 B per
entry) is built in shared memory when it fits beside the pipeline; for populations of
thousands of haplotypes it lives in the workspace instead (both cases below: one population
of 6,000 -- a 192 KB table -- and three of up to 1,800 with 16 bins, where per-warp staging
takes the room).  Pair tallies must equal the plain kernel's and the oracle's exactly, bin
sums within the path's 1e-6 per bin."""
import numpy as np
import pytest

from oracle import ld_oracle as O
from pg_gpu_b200 import parse, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _region(sizes, m, seed):
    rng = np.random.default_rng(seed)
    hap, pos = synth.haplotype_region(rng, sizes, m, m * 200, 0.02)
    keep = (np.sum(hap == 0, axis=0) > 0) & (np.sum(hap == 1, axis=0) > 0)
    off = np.concatenate([[0], np.cumsum(sizes)])
    rows = [np.arange(off[p], off[p + 1]) for p in range(len(sizes))]
    return hap[:, keep].copy(), pos[keep].astype(np.float64), rows


@pytest.mark.parametrize("sizes,n_bins", [([6000], 16), ([1600, 1500, 1800], 16),
                                           ([3500, 120, 90, 100], 16), ([60, 80, 70, 90], 30)])
def test_tc_with_reciprocal_table_in_workspace(sizes, n_bins):
    """Four populations split their statistics between the two warps of a lane quarter and,
    with 105 statistics, flush through one shared staging copy: with a 3,500-haplotype
    population the table goes to the workspace; the 30-bin case keeps it in shared memory."""
    hap, pos, rows = _region(sizes, 300, seed=sum(sizes))
    edges = np.logspace(1, 5, n_bins + 1)
    kw = dict(max_dist=edges[-1])
    tc = parse.Parser(hap, pos, rows, edges, method="tc", **kw)
    got = tc.run().numpy()
    assert tc.method == "tc"
    want = parse.Parser(hap, pos, rows, edges, method="plain", **kw).run().numpy()
    np.testing.assert_array_equal(got["pairs"], want["pairs"])
    np.testing.assert_allclose(got["sums"], want["sums"], rtol=1e-6, atol=1e-300)
    ref = O.bin_sums(hap, pos, rows, edges, max_dist=edges[-1])
    np.testing.assert_array_equal(got["pairs"], ref["pairs"])
    scale = np.maximum(np.abs(ref["sums"]), 1e-300)
    assert float(np.max(np.abs(got["sums"] - ref["sums"]) / scale)) < 1e-6
