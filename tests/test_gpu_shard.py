"""A parse split into anchor ranges, each rank's slab (its anchors plus the right halo of
max_dist) parsed on its own through the library with ``anchor_end``, and the outputs summed
-- what the ranks of a multi-GPU run do, here one after another on one GPU (the rank parses
never wait on one another).  Against one parse of the whole input: pair tallies
bit-exact, sums to 1e-12 on the tensor-core path (a rank's row blocks are the whole
parse's; only the final sum of the rank outputs adds FP64 totals in another grouping) and
1e-11 on the plain path (a rank's 8-SNP row chunks start after the halos of its earlier
window segments, so its FP64 partial sums group pairs differently; cancelling bins)."""
import numpy as np
import pytest

from pg_gpu_b200 import _lib, parse, shard, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _split_parse(w, world, method):
    wo = [0, w.n_var] if w.window_offsets is None else list(w.window_offsets)
    rows, _ = _lib.tc_row_blocks(w.genotypes)
    total, slabs = None, []
    for seg in shard.split_anchors(w.positions, wo, w.max_dist, world, align=rows):
        if not seg:
            continue
        snps, offs, ends = shard.slab_of(seg)
        slabs.append(len(snps))
        r = parse.Parser(w.data[:, snps], w.positions[snps], w.pop_rows, w.edges, genotypes=w.genotypes,
                         method=method, max_dist=w.max_dist, window_offsets=offs, anchor_end=ends,
                         snp_block=None if w.snp_block is None else w.snp_block[snps],
                         n_blocks=w.n_blocks).run().numpy()
        total = r if total is None else {k: total[k] + r[k] for k in total}
    return total, slabs


@pytest.mark.parametrize("cfg,scale,method", [(5, 0.01, "tc"), (1, 1.0, "tc"), (4, 0.004, "tc"), (3, 0.02, "tc"),
                                              (5, 0.005, "plain"), (4, 0.003, "plain")])
@pytest.mark.parametrize("world", [2, 3])
def test_anchor_split_matches_whole_parse(cfg, scale, method, world):
    w = synth.make_config(cfg, scale=scale)
    kw = dict(genotypes=w.genotypes, method=method, max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)
    want = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw).run().numpy()
    got, slabs = _split_parse(w, world, method)
    assert len(slabs) == world
    for k in ("pairs", "r2_counts"):
        np.testing.assert_array_equal(got[k], want[k])
    assert want["pairs"].sum() > 0
    for k in ("sums", "r2_sums"):
        np.testing.assert_allclose(got[k], want[k], rtol=1e-12 if method == "tc" else 1e-11, atol=1e-300)


def test_anchor_end_validation():
    w = synth.make_config(1, scale=0.05)
    with pytest.raises(_lib.LdkError) as e:
        parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="tc", anchor_end=[w.n_var + 1]).run()
    assert e.value.code == _lib.LDK_ERR_ARG
    with pytest.raises(ValueError):
        parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="tc", anchor_end=[1, 2])
    # no anchors: nothing is binned
    r = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="tc", anchor_end=[0]).run().numpy()
    assert r["pairs"].sum() == 0 and not r["sums"].any()
