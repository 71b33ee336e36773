"""Host-side parse API on the GPU.  parse.Pipeline: a stream of same-shape batches from
pinned host memory, double-buffered; each batch's results, copied back through the pipeline,
must equal a resident Parser run on the same input (bit-exact: the bin sums are
order-independent).  method="auto": the plain kernel where the tensor-core kernel
cannot stage the shape."""
import numpy as np
import pytest

from pg_gpu_b200 import parse, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batches(w, n, seed):
    """n haplotype matrices of the workload's shape: alleles flipped at random (missing
    calls kept), so every batch has different counts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        x = w.data.copy()
        flip = (rng.random(x.shape) < 0.1) & (x >= 0)
        x[flip] = 1 - x[flip]
        out.append(x)
    return out


@pytest.mark.parametrize("slots", [1, 2])
def test_pipeline_matches_resident_parses(slots):
    w = synth.make_config(4, scale=0.004)
    kw = dict(genotypes=w.genotypes, method="tc", max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)
    reps_w = torch.as_tensor(w.replicate_weights, dtype=torch.int32, device="cuda")

    def make_slot():
        p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
        rw = reps_w.clone()
        return p, {"X": p.X, "pos": p.pos, "block": p.block, "reps_w": rw}, \
            (lambda out: (parse.block_combine(out.sums, rw),))

    pipe = parse.Pipeline(make_slot, slots=slots)
    batches = _batches(w, 3, seed=11)
    pos_h = torch.from_numpy(w.positions.copy()).pin_memory()
    blk_h = torch.from_numpy(w.snp_block.copy()).pin_memory()
    rw_h = reps_w.cpu().pin_memory()
    ref = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
    sums_shape, pairs_shape = tuple(ref.out.sums.shape), tuple(ref.out.pairs.shape)
    rep_shape = (reps_w.shape[0],) + sums_shape[1:]
    outs = [[torch.empty(sums_shape, dtype=torch.float64).pin_memory(),
             torch.empty(pairs_shape, dtype=torch.int64).pin_memory(),
             torch.empty(rep_shape, dtype=torch.float64).pin_memory()] for _ in batches]
    for b, o in zip(batches, outs):
        pipe.submit({"X": torch.from_numpy(b).pin_memory(), "pos": pos_h, "block": blk_h, "reps_w": rw_h}, o)
    pipe.drain()
    torch.cuda.synchronize()
    pipe.status()
    for b, o in zip(batches, outs):
        r = parse.Parser(b, w.positions, w.pop_rows, w.edges, **kw).run()
        want_sums = r.sums.cpu().numpy()
        np.testing.assert_array_equal(o[1].numpy(), r.pairs.cpu().numpy())
        np.testing.assert_array_equal(o[0].numpy(), want_sums)
        want_reps = parse.block_combine(r.sums, reps_w).cpu().numpy()
        np.testing.assert_array_equal(o[2].numpy(), want_reps)
    # the batches differ, so a slot that kept an earlier batch's inputs would have failed
    assert not np.array_equal(outs[0][0].numpy(), outs[1][0].numpy())


def test_pipeline_rejects_mismatched_inputs():
    w = synth.make_config(2, scale=0.004)

    def make_slot():
        p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="tc", max_dist=w.max_dist)
        return p, {"X": p.X, "pos": p.pos}, None

    pipe = parse.Pipeline(make_slot, slots=2)
    with pytest.raises(KeyError):
        pipe.submit({"X": torch.from_numpy(w.data).pin_memory()}, [None, None])
    with pytest.raises(ValueError):
        pipe.submit({"X": torch.from_numpy(w.data).pin_memory(),
                     "pos": torch.from_numpy(w.positions).pin_memory()}, [None])


def test_auto_method_switches_to_plain_where_tc_cannot_stage():
    """Four genotype populations with 40 bins exceed the tensor-core kernel's shared-memory
    staging (36 bins fit): "tc" refuses with LDK_ERR_UNSUPPORTED, "auto" runs the plain FP64
    kernel and matches it; on a shape the tensor-core kernel stages, "auto" keeps it."""
    from pg_gpu_b200 import _lib
    w = synth.make_config(3, scale=0.01)
    n = w.data.shape[0]
    q = n // 4
    rows = [np.arange(k * q, (k + 1) * q) for k in range(4)]
    edges = np.linspace(0, w.max_dist, 41)
    with pytest.raises(_lib.LdkError) as e:
        parse.Parser(w.data, w.positions, rows, edges, genotypes=True, method="tc", max_dist=w.max_dist).run()
    assert e.value.code == _lib.LDK_ERR_UNSUPPORTED
    auto = parse.Parser(w.data, w.positions, rows, edges, genotypes=True, method="auto", max_dist=w.max_dist)
    got = auto.run().numpy()
    assert auto.method == "plain"
    want = parse.Parser(w.data, w.positions, rows, edges, genotypes=True, method="plain",
                        max_dist=w.max_dist).run().numpy()
    np.testing.assert_array_equal(got["pairs"], want["pairs"])
    np.testing.assert_array_equal(got["sums"], want["sums"])
    kept = parse.Parser(w.data, w.positions, rows[:2], w.edges, genotypes=True, method="auto", max_dist=w.max_dist)
    kept.run()
    assert kept.method == "tc"


def test_auto_method_uses_plain_for_small_bootstrap_blocks():
    """Bootstrap blocks of 20 SNPs: a 64-SNP tensor-core row block would span four, more
    than it stages, so "tc" stops with a device error and "auto" runs the plain kernel."""
    from pg_gpu_b200 import _lib
    w = synth.make_config(2, scale=0.01)
    blocks = (np.arange(w.n_var) // 20).astype(np.int32)
    nblk = int(blocks.max()) + 1
    kw = dict(max_dist=w.max_dist, snp_block=blocks, n_blocks=nblk)
    with pytest.raises(_lib.LdkError):
        parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="tc", **kw).run()
    auto = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="auto", **kw)
    got = auto.run().numpy()
    assert auto.method == "plain"
    want = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method="plain", **kw).run().numpy()
    np.testing.assert_array_equal(got["pairs"], want["pairs"])
    np.testing.assert_array_equal(got["sums"], want["sums"])


def test_pipeline_status_reports_an_earlier_batch_error():
    """Four batches through two slots; the second batch's bootstrap-block ids jump inside a
    tensor-core row block (a device error, LDK_DEVERR_BLOCK_SPAN).  Its slot parses the
    fourth, valid batch afterwards, which clears the slot's status word -- status() must
    still raise, naming batch 1."""
    from pg_gpu_b200 import _lib
    w = synth.make_config(4, scale=0.004)
    kw = dict(genotypes=w.genotypes, method="tc", max_dist=w.max_dist, window_offsets=w.window_offsets,
              snp_block=w.snp_block, n_blocks=w.n_blocks)

    def make_slot():
        p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
        return p, {"X": p.X, "pos": p.pos, "block": p.block}, None

    pipe = parse.Pipeline(make_slot, slots=2)
    x_h = torch.from_numpy(w.data.copy()).pin_memory()
    pos_h = torch.from_numpy(w.positions.copy()).pin_memory()
    good = torch.from_numpy(w.snp_block.copy()).pin_memory()
    bad = torch.from_numpy((np.arange(w.n_var) % w.n_blocks).astype(np.int32)).pin_memory()
    ref = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw)
    shapes = (tuple(ref.out.sums.shape), tuple(ref.out.pairs.shape))
    outs = [[torch.empty(shapes[0], dtype=torch.float64).pin_memory(),
             torch.empty(shapes[1], dtype=torch.int64).pin_memory()] for _ in range(4)]
    for k in range(4):
        pipe.submit({"X": x_h, "pos": pos_h, "block": bad if k == 1 else good}, outs[k])
    pipe.drain()
    with pytest.raises(_lib.LdkError) as e:
        pipe.status()
    assert e.value.code == _lib.LDK_ERR_DEVICE
    assert "batch 1" in str(e.value) and "bootstrap blocks" in str(e.value)
    # the error was reported once; later batches are checked afresh
    pipe.submit({"X": x_h, "pos": pos_h, "block": good}, outs[0])
    pipe.drain()
    pipe.status()
