"""ldk_parse_noalloc: the parse for callers that cannot allocate device memory (a host
runtime behind a JNI / cgo / N-API layer with no device allocator of its own, or an
application whose memory manager forbids allocations outside its own pool).  Its scratch
is a static device array inside the library, so the caller passes only inputs and
outputs.

Checked through the C ABI against ldk_parse (which takes a caller workspace) on two
calls in a row -- the array keeps the previous call's contents, so the second call
shows that everything that must start at zero is cleared -- with the tolerances of the
other GPU tests; and a parse larger than the array is rejected with a clear error.
This file sorts last so that a run stopping at the first failure has run every other
test first."""
import ctypes

import numpy as np
import pytest

from pg_gpu_b200 import _lib, parse, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = {"plain": 1e-12, "tc": 1e-6}


def _outputs_like(p):
    o = p.out
    outs = parse.ParseResult(sums=torch.full_like(o.sums, 7.0), r2_sums=torch.full_like(o.r2_sums, 7.0),
                             pairs=torch.full_like(o.pairs, 7), r2_counts=torch.full_like(o.r2_counts, 7))
    s = _lib.ParseOut()
    s.sums, s.r2_sums = _lib.ptr(outs.sums), _lib.ptr(outs.r2_sums)
    s.pairs, s.r2_counts = _lib.ptr(outs.pairs), _lib.ptr(outs.r2_counts)
    return outs, s


def _check_same(got, want, tol):
    g, w = got.numpy(), want.numpy()
    np.testing.assert_array_equal(g["pairs"], w["pairs"])
    np.testing.assert_array_equal(g["r2_counts"], w["r2_counts"])
    assert w["pairs"].sum() > 0
    for k in ("sums", "r2_sums"):
        d = np.abs(g[k] - w[k]) / np.maximum(np.abs(w[k]), 1e-300)
        assert float(d.max()) < tol, k


@pytest.mark.parametrize("method,cfg,scale", [("tc", 4, 0.004), ("plain", 4, 0.002), ("tc", 1, 0.05)])
def test_noalloc_matches_workspace_entry_point(method, cfg, scale):
    lib = _lib.load()
    w = synth.make_config(cfg, scale=scale)
    p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method=method, max_dist=w.max_dist,
                     window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks)
    assert lib.ldk_parse_workspace_size(ctypes.byref(p.desc)) <= _lib.NOALLOC_SCRATCH_BYTES
    want = p.run()
    torch.cuda.synchronize()
    for _ in range(2):
        got, o = _outputs_like(p)
        _lib.check(lib.ldk_parse_noalloc(ctypes.byref(p.desc), ctypes.byref(o), _lib.stream_handle()))
        torch.cuda.synchronize()
        _check_same(got, want, TOL[method])


def test_noalloc_rank_slab_matches_workspace_entry_point():
    """One rank's slab of an anchor split (anchors plus right halo, ``anchor_end``): the
    no-allocation entry point lists its row blocks on the device, which must stop at the
    anchor end as the host-built list of ldk_parse does."""
    from pg_gpu_b200 import shard
    lib = _lib.load()
    w = synth.make_config(5, scale=0.01)
    seg = shard.split_anchors(w.positions, [0, w.n_var], w.max_dist, 3)[1]
    sw = shard.slab_workload(w, seg)
    p = parse.Parser(sw.data, sw.positions, sw.pop_rows, sw.edges, method="tc", max_dist=sw.max_dist,
                     window_offsets=sw.window_offsets, anchor_end=sw.anchor_end)
    want = p.run()
    torch.cuda.synchronize()
    for _ in range(2):
        got, o = _outputs_like(p)
        _lib.check(lib.ldk_parse_noalloc(ctypes.byref(p.desc), ctypes.byref(o), _lib.stream_handle()))
        torch.cuda.synchronize()
        _check_same(got, want, TOL["tc"])


def test_noalloc_rejects_oversized_parse():
    lib = _lib.load()
    rng = np.random.default_rng(5)
    n_hap, n_var = 300, 120_000  # tensor-core planes: 120,000 x 2 x 384 B > 64 MiB
    hap = (rng.random((n_hap, n_var)) < 0.3).astype(np.int8)
    pos = np.arange(n_var, dtype=np.float64) * 10.0
    p = parse.Parser(hap, pos, [np.arange(n_hap)], [0.0, 50.0, 100.0], method="tc")
    assert lib.ldk_parse_workspace_size(ctypes.byref(p.desc)) > _lib.NOALLOC_SCRATCH_BYTES
    _, o = _outputs_like(p)
    rc = lib.ldk_parse_noalloc(ctypes.byref(p.desc), ctypes.byref(o), _lib.stream_handle())
    assert rc == _lib.LDK_ERR_UNSUPPORTED
    assert b"static array holds" in lib.ldk_last_error()
