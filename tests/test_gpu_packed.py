"""Packed ingest (LDK_X_PACKED2, ``parse.pack_codes``): the tensor-core parse of a matrix
stored in two bits per entry gives the same bits as the parse of the int8 matrix (the
plane preparation unpacks each code into the same indicator planes), for haplotypes and
genotypes, with windows, bootstrap blocks and missing calls, at n_var not a multiple of
four; through ``Pipeline`` from pinned host memory too.  The plain method refuses it."""
import numpy as np
import pytest

from pg_gpu_b200 import _lib, parse, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _kw(w):
    return dict(genotypes=w.genotypes, method="tc", max_dist=w.max_dist, window_offsets=w.window_offsets,
                snp_block=w.snp_block, n_blocks=w.n_blocks)


@pytest.mark.parametrize("cfg,scale,trim", [(5, 0.01, 3), (3, 0.02, 1), (4, 0.004, 0), (2, 0.01, 2)])
def test_packed_parse_equals_int8_parse(cfg, scale, trim):
    w = synth.make_config(cfg, scale=scale)
    data, pos = w.data, w.positions
    kw = _kw(w)
    if trim:  # n_var not a multiple of 4 (one window: drop the last SNPs)
        assert w.window_offsets is None
        data, pos = data[:, :-trim], pos[:-trim]
        if w.snp_block is not None:
            kw["snp_block"] = w.snp_block[:-trim]
    want = parse.Parser(data, pos, w.pop_rows, w.edges, **kw).run().numpy()
    got = parse.Parser(parse.pack_codes(data), pos, w.pop_rows, w.edges, packed=True, **kw).run().numpy()
    assert want["pairs"].sum() > 0
    for k in ("pairs", "r2_counts", "sums", "r2_sums"):
        np.testing.assert_array_equal(got[k], want[k])


def test_packed_rejected_by_plain_method():
    w = synth.make_config(1, scale=0.05)
    with pytest.raises(_lib.LdkError) as e:
        parse.Parser(parse.pack_codes(w.data), w.positions, w.pop_rows, w.edges, packed=True, method="plain").run()
    assert e.value.code == _lib.LDK_ERR_UNSUPPORTED


def test_packed_pipeline_matches_resident():
    w = synth.make_config(5, scale=0.01)
    kw = _kw(w)
    packed = parse.pack_codes(w.data)

    def make_slot():
        p = parse.Parser(packed, w.positions, w.pop_rows, w.edges, packed=True, **kw)
        return p, {"X": p.X, "pos": p.pos}, None

    pipe = parse.Pipeline(make_slot, slots=2)
    ref = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, **kw).run().numpy()
    x_h = torch.from_numpy(packed.view(np.int8)).pin_memory()
    pos_h = torch.from_numpy(w.positions.copy()).pin_memory()
    outs = [[torch.empty(ref["sums"].shape, dtype=torch.float64).pin_memory(),
             torch.empty(ref["pairs"].shape, dtype=torch.int64).pin_memory()] for _ in range(3)]
    for o in outs:
        pipe.submit({"X": x_h, "pos": pos_h}, o)
    pipe.drain()
    pipe.status()
    for o in outs:
        np.testing.assert_array_equal(o[0].numpy(), ref["sums"])
        np.testing.assert_array_equal(o[1].numpy(), ref["pairs"])


@pytest.mark.parametrize("cfg,scale", [(4, 0.004), (3, 0.02)])
def test_plane_gather_forms_agree(cfg, scale):
    """The plane preparation's gather forms give the same planes: rows that start off a
    4-byte boundary (odd row stride: two aligned words joined per quad), the same matrix in
    a buffer whose row stride is padded to a multiple of four (one word per quad), the
    padded buffer read from a base one byte past a word boundary, and the packed form;
    checked through the parse outputs, bit for bit, with an odd SNP count."""
    from pg_gpu_b200 import _lib
    import ctypes
    w = synth.make_config(cfg, scale=scale)
    kw = _kw(w)
    n_var = w.n_var if w.n_var % 2 else w.n_var - 1
    if n_var != w.n_var:  # keep the window offsets valid: drop the last SNP of the last window
        data, pos = w.data[:, :n_var], w.positions[:n_var]
        if w.window_offsets is not None:
            kw["window_offsets"] = np.concatenate([w.window_offsets[:-1], [n_var]])
        if w.snp_block is not None:
            kw["snp_block"] = w.snp_block[:n_var]
    else:
        data, pos = w.data, w.positions
    p = parse.Parser(data, pos, w.pop_rows, w.edges, **kw)
    assert p.desc.ld_x % 4 != 0
    odd = {k: v.copy() for k, v in p.run().numpy().items()}
    ld = (n_var + 15) // 16 * 16
    padded = torch.zeros((data.shape[0], ld), dtype=torch.int8, device="cuda")
    padded[:, :n_var] = torch.as_tensor(data, device="cuda")
    p.desc.X, p.desc.ld_x = _lib.ptr(padded), ld
    wide = {k: v.copy() for k, v in p.run().numpy().items()}
    shifted = torch.zeros((data.shape[0], ld + 16), dtype=torch.int8, device="cuda")
    shifted[:, 1:n_var + 1] = torch.as_tensor(data, device="cuda")
    p.desc.X, p.desc.ld_x = shifted.data_ptr() + 1, ld + 16
    unaligned = {k: v.copy() for k, v in p.run().numpy().items()}
    packed = parse.Parser(parse.pack_codes(data), pos, w.pop_rows, w.edges, packed=True, **kw).run().numpy()
    assert odd["pairs"].sum() > 0
    for k in ("pairs", "r2_counts", "sums", "r2_sums"):
        np.testing.assert_array_equal(wide[k], odd[k])
        np.testing.assert_array_equal(unaligned[k], odd[k])
        np.testing.assert_array_equal(packed[k], odd[k])
