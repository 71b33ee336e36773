"""The C-ABI library loads and exports every entry point of include/ldk.h (no GPU);
ctypes mirrors of the descriptor structs match the C layout."""
import os
import re
import subprocess
import tempfile

import pytest

from pg_gpu_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "ldk.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"LDK_API\s+[\w\s\*]+?\b(ldk_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.EXPORTS, f"{s} has no ctypes signature"
    assert lib.ldk_version() >= 10000
    assert [lib.ldk_n_stats(p) for p in (1, 2, 3, 4)] == [3, 15, 45, 105]


def test_struct_layout_matches_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "ldk.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(ldk_parse_t), offsetof(ldk_parse_t, pop_offsets),
         offsetof(ldk_parse_t, max_dist), offsetof(ldk_parse_t, edges), offsetof(ldk_parse_t, window_offsets),
         offsetof(ldk_parse_t, method), offsetof(ldk_parse_t, anchor_end), offsetof(ldk_parse_t, x_format),
         sizeof(ldk_parse_out_t), offsetof(ldk_parse_out_t, r2_counts));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    D, O = _lib.ParseDesc, _lib.ParseOut
    import ctypes
    want = [ctypes.sizeof(D), D.pop_offsets.offset, D.max_dist.offset, D.edges.offset,
            D.window_offsets.offset, D.method.offset, D.anchor_end.offset, D.x_format.offset,
            ctypes.sizeof(O), O.r2_counts.offset]
    assert got == want


def test_validation_errors_without_gpu():
    """Argument validation runs on the host: a bad descriptor sizes no workspace."""
    import ctypes
    lib = _lib.load()
    d = _lib.ParseDesc()
    d.n_pops = 5
    d.n_bins = 4
    assert lib.ldk_parse_workspace_size(ctypes.byref(d)) == 0
    assert b"n_pops" in lib.ldk_last_error()
    d.n_pops = 1
    d.n_bins = 2
    d.edges[0], d.edges[1], d.edges[2] = 0.0, 10.0, 5.0
    assert lib.ldk_parse_workspace_size(ctypes.byref(d)) == 0
    assert b"edges" in lib.ldk_last_error()


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.require_cuda()


def test_autotune_table_file_round_trip(tmp_path):
    """The tuning table's JSON file (host-only entry points): a written table loads back
    entry for entry, clearing empties it, and a file that is not such a table is refused."""
    import json
    _lib.autotune_clear()
    assert _lib.autotune_count()[0] == 0
    src = tmp_path / "table.json"
    entries = [{"pops": 3, "genotypes": 0, "k_bytes": 512, "bins": 16, "cutoff_decade": 6, "window_log2": 11,
                "tile_variant": 1, "tile_partners": 16, "order": 1, "ms": 12.5},
               {"pops": 1, "genotypes": 1, "k_bytes": 512, "bins": 20, "cutoff_decade": 5, "window_log2": 16,
                "tile_variant": 0, "tile_partners": 16, "order": 0, "ms": 9.0}]
    src.write_text('{"format": "ldk-autotune", "version": 1, "entries": [\n'
                   + ",\n".join(json.dumps(e) for e in entries) + "\n]}\n")
    assert _lib.autotune_load(str(src)) == 2
    assert _lib.autotune_count()[0] == 2
    out = tmp_path / "saved.json"
    assert _lib.autotune_save(str(out)) == 2
    saved = json.loads(out.read_text())
    assert saved["format"] == "ldk-autotune"
    key = lambda e: (e["pops"], e["genotypes"], e["k_bytes"], e["bins"], e["cutoff_decade"], e["window_log2"])  # noqa
    got = {key(e): (e["tile_variant"], e["order"]) for e in saved["entries"]}
    assert got == {key(e): (e["tile_variant"], e["order"]) for e in entries}
    # the width is written from the library's tile table, not copied from the input
    assert all(e["tile_partners"] > 0 for e in saved["entries"])
    _lib.autotune_clear()
    assert _lib.autotune_count()[0] == 0
    bad = tmp_path / "bad.json"
    bad.write_text('{"something": "else"}')
    with pytest.raises(_lib.LdkError):
        _lib.autotune_load(str(bad))
    with pytest.raises(_lib.LdkError):
        _lib.autotune_load(str(tmp_path / "missing.json"))


def test_reproducibility_query_without_gpu():
    """ldk_parse_reproducible (host-only): the plain kernel and the tensor-core shapes with a
    staging copy per epilogue warp (configurations 1-5) are bit-reproducible; four
    populations and three genotype populations with more than five bins share one staging
    copy and are not."""
    import ctypes
    lib = _lib.load()

    def desc(P, geno, nb, n_each, method=_lib.METHOD_TC):
        d = _lib.ParseDesc()
        d.n_pops, d.genotypes, d.n_bins, d.n_blocks, d.method, d.max_dist = P, geno, nb, 1, method, 1.0
        for k in range(nb + 1):
            d.edges[k] = float(k)
        for k in range(5):
            d.pop_offsets[k] = min(k, P) * n_each
        return d

    cases = {(1, 0, 4, 100): 1, (2, 0, 16, 120): 1, (3, 0, 16, 160): 1, (1, 1, 20, 500): 1, (1, 0, 32, 2000): 1,
             (4, 0, 16, 150): 0, (3, 1, 6, 160): 0, (3, 1, 5, 160): 1}
    for (P, g, nb, n), want in cases.items():
        assert lib.ldk_parse_reproducible(ctypes.byref(desc(P, g, nb, n))) == want, (P, g, nb, n)
    assert lib.ldk_parse_reproducible(ctypes.byref(desc(4, 1, 16, 125, _lib.METHOD_PLAIN))) == 1
    bad = desc(5, 0, 4, 10)
    assert lib.ldk_parse_reproducible(ctypes.byref(bad)) == _lib.LDK_ERR_ARG
