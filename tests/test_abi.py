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
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(ldk_parse_t), offsetof(ldk_parse_t, pop_offsets),
         offsetof(ldk_parse_t, max_dist), offsetof(ldk_parse_t, edges), offsetof(ldk_parse_t, window_offsets),
         offsetof(ldk_parse_t, method), sizeof(ldk_parse_out_t), offsetof(ldk_parse_out_t, r2_counts));
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
            D.window_offsets.offset, D.method.offset, ctypes.sizeof(O), O.r2_counts.offset]
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
