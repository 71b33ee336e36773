"""The persisted tuning table on the GPU: a shape class tuned once (tile width x row-block
order), written to JSON, cleared and loaded back, is used by a new parse without tuning
again, with the same tile width and the same result bits; a fresh process started with
LDK_AUTOTUNE_CACHE pointing at the file starts from it without tuning."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from pg_gpu_b200 import _lib, parse, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _parser(w):
    return parse.Parser(w.data, w.positions, w.pop_rows, w.edges, genotypes=w.genotypes, method="tc",
                        max_dist=w.max_dist, window_offsets=w.window_offsets, snp_block=w.snp_block,
                        n_blocks=w.n_blocks)


def test_persisted_table_is_used_without_retuning(tmp_path):
    w = synth.make_config(4, scale=0.004)  # several windows: two widths x two orders
    path = str(tmp_path / "tune.json")
    _lib.autotune_clear()
    try:
        _lib.autotune(True)
        p = _parser(w)
        first = {k: v.copy() for k, v in p.run().numpy().items()}
        n, tunings = _lib.autotune_count()
        assert n == 1 and tunings >= 1
        width = p.tile_width()
        assert _lib.autotune_save(path) == 1
        entry = json.load(open(path))["entries"][0]
        assert entry["tile_partners"] == width and entry["order"] in (0, 1) and entry["ms"] > 0
        _lib.autotune_clear()
        assert _lib.autotune_load(path) == 1
        q = _parser(w)
        again = q.run().numpy()
        assert _lib.autotune_count() == (1, tunings)  # no new tuning
        assert q.tile_width() == width
        for k in ("pairs", "r2_counts", "sums", "r2_sums"):
            np.testing.assert_array_equal(again[k], first[k])
    finally:
        _lib.autotune(False)
        _lib.autotune_clear()

    code = ("import sys; sys.path.insert(0, %r)\n"
            "from pg_gpu_b200 import _lib, parse, synth\n"
            "w = synth.make_config(4, scale=0.004)\n"
            "p = parse.Parser(w.data, w.positions, w.pop_rows, w.edges, method='tc', max_dist=w.max_dist,\n"
            "                 window_offsets=w.window_offsets, snp_block=w.snp_block, n_blocks=w.n_blocks)\n"
            "p.run()\n"
            "print(_lib.autotune_count(), p.tile_width())\n" % REPO)
    env = dict(os.environ, LDK_AUTOTUNE="1", LDK_AUTOTUNE_CACHE=path)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == f"(1, 0) {width}"
