"""pg_gpu's own haplotype estimator kernels on the CPU: the kernel bodies compiled for the
host by ``oracle/build_ref.py`` (``oracle/_ref/libpgref.so``; each CUDA thread becomes one
iteration of a host loop), driven by a restatement of pg_gpu's dispatch of them.

Test infrastructure and the reference arm of ``bench.py`` only: never imported by the
package.  The reference's Python modules stay in its checkout (they do not travel with
this repository); what travels is the compiled library of its kernels.  Restated here,
in this file's own code:

* ``PopData`` features (``ld_pipeline.py:465-482``): float64 counts c1..c4, n = n_valid (or
  the count sum), D = c2 c3 - c1 c4, pA = c1 + c2, qA = c3 + c4, pB = c1 + c3, qB = c2 + c4,
  concatenated over populations as ``_HapPopFlat`` does (``haplotype_kernels.py:312-327``),
  index = population * N + pair;
* the grouping of raw calls into kernel launches and their arguments
  (``compute_all_dd_hap`` / ``compute_all_dz_hap`` / ``compute_all_pi2_hap``,
  ``haplotype_kernels.py:335-582``);
* the weighted assembly of the moments statistics from the raw calls
  (``compute_multi_pop_statistics_batch_hap``, ``haplotype_kernels.py:584-640``), with the
  averaging specs of ``generate_stat_specs`` (``ld_pipeline.py:388-457``; the oracle's
  ``stat_specs`` reproduces them).

pg_gpu runs this path for one, three and four populations; two populations go through
``compute_two_pop_statistics_batch`` (``ld_pipeline.py:271-322``, NumPy formulas), which the
oracle restates (``ld_oracle.hap_stats``).
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
_LIB = None


def available() -> bool:
    return os.path.exists(os.path.join(REF_OUT, "libpgref.so")) and os.path.exists(
        os.path.join(REF_OUT, "kernels.json"))


def _kernels():
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError("oracle/_ref is not built (python oracle/build_ref.py)")
        lib = ctypes.CDLL(os.path.join(REF_OUT, "libpgref.so"))
        with open(os.path.join(REF_OUT, "kernels.json")) as f:
            table = json.load(f)
        by_name = {}
        for ent in table.values():
            if ent["module"] == "haplotype_kernels":
                fn = getattr(lib, ent["symbol"])
                fn.restype = None
                by_name[ent["attr"]] = (fn, ent["params"])
        _LIB = by_name
    return _LIB


def _launch(name, args, M):
    """One launch of kernel ``name`` over M outputs: grid of ceil(M / 256) blocks of 256
    threads (haplotype_kernels.py:11-13), run as a host loop."""
    fn, params = _kernels()[name]
    if len(args) != len(params):
        raise TypeError(f"{name}: {len(args)} arguments for {len(params)} parameters")
    keep, cargs = [], []
    for a, t in zip(args, params):
        if t == "ptr":
            a = np.ascontiguousarray(a)
            keep.append(a)
            cargs.append(ctypes.c_void_p(a.ctypes.data))
        elif t == "i64":
            cargs.append(ctypes.c_longlong(int(a)))
        else:
            cargs.append(ctypes.c_int(int(a)))
    cargs.append(ctypes.c_longlong((int(M) + 255) // 256 * 256))
    fn(*cargs)


class _Flat:
    """PopData features of every population, concatenated (index = pop * N + pair)."""

    def __init__(self, counts_list, n_valid_list):
        c = [np.asarray(x, dtype=np.float64) for x in counts_list]
        self.N = c[0].shape[0]
        self.c1 = np.concatenate([x[:, 0] for x in c])
        self.c2 = np.concatenate([x[:, 1] for x in c])
        self.c3 = np.concatenate([x[:, 2] for x in c])
        self.c4 = np.concatenate([x[:, 3] for x in c])
        ns = []
        for x, nv in zip(c, n_valid_list or [None] * len(c)):
            ns.append(np.asarray(nv, dtype=np.float64) if nv is not None else x[:, 0] + x[:, 1] + x[:, 2] + x[:, 3])
        self.n = np.concatenate(ns)
        self.D = self.c2 * self.c3 - self.c1 * self.c4
        self.pA = self.c1 + self.c2
        self.qA = self.c3 + self.c4
        self.pB = self.c1 + self.c3
        self.qB = self.c2 + self.c4

    def expand(self, pops):
        return (np.asarray(pops, dtype=np.int32)[:, None] * self.N
                + np.arange(self.N, dtype=np.int32)[None, :]).ravel().astype(np.int32)


def _dd(F, calls):
    out = {}
    single = [c for c in calls if c[0] == c[1]]
    between = [c for c in calls if c[0] != c[1]]
    if single:
        M = len(single) * F.N
        r = np.empty(M)
        _launch("_DD_SINGLE_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.expand([c[0] for c in single]), r, M), M)
        out.update({c: r[k * F.N:(k + 1) * F.N] for k, c in enumerate(single)})
    if between:
        M = len(between) * F.N
        r = np.empty(M)
        _launch("_DD_BETWEEN_KERN", (F.D, F.n, F.expand([c[0] for c in between]),
                                     F.expand([c[1] for c in between]), r, M), M)
        out.update({c: r[k * F.N:(k + 1) * F.N] for k, c in enumerate(between)})
    return out


def _dz_group(c):
    p1, p2, p3 = c
    if p1 == p2 == p3:
        return "same"
    if p1 == p2:
        return "p1p2"
    if p1 == p3:
        return "p1p3"
    if p2 == p3:
        return "p2p3"
    return "diff"


def _dz(F, calls):
    out = {}
    for g in ("same", "p1p2", "p1p3", "p2p3", "diff"):
        cs = [c for c in calls if _dz_group(c) == g]
        if not cs:
            continue
        M = len(cs) * F.N
        r = np.empty(M)
        I = F.expand([c[0] for c in cs])
        if g == "diff":
            _launch("_DZ_DIFF_KERN", (F.D, F.n, F.pA, F.qA, F.c1, F.c2, F.c3, F.c4, I,
                                      F.expand([c[1] for c in cs]), F.expand([c[2] for c in cs]), r, M), M)
        elif g == "p1p2":
            _launch("_DZ_IIJ_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, I,
                                     F.expand([c[2] for c in cs]), r, M), M)
        elif g == "p1p3":
            _launch("_DZ_IJI_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, I,
                                     F.expand([c[1] for c in cs]), r, M), M)
        elif g == "p2p3":
            _launch("_DZ_IJJ_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, I,
                                     F.expand([c[1] for c in cs]), r, M), M)
        else:
            _launch("_DZ_III_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, I, r, M), M)
        out.update({c: r[k * F.N:(k + 1) * F.N] for k, c in enumerate(cs)})
    return out


def _pi2_group(c):
    i, j, k, l = c
    cnt = {}
    for p in c:
        cnt[p] = cnt.get(p, 0) + 1
    nu, mc = len(cnt), max(cnt.values())
    if nu == 1:
        return "same"
    if mc == 3:
        return "triple"
    if i == j and k == l:
        return "iikk"
    if i == j:
        return "iikl"
    if k == l:
        return "ijkk"
    if (i == k and j == l) or (i == l and j == k):
        return "ijij"
    return "shared" if nu == 3 else "alldiff"


def _shared_roles(c):
    i, j, k, l = c
    if i == k:
        return i, j, l
    if i == l:
        return i, j, k
    if j == k:
        return j, i, l
    if j == l:
        return j, i, k
    return 0, 0, 0


def _triple_roles(c):
    cnt = {}
    for p in c:
        cnt[p] = cnt.get(p, 0) + 1
    return [p for p, n in cnt.items() if n == 3][0], [p for p, n in cnt.items() if n == 1][0]


def _pi2(F, calls):
    out = {}
    col = lambda cs, q: F.expand([c[q] for c in cs])  # noqa: E731
    for g in ("same", "triple", "iikk", "iikl", "ijkk", "ijij", "shared", "alldiff"):
        cs = [c for c in calls if _pi2_group(c) == g]
        if not cs:
            continue
        M = len(cs) * F.N
        r = np.empty(M)
        if g == "alldiff":
            _launch("_PI2_ALLDIFF_KERN", (F.pA, F.qA, F.pB, F.qB, F.n, col(cs, 0), col(cs, 1), col(cs, 2),
                                          col(cs, 3), r, M), M)
        elif g == "iikk":
            _launch("_PI2_IIKK_KERN", (F.pA, F.qA, F.pB, F.qB, F.n, col(cs, 0), col(cs, 2), r, M), M)
        elif g == "iikl":
            _launch("_PI2_IIKL_KERN", (F.pA, F.qA, F.pB, F.qB, F.n, col(cs, 0), col(cs, 2), col(cs, 3), r, M), M)
        elif g == "ijkk":
            _launch("_PI2_IJKK_KERN", (F.pA, F.qA, F.pB, F.qB, F.n, col(cs, 0), col(cs, 1), col(cs, 2), r, M), M)
        elif g == "shared":
            roles = [_shared_roles(c) for c in cs]
            _launch("_PI2_SHARED_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, F.pB, F.qB,
                                         F.expand([x[0] for x in roles]), F.expand([x[1] for x in roles]),
                                         F.expand([x[2] for x in roles]), r, M), M)
        elif g == "triple":
            roles = [_triple_roles(c) for c in cs]
            _launch("_PI2_TRIPLE_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, F.pB, F.qB,
                                         F.expand([x[0] for x in roles]), F.expand([x[1] for x in roles]), r, M), M)
        elif g == "ijij":
            _launch("_PI2_IJIJ_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, F.pA, F.qA, F.pB, F.qB, col(cs, 0), col(cs, 1),
                                       r, M), M)
        else:
            _launch("_PI2_IIII_KERN", (F.c1, F.c2, F.c3, F.c4, F.n, col(cs, 0), r, M), M)
        out.update({c: r[k * F.N:(k + 1) * F.N] for k, c in enumerate(cs)})
    return out


def hap_stats(counts_list, n_valid_list=None):
    """(N, n_stats) moments-ordered statistics of P populations through pg_gpu's own
    kernels, the oracle's ``hap_stats`` signature."""
    from oracle import ld_oracle as O
    P = len(counts_list)
    specs = O.stat_specs(P)
    F = _Flat(counts_list, n_valid_list)
    unique = {(st, tuple(pi)) for _, calls in specs for _, st, pi in calls}
    raw = {}
    for kind, fn in (("dd", _dd), ("dz", _dz), ("pi2", _pi2)):
        calls = sorted(pi for st, pi in unique if st == kind)
        if calls:
            raw.update({(kind, pi): v for pi, v in fn(F, calls).items()})
    out = np.zeros((F.N, len(specs)))
    for s, (_, calls) in enumerate(specs):
        out[:, s] = sum(w * raw[(st, tuple(pi))] for w, st, pi in calls)
    return out
