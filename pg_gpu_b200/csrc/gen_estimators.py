"""Generate ``ldk_estimators.cuh``: straight-line two-locus LD estimators for P = 1..4.

The moments statistics of P populations (names and averaging weights as in
``ld_pipeline.py:357-457`` of pg_gpu) are sums of raw estimator calls DD(i,j), Dz(i,j,k),
pi2(i,j,k,l).  Every raw call of the haplotype path is a product of per-population
features (counts, allele counts, D, and a handful of quadratic/cubic count
polynomials) times per-population reciprocal denominators, so a pair's full statistic
vector is computed here as

  1. per population: features + reciprocals 1/n, 1/(n(n-1)), 1/(n(n-1)(n-2)),
     1/(n(n-1)(n-2)(n-3)) (0 where the reference's guard ``den > 0`` fails);
  2. per distinct raw call (calls equal by symmetry evaluated once): a few products;
  3. per statistic: the weighted sum, added into an accumulator.

The feature algebra was derived with sympy from the reference's formulas
(``haplotype_kernels.py:69-304``); ``check()`` re-verifies every identity
symbolically and the unit tests evaluate the same expression strings with NumPy
against the float64 oracle.  The genotype path (``genotype_kernels.py``) keeps the
reference's polynomial forms, which are written once in
``ldk_geno_poly.cuh`` and shared by every kernel.

Run ``python -m pg_gpu_b200.csrc.gen_estimators`` to regenerate; ``build()`` does it.
"""
from __future__ import annotations

import functools
import os

HERE = os.path.dirname(os.path.abspath(__file__))

# ---------------------------------------------------------------------------
# statistic specs (moments order and _call_sgc averaging)
# ---------------------------------------------------------------------------


def ld_names(P):
    names = []
    for i in range(P):
        for j in range(i, P):
            names.append(("dd", (i, j)))
    for i in range(P):
        for j in range(P):
            for k in range(j, P):
                names.append(("dz", (i, j, k)))
    for i in range(P):
        for j in range(i, P):
            for k in range(i, P):
                for l in range(k, P):
                    if k == i == l and j != i:
                        continue
                    if i == k and l < j:
                        continue
                    names.append(("pi2", (i, j, k, l)))
    return names


def stat_name(kind, p):
    return {"dd": "DD", "dz": "Dz", "pi2": "pi2"}[kind] + "_" + "_".join(str(x) for x in p)


def stat_specs(P):
    out = []
    for kind, p in ld_names(P):
        if kind == "dd":
            calls = [(1.0, "dd", p)]
        elif kind == "dz":
            i, j, k = p
            calls = [(1.0, "dz", p)] if j == k else [(0.5, "dz", (i, j, k)), (0.5, "dz", (i, k, j))]
        else:
            i, j, k, l = p
            if i == j and k == l:
                qs = [(1.0, p)] if i == k else [(0.5, (i, j, k, l)), (0.5, (k, l, i, j))]
            elif i == j:
                qs = [(0.25, q) for q in ((i, j, k, l), (i, j, l, k), (k, l, i, j), (l, k, i, j))]
            elif k == l:
                qs = [(0.25, q) for q in ((i, j, k, l), (j, i, k, l), (k, l, i, j), (k, l, j, i))]
            else:
                qs = [(0.125, q) for q in ((i, j, k, l), (i, j, l, k), (j, i, k, l), (j, i, l, k),
                                            (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i))]
            calls = [(w, "pi2", q) for w, q in qs]
        out.append((stat_name(kind, p), calls))
    return out


def _pi2_case(p):
    i, j, k, l = p
    cnt = {}
    for q in p:
        cnt[q] = cnt.get(q, 0) + 1
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
    if nu == 3:
        return "shared"
    return "alldiff"


def _counts_of(p):
    cnt = {}
    for q in p:
        cnt[q] = cnt.get(q, 0) + 1
    return cnt


def canonical(kind, p, geno=False):
    """Canonical (case, args) of a raw call; calls with equal canonical form are equal."""
    if kind == "dd":
        return ("dd1", (p[0],)) if p[0] == p[1] else ("dd2", p)
    if kind == "dz":
        a, b, c = p
        if a == b == c:
            return ("dz_iii", (a,))
        if a == b:
            return ("dz_iij", (a, c))
        if a == c:
            return ("dz_iji", (a, b))
        if b == c:
            return ("dz_ijj", (a, b))
        return ("dz_ijk", p)
    case = _pi2_case(p)
    i, j, k, l = p
    if case == "same":
        return ("pi2_same", (i,))
    if case == "triple":
        cnt = _counts_of(p)
        t = [q for q, c in cnt.items() if c == 3][0]
        s = [q for q, c in cnt.items() if c == 1][0]
        if geno:
            return ("pi2_iiij" if (i == t and j == t) else "pi2_ijii", (t, s))
        return ("pi2_triple", (t, s))
    if case == "iikk":
        return ("pi2_iikk", (i, k))
    if case == "iikl":
        return ("pi2_iikl", (i,) + tuple(sorted((k, l))))
    if case == "ijkk":
        return ("pi2_ijkk", tuple(sorted((i, j))) + (k,))
    if case == "ijij":
        return ("pi2_ijij", (i, j))
    if case == "shared":
        if i == k:
            r = (i, j, l)
        elif i == l:
            r = (i, j, k)
        elif j == k:
            r = (j, i, l)
        else:
            r = (j, i, k)
        return ("pi2_shared", r)
    return ("pi2_alldiff", tuple(sorted((i, j))) + tuple(sorted((k, l))))


# ---------------------------------------------------------------------------
# haplotype path: per-population features and raw-call expressions
# ---------------------------------------------------------------------------

# Per-population feature definitions (C and Python share the syntax).  x.c1..c4 are the
# two-locus counts n11, n10, n01, n00 of ld_statistics.py:281-290; x.ns their sum; x.n the
# sample size used in denominators (n_valid; equal to ns on the haplotype path).
HAP_FEATURES = [
    ("pA", "x.c1 + x.c2"),
    ("qA", "x.c3 + x.c4"),
    ("pB", "x.c1 + x.c3"),
    ("qB", "x.c2 + x.c4"),
    ("E", "x.c1 * x.c4 - x.c2 * x.c3"),          # = -D of ld_pipeline.py:478
    ("a", "x.qA - x.pA"),
    ("b", "x.qB - x.pB"),
    ("s", "(x.c2 + x.c3) - (x.c1 + x.c4)"),
    ("fA", "x.pA * x.qA"),
    ("fB", "x.pB * x.qB"),
    # coefficients of the bilinear pi2(i,j,i,j) correction and of pi2 shared
    ("Q1", "x.c1 * (1 - x.ns + x.c4) - x.c2 * x.c3"),
    ("Q2", "x.c2 * (1 - x.ns + x.c3) - x.c1 * x.c4"),
    ("Q3", "x.c3 * (1 - x.ns + x.c2) - x.c1 * x.c4"),
    ("Q4", "x.c4 * (1 - x.ns + x.c1) - x.c2 * x.c3"),
    ("L1", "x.c4 * (x.ns - x.c1) + x.c2 * x.c3"),
    ("L2", "x.c3 * (x.ns - x.c2) + x.c1 * x.c4"),
    ("L3", "x.c2 * (x.ns - x.c3) + x.c1 * x.c4"),
    ("L4", "x.c1 * (x.ns - x.c4) + x.c2 * x.c3"),
    # pi2 with one population three times: 2*num = pB_s*T1_t + qB_s*T2_t
    ("T1", "x.fA * x.qB - x.c1 * x.c4 - x.c2 * x.c3 - 2 * x.c2 * x.c4"),
    ("T2", "x.fA * x.pB - 2 * x.c1 * x.c3 - x.c1 * x.c4 - x.c2 * x.c3"),
    # single-population numerators
    ("DDs", "x.E * x.E - x.c1 * x.c4 * (x.c1 + x.c4 - 1) - x.c2 * x.c3 * (x.c2 + x.c3 - 1)"),
    ("DZs", "x.E * x.a * x.b + x.E * x.s + 2 * (x.c2 * x.c3 + x.c1 * x.c4)"),
    ("PIs", "x.fA * x.fB - x.c1 * x.c4 * (-1 + x.c1 + 3 * x.c2 + 3 * x.c3 + x.c4)"
            " - x.c2 * x.c3 * (-1 + 3 * x.c1 + x.c2 + x.c3 + 3 * x.c4)"),
]

# which features each case reads (besides counts); drives what is computed per P
HAP_CASE_FEATURES = {
    "dd1": ["DDs", "r4"], "dd2": ["E", "r2"],
    "dz_iii": ["DZs", "r4"], "dz_iij": ["a", "E", "b", "r3", "r1"],
    "dz_iji": ["a", "E", "b", "r3", "r1"], "dz_ijj": ["E", "s", "a", "b", "r2"],
    "dz_ijk": ["E", "a", "b", "r2", "r1"],
    "pi2_same": ["PIs", "r4"], "pi2_iikk": ["fA", "fB", "r2"],
    "pi2_iikl": ["fA", "pB", "qB", "r2", "r1"], "pi2_ijkk": ["fB", "pA", "qA", "r2", "r1"],
    "pi2_alldiff": ["pA", "qA", "pB", "qB", "r1"], "pi2_triple": ["T1", "T2", "pB", "qB", "r3", "r1"],
    "pi2_ijij": ["pA", "qA", "pB", "qB", "Q1", "Q2", "Q3", "Q4", "L1", "L2", "L3", "L4", "r2"],
    "pi2_shared": ["pA", "qA", "pB", "qB", "L1", "L2", "L3", "L4", "r2", "r1"],
}


def hap_call_expr(case, args):
    """Expression (C and Python syntax) of one canonical raw haplotype call."""
    f = lambda p, name: f"f[{p}].{name}"  # noqa: E731
    if case == "dd1":
        (i,) = args
        return f"{f(i,'DDs')} * {f(i,'r4')}"
    if case == "dd2":
        i, j = args
        return f"({f(i,'E')} * {f(j,'E')}) * ({f(i,'r2')} * {f(j,'r2')})"
    if case == "dz_iii":
        (i,) = args
        return f"{f(i,'DZs')} * {f(i,'r4')}"
    if case == "dz_iij":
        i, j = args
        return f"({f(i,'a')} * {f(i,'E')} * {f(j,'b')}) * ({f(i,'r3')} * {f(j,'r1')})"
    if case == "dz_iji":
        i, j = args
        return f"({f(i,'b')} * {f(i,'E')} * {f(j,'a')}) * ({f(i,'r3')} * {f(j,'r1')})"
    if case == "dz_ijj":
        i, j = args
        return (f"({f(i,'E')} * ({f(j,'s')} + {f(j,'b')} * {f(j,'a')}))"
                f" * ({f(i,'r2')} * {f(j,'r2')})")
    if case == "dz_ijk":
        i, j, k = args
        return (f"({f(i,'E')} * {f(j,'a')} * {f(k,'b')})"
                f" * ({f(i,'r2')} * {f(j,'r1')} * {f(k,'r1')})")
    if case == "pi2_same":
        (i,) = args
        return f"{f(i,'PIs')} * {f(i,'r4')}"
    if case == "pi2_iikk":
        i, k = args
        return f"({f(i,'fA')} * {f(k,'fB')}) * ({f(i,'r2')} * {f(k,'r2')})"
    if case == "pi2_iikl":
        i, k, l = args
        return (f"0.5 * ({f(i,'fA')} * ({f(k,'pB')} * {f(l,'qB')} + {f(k,'qB')} * {f(l,'pB')}))"
                f" * ({f(i,'r2')} * {f(k,'r1')} * {f(l,'r1')})")
    if case == "pi2_ijkk":
        i, j, k = args
        return (f"0.5 * ({f(k,'fB')} * ({f(i,'pA')} * {f(j,'qA')} + {f(i,'qA')} * {f(j,'pA')}))"
                f" * ({f(k,'r2')} * {f(i,'r1')} * {f(j,'r1')})")
    if case == "pi2_alldiff":
        i, j, k, l = args
        return (f"0.25 * (({f(i,'pA')} * {f(j,'qA')} + {f(i,'qA')} * {f(j,'pA')})"
                f" * ({f(k,'pB')} * {f(l,'qB')} + {f(k,'qB')} * {f(l,'pB')}))"
                f" * ({f(i,'r1')} * {f(j,'r1')} * {f(k,'r1')} * {f(l,'r1')})")
    if case == "pi2_triple":
        t, s = args
        return (f"0.5 * ({f(s,'pB')} * {f(t,'T1')} + {f(s,'qB')} * {f(t,'T2')})"
                f" * ({f(t,'r3')} * {f(s,'r1')})")
    if case == "pi2_ijij":
        i, j = args
        HA = f"({f(i,'pA')} * {f(j,'qA')} + {f(i,'qA')} * {f(j,'pA')})"
        HB = f"({f(i,'pB')} * {f(j,'qB')} + {f(i,'qB')} * {f(j,'pB')})"
        corr = (f"({f(i,'Q1')} * {f(j,'c4')} + {f(i,'Q2')} * {f(j,'c3')} + {f(i,'Q3')} * {f(j,'c2')}"
                f" + {f(i,'Q4')} * {f(j,'c1')} - ({f(i,'c1')} * {f(j,'L1')} + {f(i,'c2')} * {f(j,'L2')}"
                f" + {f(i,'c3')} * {f(j,'L3')} + {f(i,'c4')} * {f(j,'L4')}))")
        return f"0.25 * ({HA} * {HB} + {corr}) * ({f(i,'r2')} * {f(j,'r2')})"
    if case == "pi2_shared":
        s, a, b = args
        F1 = f"({f(s,'L1')} - {f(s,'c4')})"
        F2 = f"({f(s,'L2')} - {f(s,'c3')})"
        F3 = f"({f(s,'L3')} - {f(s,'c2')})"
        F4 = f"({f(s,'L4')} - {f(s,'c1')})"
        return (f"0.25 * ({f(a,'pA')} * ({f(b,'pB')} * {F1} + {f(b,'qB')} * {F2})"
                f" + {f(a,'qA')} * ({f(b,'pB')} * {F3} + {f(b,'qB')} * {F4}))"
                f" * ({f(s,'r2')} * {f(a,'r1')} * {f(b,'r1')})")
    raise ValueError(case)


# Case ids of ldk_raw_hap (order is part of the C ABI).
RAW_CASES = ["dd1", "dd2", "dz_iii", "dz_iij", "dz_iji", "dz_ijj", "dz_ijk", "pi2_same",
             "pi2_iikk", "pi2_iikl", "pi2_ijkk", "pi2_alldiff", "pi2_triple", "pi2_ijij",
             "pi2_shared"]
RAW_ARITY = {"dd1": 1, "dd2": 2, "dz_iii": 1, "dz_iij": 2, "dz_iji": 2, "dz_ijj": 2, "dz_ijk": 3,
             "pi2_same": 1, "pi2_iikk": 2, "pi2_iikl": 3, "pi2_ijkk": 3, "pi2_alldiff": 4,
             "pi2_triple": 2, "pi2_ijij": 2, "pi2_shared": 3}


def emit_raw_dispatch():
    L = ["template <typename T>",
         "LDK_DEV T hap_raw_by_case(int case_id, const int* g, const HapFeat<T>* f) {",
         "    switch (case_id) {"]
    for cid, case in enumerate(RAW_CASES):
        args = tuple(f"g[{k}]" for k in range(RAW_ARITY[case]))
        expr = hap_call_expr(case, args)
        L.append(f"    case {cid}: return {_cexpr(expr)};  // {case}")
    L.append("    default: return T(0);")
    L.append("    }")
    L.append("}")
    return "\n".join(L)


def plan(P, geno=False):
    """(calls, stats): distinct canonical calls in first-use order and, per statistic,
    the list of (weight, call index)."""
    calls, index, stats = [], {}, []
    for name, cl in stat_specs(P):
        terms = {}
        for w, kind, p in cl:
            key = canonical(kind, p, geno)
            if key not in index:
                index[key] = len(calls)
                calls.append(key)
            terms[index[key]] = terms.get(index[key], 0.0) + w
        stats.append((name, sorted(terms.items())))
    return calls, stats


def hap_features_needed(P):
    calls, _ = plan(P)
    need = set()
    for case, _ in calls:
        need.update(HAP_CASE_FEATURES[case])
    # close over feature dependencies
    order = [n for n, _ in HAP_FEATURES]
    deps = {n: {d.split(".")[1].split()[0].rstrip(")") for d in e.replace("(", " ").split() if d.startswith("x.")}
            for n, e in HAP_FEATURES}
    changed = True
    while changed:
        changed = False
        for n in list(need):
            for d in deps.get(n, ()):
                if d in order and d not in need:
                    need.add(d)
                    changed = True
    return [n for n in order if n in need], sorted(r for r in need if r.startswith("r"))


# ---------------------------------------------------------------------------
# genotype path (moments order g1..g9 = n22, n21, n20, n12, n11, n10, n02, n01, n00)
# ---------------------------------------------------------------------------

# 16x the polynomial part of genotype DD(i,i) (genotype_kernels.py:43-68)
GENO_DD_POLY = (
    "(x.g2 * x.g4 - x.g2 * x.g2 * x.g4 + 4 * x.g3 * x.g4 - 4 * x.g2 * x.g3 * x.g4 - 4 * x.g3 * x.g3 * "
    "x.g4) + (-x.g2 * x.g4 * x.g4 - 4 * x.g3 * x.g4 * x.g4) + (x.g1 * x.g5 - x.g1 * x.g1 * x.g5 + "
    "x.g3 * x.g5 + 2 * x.g1 * x.g3 * x.g5 - x.g3 * x.g3 * x.g5 - 4 * x.g3 * x.g4 * x.g5 - x.g1 * x.g5 "
    "* x.g5 - x.g3 * x.g5 * x.g5) + (4 * x.g1 * x.g6 - 4 * x.g1 * x.g1 * x.g6 + x.g2 * x.g6 - 4 * "
    "x.g1 * x.g2 * x.g6 - x.g2 * x.g2 * x.g6 + 2 * x.g2 * x.g4 * x.g6 - 4 * x.g1 * x.g5 * x.g6 - 4 * "
    "x.g1 * x.g6 * x.g6 - x.g2 * x.g6 * x.g6) + (4 * x.g2 * x.g7 - 4 * x.g2 * x.g2 * x.g7 + 16 * x.g3 "
    "* x.g7 - 16 * x.g2 * x.g3 * x.g7 - 16 * x.g3 * x.g3 * x.g7 - 4 * x.g2 * x.g4 * x.g7 - 16 * x.g3 "
    "* x.g4 * x.g7 + x.g5 * x.g7 + 2 * x.g1 * x.g5 * x.g7 - 4 * x.g2 * x.g5 * x.g7 - 18 * x.g3 * x.g5 "
    "* x.g7 - x.g5 * x.g5 * x.g7 + 4 * x.g6 * x.g7 + 8 * x.g1 * x.g6 * x.g7 - 16 * x.g3 * x.g6 * x.g7 "
    "- 4 * x.g5 * x.g6 * x.g7 - 4 * x.g6 * x.g6 * x.g7 - 4 * x.g2 * x.g7 * x.g7 - 16 * x.g3 * x.g7 * "
    "x.g7 - x.g5 * x.g7 * x.g7 - 4 * x.g6 * x.g7 * x.g7) + (4 * x.g1 * x.g8 - 4 * x.g1 * x.g1 * x.g8 "
    "+ 4 * x.g3 * x.g8 + 8 * x.g1 * x.g3 * x.g8 - 4 * x.g3 * x.g3 * x.g8 + x.g4 * x.g8 - 4 * x.g1 * "
    "x.g4 * x.g8 + 2 * x.g2 * x.g4 * x.g8 - x.g4 * x.g4 * x.g8 - 4 * x.g1 * x.g5 * x.g8 - 4 * x.g3 * "
    "x.g5 * x.g8 + x.g6 * x.g8 + 2 * x.g2 * x.g6 * x.g8 - 4 * x.g3 * x.g6 * x.g8 + 2 * x.g4 * x.g6 * "
    "x.g8 - x.g6 * x.g6 * x.g8 - 16 * x.g3 * x.g7 * x.g8 - 4 * x.g6 * x.g7 * x.g8 - 4 * x.g1 * x.g8 * "
    "x.g8 - 4 * x.g3 * x.g8 * x.g8 - x.g4 * x.g8 * x.g8 - x.g6 * x.g8 * x.g8) + (16 * x.g1 * x.g9 - "
    "16 * x.g1 * x.g1 * x.g9 + 4 * x.g2 * x.g9 - 16 * x.g1 * x.g2 * x.g9 - 4 * x.g2 * x.g2 * x.g9 + 4 "
    "* x.g4 * x.g9 - 16 * x.g1 * x.g4 * x.g9 + 8 * x.g3 * x.g4 * x.g9 - 4 * x.g4 * x.g4 * x.g9 + x.g5 "
    "* x.g9 - 18 * x.g1 * x.g5 * x.g9 - 4 * x.g2 * x.g5 * x.g9 + 2 * x.g3 * x.g5 * x.g9 - 4 * x.g4 * "
    "x.g5 * x.g9 - x.g5 * x.g5 * x.g9 - 16 * x.g1 * x.g6 * x.g9 - 4 * x.g2 * x.g6 * x.g9 + 8 * x.g2 * "
    "x.g7 * x.g9 + 2 * x.g5 * x.g7 * x.g9 - 16 * x.g1 * x.g8 * x.g9 - 4 * x.g4 * x.g8 * x.g9 - 16 * "
    "x.g1 * x.g9 * x.g9 - 4 * x.g2 * x.g9 * x.g9 - 4 * x.g4 * x.g9 * x.g9 - x.g5 * x.g9 * x.g9) "
)

# quartic part of genotype Dz(i,i,i) (genotype_kernels.py:249-269)
GENO_DZ_QUARTIC = (
    "-(x.g2 * x.g4) + 3 * x.g1 * x.g2 * x.g4 + x.g2 * x.g2 * x.g4 + 2 * x.g3 * x.g4 + 4 * x.g1 * x.g3 "
    "* x.g4 - x.g2 * x.g3 * x.g4 - 4 * x.g3 * x.g3 * x.g4 + x.g2 * x.g4 * x.g4 + 2 * x.g3 * x.g4 * "
    "x.g4 + 2 * x.g1 * x.g5 - 3 * x.g1 * x.g1 * x.g5 - x.g1 * x.g2 * x.g5 + 2 * x.g3 * x.g5 + 2 * "
    "x.g1 * x.g3 * x.g5 - x.g2 * x.g3 * x.g5 - 3 * x.g3 * x.g3 * x.g5 - x.g1 * x.g4 * x.g5 + x.g3 * "
    "x.g4 * x.g5 + 2 * x.g1 * x.g6 - 4 * x.g1 * x.g1 * x.g6 - x.g2 * x.g6 - x.g1 * x.g2 * x.g6 + x.g2 "
    "* x.g2 * x.g6 + 4 * x.g1 * x.g3 * x.g6 + 3 * x.g2 * x.g3 * x.g6 - 2 * x.g1 * x.g4 * x.g6 - 2 * "
    "x.g2 * x.g4 * x.g6 - 2 * x.g3 * x.g4 * x.g6 + x.g1 * x.g5 * x.g6 - x.g3 * x.g5 * x.g6 + 2 * x.g1 "
    "* x.g6 * x.g6 + x.g2 * x.g6 * x.g6 + 2 * x.g2 * x.g7 + 4 * x.g1 * x.g2 * x.g7 + 2 * x.g2 * x.g2 "
    "* x.g7 + 8 * x.g3 * x.g7 + 4 * x.g1 * x.g3 * x.g7 - 4 * x.g3 * x.g3 * x.g7 - x.g2 * x.g4 * x.g7 "
    "+ 2 * x.g5 * x.g7 + 2 * x.g1 * x.g5 * x.g7 + x.g2 * x.g5 * x.g7 + 2 * x.g3 * x.g5 * x.g7 - x.g4 "
    "* x.g5 * x.g7 + 2 * x.g6 * x.g7 - x.g2 * x.g6 * x.g7 - 2 * x.g4 * x.g6 * x.g7 + x.g5 * x.g6 * "
    "x.g7 + 2 * x.g6 * x.g6 * x.g7 - 4 * x.g2 * x.g7 * x.g7 - 4 * x.g3 * x.g7 * x.g7 - 3 * x.g5 * "
    "x.g7 * x.g7 - 4 * x.g6 * x.g7 * x.g7 + 2 * x.g1 * x.g8 - 4 * x.g1 * x.g1 * x.g8 - 2 * x.g1 * "
    "x.g2 * x.g8 + 2 * x.g3 * x.g8 - 2 * x.g2 * x.g3 * x.g8 - 4 * x.g3 * x.g3 * x.g8 - x.g4 * x.g8 - "
    "x.g1 * x.g4 * x.g8 - 2 * x.g2 * x.g4 * x.g8 - x.g3 * x.g4 * x.g8 + x.g4 * x.g4 * x.g8 + x.g1 * "
    "x.g5 * x.g8 + x.g3 * x.g5 * x.g8 - x.g6 * x.g8 - x.g1 * x.g6 * x.g8 - 2 * x.g2 * x.g6 * x.g8 - "
    "x.g3 * x.g6 * x.g8 - 2 * x.g4 * x.g6 * x.g8 + x.g6 * x.g6 * x.g8 + 4 * x.g1 * x.g7 * x.g8 - 2 * "
    "x.g2 * x.g7 * x.g8 + 3 * x.g4 * x.g7 * x.g8 - x.g5 * x.g7 * x.g8 - x.g6 * x.g7 * x.g8 + 2 * x.g1 "
    "* x.g8 * x.g8 + 2 * x.g3 * x.g8 * x.g8 + x.g4 * x.g8 * x.g8 + x.g6 * x.g8 * x.g8 + 8 * x.g1 * "
    "x.g9 - 4 * x.g1 * x.g1 * x.g9 + 2 * x.g2 * x.g9 + 2 * x.g2 * x.g2 * x.g9 + 4 * x.g1 * x.g3 * "
    "x.g9 + 4 * x.g2 * x.g3 * x.g9 + 2 * x.g4 * x.g9 - x.g2 * x.g4 * x.g9 + 2 * x.g4 * x.g4 * x.g9 + "
    "2 * x.g5 * x.g9 + 2 * x.g1 * x.g5 * x.g9 + x.g2 * x.g5 * x.g9 + 2 * x.g3 * x.g5 * x.g9 + x.g4 * "
    "x.g5 * x.g9 - x.g2 * x.g6 * x.g9 - 2 * x.g4 * x.g6 * x.g9 - x.g5 * x.g6 * x.g9 + 4 * x.g1 * x.g7 "
    "* x.g9 + 4 * x.g3 * x.g7 * x.g9 + 4 * x.g4 * x.g7 * x.g9 + 2 * x.g5 * x.g7 * x.g9 + 4 * x.g6 * "
    "x.g7 * x.g9 - 2 * x.g2 * x.g8 * x.g9 + 4 * x.g3 * x.g8 * x.g9 - x.g4 * x.g8 * x.g9 - x.g5 * x.g8 "
    "* x.g9 + 3 * x.g6 * x.g8 * x.g9 - 4 * x.g1 * x.g9 * x.g9 - 4 * x.g2 * x.g9 * x.g9 - 4 * x.g4 * "
    "x.g9 * x.g9 - 3 * x.g5 * x.g9 * x.g9 "
)

# 16x the correction part of genotype pi2(i,i,i,i) (genotype_kernels.py:377-403)
GENO_PI2_CORR = (
    "(13 * x.g2 * x.g4 - 16 * x.g1 * x.g2 * x.g4 - 11 * x.g2 * x.g2 * x.g4 + 16 * x.g3 * x.g4 - 28 * "
    "x.g1 * x.g3 * x.g4 - 24 * x.g2 * x.g3 * x.g4) + (-8 * x.g3 * x.g3 * x.g4 - 11 * x.g2 * x.g4 * "
    "x.g4 - 20 * x.g3 * x.g4 * x.g4 - 6 * x.g5 + 12 * x.g1 * x.g5 - 4 * x.g1 * x.g1 * x.g5 + 17 * "
    "x.g2 * x.g5) + (-20 * x.g1 * x.g2 * x.g5 - 11 * x.g2 * x.g2 * x.g5 + 12 * x.g3 * x.g5 - 28 * "
    "x.g1 * x.g3 * x.g5 - 20 * x.g2 * x.g3 * x.g5 - 4 * x.g3 * x.g3 * x.g5) + (17 * x.g4 * x.g5 - 20 "
    "* x.g1 * x.g4 * x.g5 - 32 * x.g2 * x.g4 * x.g5 - 40 * x.g3 * x.g4 * x.g5 - 11 * x.g4 * x.g4 * "
    "x.g5 + 11 * x.g5 * x.g5) + (-16 * x.g1 * x.g5 * x.g5 - 17 * x.g2 * x.g5 * x.g5 - 16 * x.g3 * "
    "x.g5 * x.g5 - 17 * x.g4 * x.g5 * x.g5 - 6 * x.g5 * x.g5 * x.g5 + 16 * x.g1 * x.g6 - 8 * x.g1 * "
    "x.g1 * x.g6) + (13 * x.g2 * x.g6 - 24 * x.g1 * x.g2 * x.g6 - 11 * x.g2 * x.g2 * x.g6 - 28 * x.g1 "
    "* x.g3 * x.g6 - 16 * x.g2 * x.g3 * x.g6 + 24 * x.g4 * x.g6) + (-36 * x.g1 * x.g4 * x.g6 - 38 * "
    "x.g2 * x.g4 * x.g6 - 36 * x.g3 * x.g4 * x.g6 - 20 * x.g4 * x.g4 * x.g6 + 17 * x.g5 * x.g6 - 40 * "
    "x.g1 * x.g5 * x.g6) + (-32 * x.g2 * x.g5 * x.g6 - 20 * x.g3 * x.g5 * x.g6 - 42 * x.g4 * x.g5 * "
    "x.g6 - 17 * x.g5 * x.g5 * x.g6 - 20 * x.g1 * x.g6 * x.g6 - 11 * x.g2 * x.g6 * x.g6) + (-20 * "
    "x.g4 * x.g6 * x.g6 - 11 * x.g5 * x.g6 * x.g6 + 16 * x.g2 * x.g7 - 28 * x.g1 * x.g2 * x.g7 - 20 * "
    "x.g2 * x.g2 * x.g7 + 16 * x.g3 * x.g7) + (-48 * x.g1 * x.g3 * x.g7 - 44 * x.g2 * x.g3 * x.g7 - "
    "16 * x.g3 * x.g3 * x.g7 - 24 * x.g2 * x.g4 * x.g7 - 44 * x.g3 * x.g4 * x.g7) + (12 * x.g5 * x.g7 "
    "- 28 * x.g1 * x.g5 * x.g7 - 40 * x.g2 * x.g5 * x.g7 - 48 * x.g3 * x.g5 * x.g7 - 20 * x.g4 * x.g5 "
    "* x.g7 - 16 * x.g5 * x.g5 * x.g7) + (16 * x.g6 * x.g7 - 48 * x.g1 * x.g6 * x.g7 - 48 * x.g2 * "
    "x.g6 * x.g7 - 44 * x.g3 * x.g6 * x.g7 - 36 * x.g4 * x.g6 * x.g7 - 40 * x.g5 * x.g6 * x.g7) + "
    "(-20 * x.g6 * x.g6 * x.g7 - 8 * x.g2 * x.g7 * x.g7 - 16 * x.g3 * x.g7 * x.g7 - 4 * x.g5 * x.g7 * "
    "x.g7 - 8 * x.g6 * x.g7 * x.g7 + 16 * x.g1 * x.g8 - 8 * x.g1 * x.g1 * x.g8) + (24 * x.g2 * x.g8 - "
    "36 * x.g1 * x.g2 * x.g8 - 20 * x.g2 * x.g2 * x.g8 + 16 * x.g3 * x.g8 - 48 * x.g1 * x.g3 * x.g8 - "
    "36 * x.g2 * x.g3 * x.g8 - 8 * x.g3 * x.g3 * x.g8) + (13 * x.g4 * x.g8 - 24 * x.g1 * x.g4 * x.g8 "
    "- 38 * x.g2 * x.g4 * x.g8 - 48 * x.g3 * x.g4 * x.g8 - 11 * x.g4 * x.g4 * x.g8 + 17 * x.g5 * x.g8 "
    "- 40 * x.g1 * x.g5 * x.g8) + (-42 * x.g2 * x.g5 * x.g8 - 40 * x.g3 * x.g5 * x.g8 - 32 * x.g4 * "
    "x.g5 * x.g8 - 17 * x.g5 * x.g5 * x.g8 + 13 * x.g6 * x.g8 - 48 * x.g1 * x.g6 * x.g8) + (-38 * "
    "x.g2 * x.g6 * x.g8 - 24 * x.g3 * x.g6 * x.g8 - 38 * x.g4 * x.g6 * x.g8 - 32 * x.g5 * x.g6 * x.g8 "
    "- 11 * x.g6 * x.g6 * x.g8 - 28 * x.g1 * x.g7 * x.g8) + (-36 * x.g2 * x.g7 * x.g8 - 44 * x.g3 * "
    "x.g7 * x.g8 - 16 * x.g4 * x.g7 * x.g8 - 20 * x.g5 * x.g7 * x.g8 - 24 * x.g6 * x.g7 * x.g8 - 20 * "
    "x.g1 * x.g8 * x.g8) + (-20 * x.g2 * x.g8 * x.g8 - 20 * x.g3 * x.g8 * x.g8 - 11 * x.g4 * x.g8 * "
    "x.g8 - 11 * x.g5 * x.g8 * x.g8 - 11 * x.g6 * x.g8 * x.g8 + 16 * x.g1 * x.g9 - 16 * x.g1 * x.g1 * "
    "x.g9) + (16 * x.g2 * x.g9 - 44 * x.g1 * x.g2 * x.g9 - 20 * x.g2 * x.g2 * x.g9 - 48 * x.g1 * x.g3 "
    "* x.g9 - 28 * x.g2 * x.g3 * x.g9 + 16 * x.g4 * x.g9) + (-44 * x.g1 * x.g4 * x.g9 - 48 * x.g2 * "
    "x.g4 * x.g9 - 48 * x.g3 * x.g4 * x.g9 - 20 * x.g4 * x.g4 * x.g9 + 12 * x.g5 * x.g9 - 48 * x.g1 * "
    "x.g5 * x.g9) + (-40 * x.g2 * x.g5 * x.g9 - 28 * x.g3 * x.g5 * x.g9 - 40 * x.g4 * x.g5 * x.g9 - "
    "16 * x.g5 * x.g5 * x.g9 - 44 * x.g1 * x.g6 * x.g9 - 24 * x.g2 * x.g6 * x.g9) + (-36 * x.g4 * "
    "x.g6 * x.g9 - 20 * x.g5 * x.g6 * x.g9 - 48 * x.g1 * x.g7 * x.g9 - 48 * x.g2 * x.g7 * x.g9 - 48 * "
    "x.g3 * x.g7 * x.g9 - 28 * x.g4 * x.g7 * x.g9) + (-28 * x.g5 * x.g7 * x.g9 - 28 * x.g6 * x.g7 * "
    "x.g9 - 44 * x.g1 * x.g8 * x.g9 - 36 * x.g2 * x.g8 * x.g9 - 28 * x.g3 * x.g8 * x.g9 - 24 * x.g4 * "
    "x.g8 * x.g9) + (-20 * x.g5 * x.g8 * x.g9 - 16 * x.g6 * x.g8 * x.g9 - 16 * x.g1 * x.g9 * x.g9 - 8 "
    "* x.g2 * x.g9 * x.g9 - 8 * x.g4 * x.g9 * x.g9 - 4 * x.g5 * x.g9 * x.g9) "
)

# Per-population genotype features (pg_gpu genotype_kernels.py:412-492 and :176-197).
# x.ns = sum of the nine counts, x.n = n_valid (equal on the genotype path).
GENO_FEATURES = [
    ("xAB", "x.g1 + 0.5 * x.g2 + 0.5 * x.g4 + 0.25 * x.g5"),
    ("xAb", "0.5 * x.g2 + x.g3 + 0.25 * x.g5 + 0.5 * x.g6"),
    ("xaB", "0.5 * x.g4 + 0.25 * x.g5 + x.g7 + 0.5 * x.g8"),
    ("xab", "0.25 * x.g5 + 0.5 * x.g6 + 0.5 * x.g8 + x.g9"),
    ("D", "x.xAB * x.xab - x.xAb * x.xaB"),
    ("pA", "x.g1 + x.g2 + x.g3 + 0.5 * (x.g4 + x.g5 + x.g6)"),
    ("qA", "0.5 * (x.g4 + x.g5 + x.g6) + x.g7 + x.g8 + x.g9"),
    ("pB", "x.g1 + 0.5 * x.g2 + x.g4 + 0.5 * x.g5 + x.g7 + 0.5 * x.g8"),
    ("qB", "0.5 * x.g2 + x.g3 + 0.5 * x.g5 + x.g6 + 0.5 * x.g8 + x.g9"),
    ("BL", "(4 * x.pA * x.qA - (x.g4 + x.g5 + x.g6)) * x.inn1"),
    ("BR", "(4 * x.pB * x.qB - (x.g2 + x.g5 + x.g8)) * x.inn1"),
    ("C00", "(x.pA * x.pB - x.xAB) * x.inn1"),
    ("C01", "(x.pA * x.qB - x.xAb) * x.inn1"),
    ("C10", "(x.qA * x.pB - x.xaB) * x.inn1"),
    ("C11", "(x.qA * x.qB - x.xab) * x.inn1"),
    ("Bsgn", "x.xAB - x.xAb - x.xaB + x.xab"),
    ("p", "x.pA * x.invn"),
    ("r", "x.qA * x.invn"),
    ("q", "x.pB * x.invn"),
    ("s", "x.qB * x.invn"),
    ("L0", "x.g5 + 2 * x.g6 + 2 * x.g8 + 4 * x.g9"),
    ("AQ3", "-(x.qB * (3 * x.g4 + 3 * x.g5 + 3 * x.g6 + 4 * x.g7 + 4 * x.g8 + 4 * x.g9)) / 8"
            " + x.pA * x.qB * x.qA / 2 + (x.qA * x.L0) / 8 + (x.g5 + 2 * x.g6) / 8 - (x.pA * x.L0) / 8"),
    ("AS3", "-(x.pB * (5 * x.g4 + 5 * x.g5 + 5 * x.g6 + 8 * x.g7 + 8 * x.g8 + 8 * x.g9)) / 8"
            " + x.pA * x.pB * x.qA / 2"
            " + (x.qA * (-2 * x.g2 - 4 * x.g3 + 4 * x.g4 + x.g5 - 2 * x.g6 + 8 * x.g7 + 4 * x.g8 + 4)) / 8"
            " + (-x.g5 - 2 * x.g6 - 4 * x.g7 - 4 * x.g8 - 4 * x.g9) / 8 + (x.pA * x.L0) / 8"),
    ("BP3", "-(x.qA * (3 * x.g2 + 4 * x.g3 + 3 * x.g5 + 4 * x.g6 + 3 * x.g8 + 4 * x.g9)) / 8"
            " + x.pB * x.qB * x.qA / 2 + (x.qB * x.L0) / 8 + (x.g5 + 2 * x.g8) / 8 - (x.pB * x.L0) / 8"),
    ("BR3", "-(x.pA * (5 * x.g2 + 8 * x.g3 + 5 * x.g5 + 8 * x.g6 + 5 * x.g8 + 8 * x.g9)) / 8"
            " + x.pA * x.pB * x.qB / 2"
            " + (x.qB * (4 * x.g2 + 8 * x.g3 - 2 * x.g4 + x.g5 + 4 * x.g6 - 4 * x.g7 - 2 * x.g8 + 4)) / 8"
            " + (-4 * x.g3 - x.g5 - 4 * x.g6 - 2 * x.g8 - 4 * x.g9) / 8 + (x.pB * x.L0) / 8"),
    ("A", "-x.g1 + x.g3 - x.g4 + x.g6 - x.g7 + x.g9"),
    ("Bv", "-x.g1 - x.g2 - x.g3 + x.g7 + x.g8 + x.g9"),
    ("Wjj", "(-x.g1 + x.g3 + x.g7 - x.g9) + x.A * x.Bv"),
    ("U", "x.D * (1 + x.Bv) + 0.25 * (2 * x.g2 * x.g7 + 4 * x.g3 * x.g7 + 2 * x.g5 * x.g7"
          " + 4 * x.g6 * x.g7 - 2 * x.g1 * x.g8 + 2 * x.g3 * x.g8 - 2 * x.g4 * x.g8 + 2 * x.g6 * x.g8"
          " - 4 * x.g1 * x.g9 - 2 * x.g2 * x.g9 - 4 * x.g4 * x.g9 - 2 * x.g5 * x.g9)"),
    ("V", "x.D * (1 + x.A) + 0.25 * (2 * x.g3 * x.g4 + 2 * x.g3 * x.g5 - 2 * x.g1 * x.g6"
          " - 2 * x.g2 * x.g6 + 4 * x.g3 * x.g7 + 2 * x.g6 * x.g7 + 4 * x.g3 * x.g8 + 2 * x.g6 * x.g8"
          " - 4 * x.g1 * x.g9 - 4 * x.g2 * x.g9 - 2 * x.g4 * x.g9 - 2 * x.g5 * x.g9)"),
    # single-population statistics, numerators over ns(ns-1)(ns-2)(ns-3) (zero if ns < 4)
    ("DD1", "4 * ((" + GENO_DD_POLY + ") * 0.0625 + x.D * x.D) * x.w4"),
    ("DZ1", "2 * (0.25 * (" + GENO_DZ_QUARTIC + ") + x.A * x.Bv * x.D) * x.w4"),
    ("PI1", "(x.pA * x.pB * x.qB * x.qA + (" + GENO_PI2_CORR + ") * 0.0625) * x.w4"),
]


# The three single-population polynomials, as pg_gpu writes them, are sums of up to 155
# integer-coefficient monomials of degree <= 3 in the nine cell counts (~950 FP64 instructions
# per population and pair with a*b + c fused).  The generated code evaluates them in
# multivariate Horner form over g1, ..., g9 instead (~400): with integer counts every
# intermediate of either form is an integer, so FP64 gives the same value exactly while the
# intermediates stay below 2^53 (more than 10^4 individuals per population before that can
# fail; the expanded form has the same limit).  check() proves each Horner form equal to its
# polynomial.
_HORNER_POLYS = {"GENO_DD_POLY": GENO_DD_POLY, "GENO_DZ_QUARTIC": GENO_DZ_QUARTIC, "GENO_PI2_CORR": GENO_PI2_CORR}


def _horner_sympy(poly):
    import sympy as sp
    from sympy.polys.polyfuncs import horner
    g = sp.symbols("g1:10")
    loc = {f"g{i + 1}": g[i] for i in range(9)}
    e = sp.expand(sp.sympify(poly.replace("x.g", "g"), locals=loc))
    return e, horner(e, *g), g


@functools.lru_cache(maxsize=None)
def horner_form(poly):
    """``poly`` (a polynomial string in x.g1 .. x.g9) in multivariate Horner form, as an
    expression string in the same variables (C and Python syntax)."""
    import re
    _, h, _ = _horner_sympy(poly)
    out = re.sub(r"\bg(\d)\b", r"x.g\1", str(h))
    if "**" in out:
        raise ValueError("power left in a Horner form")
    return out


@functools.lru_cache(maxsize=None)
def geno_features():
    """GENO_FEATURES with the three single-population polynomials in Horner form (the form
    the generated code and the NumPy evaluation use)."""
    out = []
    for n, e in GENO_FEATURES:
        for poly in _HORNER_POLYS.values():
            e = e.replace("(" + poly + ")", "(" + horner_form(poly) + ")")
        out.append((n, e))
    for n in ("DD1", "DZ1", "PI1"):
        e = dict(out)[n]
        if any(poly in e for poly in _HORNER_POLYS.values()):
            raise ValueError(f"{n}: polynomial not replaced")
    return out


def geno_call_expr(case, args):
    """Expression of one canonical raw genotype call (genotype_kernels.py:27-405)."""
    f = lambda p, name: f"f[{p}].{name}"  # noqa: E731
    if case == "dd1":
        return f(args[0], "DD1")
    if case == "dd2":
        i, j = args
        return f"4 * ({f(i,'D')} * {f(j,'D')}) * ({f(i,'r2')} * {f(j,'r2')})"
    if case == "dz_iii":
        return f(args[0], "DZ1")
    if case == "dz_iij":
        i, j = args
        return f"(2 * {f(i,'U')} * {f(j,'A')}) * ({f(i,'u3')} * {f(j,'u1')})"
    if case == "dz_iji":
        i, j = args
        return f"(2 * {f(i,'V')} * {f(j,'Bv')}) * ({f(i,'u3')} * {f(j,'u1')})"
    if case == "dz_ijj":
        i, j = args
        return f"(2 * {f(i,'D')} * {f(j,'Wjj')}) * ({f(j,'u2')} * {f(i,'u2')})"
    if case == "dz_ijk":
        i, j, k = args
        return f"(2 * {f(i,'D')} * {f(j,'Bv')} * {f(k,'A')}) * ({f(i,'u2')} * {f(j,'u1')} * {f(k,'u1')})"
    if case == "pi2_same":
        return f(args[0], "PI1")
    if case == "pi2_alldiff":
        i, j, k, l = args
        return (f"0.25 * ({f(i,'p')} * {f(j,'r')} + {f(i,'r')} * {f(j,'p')})"
                f" * ({f(k,'q')} * {f(l,'s')} + {f(k,'s')} * {f(l,'q')})")
    if case == "pi2_iikk":
        i, k = args
        return f"{f(i,'BL')} * {f(k,'BR')}"
    if case == "pi2_iikl":
        i, k, l = args
        return f"{f(i,'BL')} * 0.5 * ({f(k,'q')} * {f(l,'s')} + {f(k,'s')} * {f(l,'q')})"
    if case == "pi2_ijkk":
        i, j, k = args
        return f"0.5 * ({f(i,'p')} * {f(j,'r')} + {f(i,'r')} * {f(j,'p')}) * {f(k,'BR')}"
    if case == "pi2_shared":
        s, a, b = args
        return (f"{f(a,'r')} * ({f(s,'C00')} * {f(b,'s')} + {f(s,'C01')} * {f(b,'q')})"
                f" + {f(a,'p')} * ({f(s,'C10')} * {f(b,'s')} + {f(s,'C11')} * {f(b,'q')})")
    if case == "pi2_iiij":
        t, s = args
        return (f"({f(t,'AQ3')} * {f(s,'pB')} + {f(t,'AS3')} * {f(s,'qB')})"
                f" * ({f(t,'r3')} * {f(s,'r1')})")
    if case == "pi2_ijii":
        t, s = args
        return (f"({f(t,'BP3')} * {f(s,'pA')} + {f(t,'BR3')} * {f(s,'qA')})"
                f" * ({f(t,'r3')} * {f(s,'r1')})")
    if case == "pi2_ijij":
        i, j = args
        P_i, Q_i, R_i, S_i = f(i, "pA"), f(i, "pB"), f(i, "qA"), f(i, "qB")
        P_j, Q_j, R_j, S_j = f(j, "pA"), f(j, "pB"), f(j, "qA"), f(j, "qB")
        X01i, X10i, X11i, Bi = f(i, "xAb"), f(i, "xaB"), f(i, "xab"), f(i, "Bsgn")
        X11j, X01j, Bj = f(j, "xab"), f(j, "xAb"), f(j, "Bsgn")
        num = (f"-0.25 * ({R_i} * {S_i}) * {Q_j} - 0.25 * {X11i} * ({P_j} * {Q_j})"
               f" + 0.25 * ({R_i} * {S_i}) * ({P_j} * {Q_j}) - 0.25 * {R_i} * ({P_j} * {S_j})"
               f" - 0.25 * ({P_i} * {Q_i}) * {X11j} - 0.25 * ({R_i} * {S_i}) * {X11j}"
               f" + 0.25 * ({P_i} * {S_i}) * {X11j} + 0.25 * ({Q_i} * {R_i}) * {X11j}"
               f" - 0.25 * ({P_i} * {R_i}) * {S_j} + 0.25 * ({R_i} * (1 + {X01i} - {X10i})) * {S_j}"
               f" + 0.25 * {X11i} * ({P_j} * {S_j}) + 0.25 * ({Q_i} * {R_i}) * ({P_j} * {S_j})"
               f" + 0.25 * ({S_i} * (1 + {R_i})) * {R_j} - 0.25 * {X01i} * ({Q_j} * {R_j})"
               f" + 0.25 * ({P_i} * {S_i}) * ({Q_j} * {R_j})"
               f" - 0.25 * ({P_i} * {S_i}) * {R_j} - 0.25 * {P_i} * ({R_j} * {S_j})"
               f" + 0.25 * {X01i} * ({R_j} * {S_j}) + 0.25 * ({P_i} * {Q_i}) * ({R_j} * {S_j})"
               f" + 0.25 * {X11i} * {Bj} + 0.25 * {Bi} * {X11j} - {X11i} * {X11j}")
        _ = X01j
        return f"({num}) * ({f(i,'r2')} * {f(j,'r2')})"
    raise ValueError(case)


def geno_features_needed(P):
    calls, _ = plan(P, geno=True)
    need = {"DD1", "DZ1", "PI1"}
    per_case = {
        "dd2": ["D"], "dz_iij": ["U", "A"], "dz_iji": ["V", "Bv"], "dz_ijj": ["D", "Wjj"],
        "dz_ijk": ["D", "Bv", "A"], "pi2_alldiff": ["p", "r", "q", "s"], "pi2_iikk": ["BL", "BR"],
        "pi2_iikl": ["BL", "q", "s"], "pi2_ijkk": ["p", "r", "BR"],
        "pi2_shared": ["r", "p", "s", "q", "C00", "C01", "C10", "C11"],
        "pi2_iiij": ["AQ3", "AS3", "pB", "qB"], "pi2_ijii": ["BP3", "BR3", "pA", "qA"],
        "pi2_ijij": ["pA", "pB", "qA", "qB", "xAb", "xaB", "xab", "Bsgn"],
    }
    for case, _ in calls:
        need.update(per_case.get(case, []))
    order = [n for n, _ in GENO_FEATURES]
    changed = True
    while changed:
        changed = False
        for n, e in GENO_FEATURES:
            if n in need:
                for d in order:
                    if f"x.{d}" in e.replace("x.g", "x.#") and d not in need:
                        need.add(d)
                        changed = True
    return [n for n in order if n in need]


def emit_geno(P):
    feats = geno_features_needed(P)
    calls, stats = plan(P, geno=True)
    L = [f"// genotype path, P = {P}: {len(stats)} statistics from {len(calls)} distinct raw calls",
         "// (PREP false: the reciprocals are already set, e.g. by geno_prepare_from)",
         "template <typename T, bool PREP = true>", f"LDK_DEV void geno_features_P{P}(GenoFeat<T>& x) {{",
         "    if constexpr (PREP) geno_prepare(x);"]
    for n, e in geno_features():
        if n in feats:
            L.append(f"    x.{n} = {_cexpr(e)};")
    L.append("}")
    L.append("template <typename T, int S = 1>")
    L.append(f"LDK_DEV void geno_stats_P{P}(const GenoFeat<T>* f, T* acc) {{")
    for ci, (case, args) in enumerate(calls):
        L.append(f"    const T v{ci} = {_cexpr(geno_call_expr(case, args))};  // {case}{args}")
    for si, (name, terms) in enumerate(stats):
        groups = {}
        for idx, w in terms:
            groups.setdefault(w, []).append(f"v{idx}")
        parts = []
        for w, vs in sorted(groups.items(), reverse=True):
            sw = _fmt_weight(w)
            body = " + ".join(vs)
            parts.append(body if sw is None else f"T({sw}) * ({body})")
        L.append(f"    acc[{si} * S] += {' + '.join(parts)};  // {name}")
    L.append("}")
    return "\n".join(L)


def numpy_geno_stats(counts9_list, n_list=None):
    """Evaluate the generated genotype expressions with NumPy float64 (test helper)."""
    import numpy as np
    P = len(counts9_list)
    fs = []
    for p, c in enumerate(counts9_list):
        c = np.asarray(c, dtype=np.float64)
        x = _NS()
        for m in range(9):
            setattr(x, f"g{m + 1}", c[:, 8 - m])
        x.ns = c.sum(axis=1)
        x.n = x.ns if (n_list is None or n_list[p] is None) else np.asarray(n_list[p], np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            n, ns = x.n, x.ns
            x.inn1 = 1.0 / np.maximum(4 * n * (n - 1), 1)
            x.invn = 1.0 / n
            d1, d2 = n, n * (n - 1)
            d3 = d2 * (n - 2)
            x.r1 = np.where(d1 > 0, 1 / np.where(d1 > 0, d1, 1), 0.0)
            x.r2 = np.where(d2 > 0, 1 / np.where(d2 > 0, d2, 1), 0.0)
            x.r3 = np.where(d3 > 0, 1 / np.where(d3 > 0, d3, 1), 0.0)
            x.u1 = 1.0 / ns
            x.u2 = 1.0 / (ns * (ns - 1))
            x.u3 = 1.0 / (ns * (ns - 1) * (ns - 2))
            w4 = ns * (ns - 1) * (ns - 2) * (ns - 3)
            x.w4 = np.where(ns >= 4, 1 / np.where(ns >= 4, w4, 1), 0.0)
            for name, e in geno_features():
                setattr(x, name, eval(e, {}, {"x": x}))
        fs.append(x)
    calls, stats = plan(P, geno=True)
    with np.errstate(divide="ignore", invalid="ignore"):
        vals = [eval(geno_call_expr(case, args), {}, {"f": fs}) for case, args in calls]
    out = np.zeros((len(fs[0].g1), len(stats)))
    for si, (_, terms) in enumerate(stats):
        for idx, w in terms:
            out[:, si] += w * vals[idx]
    return out

# ---------------------------------------------------------------------------
# code emission
# ---------------------------------------------------------------------------


def _fmt_weight(w):
    return {1.0: None, 0.5: "0.5", 0.25: "0.25", 0.125: "0.125", 0.75: "0.75"}.get(w, repr(w))


def emit_hap(P):
    feats, recips = hap_features_needed(P)
    calls, stats = plan(P)
    L = []
    L.append(f"// P = {P}: {len(stats)} statistics from {len(calls)} distinct raw calls")
    L.append("template <typename T>")
    L.append(f"LDK_DEV void hap_features_P{P}(HapFeat<T>& x) {{")
    for n, e in HAP_FEATURES:
        if n in feats:
            L.append(f"    x.{n} = {_cexpr(e)};")
    L.append("}")
    L.append("template <typename T, int S = 1>")
    L.append(f"LDK_DEV void hap_stats_P{P}(const HapFeat<T>* f, T* acc) {{")
    for ci, (case, args) in enumerate(calls):
        L.append(f"    const T v{ci} = {_cexpr(hap_call_expr(case, args))};  // {case}{args}")
    for si, (name, terms) in enumerate(stats):
        groups = {}
        for idx, w in terms:
            groups.setdefault(w, []).append(f"v{idx}")
        parts = []
        for w, vs in sorted(groups.items(), reverse=True):
            sw = _fmt_weight(w)
            body = " + ".join(vs)
            parts.append(body if sw is None else f"T({sw}) * ({body})")
        L.append(f"    acc[{si} * S] += {' + '.join(parts)};  // {name}")
    L.append("}")
    return "\n".join(L)


# ---------------------------------------------------------------------------
# fused-path forms (tensor-core parse)
# ---------------------------------------------------------------------------
#
# Statistic-level expressions over per-population *scaled* features (numerator factors
# times their reciprocal denominators), written as one accumulate per product term so
# that every term is a single FMA into its sum.  Every raw call's numerator is an
# integer polynomial of the counts, exact in FP64 below 2^53, so regrouping it changes
# only the final roundings.  Two identities shorten the pi2 cases:
#   L_k = c_{5-k} ns - sigma_k E  (sigma = +1, -1, -1, +1), hence
#   F_k = L_k - c_{5-k} = c_{5-k} (ns - 1) - sigma_k E, and the pi2(i,j,i,j) correction
#   sum_k (Q_k^i c_{5-k}^j - c_k^i L_k^j) = X (1 - ns_i - ns_j) - (E_i s_j + E_j s_i),
#   X = sum_k c_{5-k}^i c_k^j, symmetric in (i, j): pi2_ijij(i, j) = pi2_ijij(j, i).
# ``check()`` verifies both symbolically.

# (name, expression): x = f[p] (HapFeat), g = this population's scaled features
FUSED_SCALED = [
    ("Er2", "x.E * x.r2"),
    ("Er2h", "0.5 * g.Er2"),
    ("Er3h", "x.E * (0.5 * x.r3)"),
    ("aEr3h", "x.a * g.Er3h"),
    ("bEr3h", "x.b * g.Er3h"),
    ("ar1", "x.a * x.r1"),
    ("br1", "x.b * x.r1"),
    ("Sr2", "(x.s + x.a * x.b) * x.r2"),
    ("r3h", "0.5 * x.r3"),
    ("T1r3h", "x.T1 * g.r3h"),
    ("T2r3h", "x.T2 * g.r3h"),
    ("pAr1", "x.pA * x.r1"),
    ("qAr1", "x.qA * x.r1"),
    ("pBr1", "x.pB * x.r1"),
    ("qBr1", "x.qB * x.r1"),
    ("r2h", "0.5 * x.r2"),
    ("fAr2h", "x.fA * g.r2h"),
    ("fBr2", "x.fB * x.r2"),
    ("r2q", "0.25 * x.r2"),
    ("fAr2q", "x.fA * g.r2q"),
    ("fBr2q", "x.fB * g.r2q"),
    ("r2e", "0.125 * x.r2"),
    ("m1", "x.ns - 1"),
    ("F1h", "(x.c4 * g.m1 - x.E) * g.r2e"),
    ("F2h", "(x.c3 * g.m1 + x.E) * g.r2e"),
    ("F3h", "(x.c2 * g.m1 + x.E) * g.r2e"),
    ("F4h", "(x.c1 * g.m1 - x.E) * g.r2e"),
]

# features of HapFeat the fused forms read directly
FUSED_BASE = ["c1", "c2", "c3", "c4", "ns", "pA", "qA", "pB", "qB", "E", "a", "b", "s", "fA", "fB",
              "T1", "T2", "DDs", "DZs", "PIs"]


def fused_plan(P):
    """Per statistic, the list of (weight, case, args) with pi2_ijij merged over its
    two argument orders."""
    out = []
    for name, cl in stat_specs(P):
        terms = {}
        for w, kind, p in cl:
            case, args = canonical(kind, p)
            if case == "pi2_ijij":
                args = tuple(sorted(args))
            terms[(case, args)] = terms.get((case, args), 0.0) + w
        out.append((name, [(w, c, a) for (c, a), w in terms.items()]))
    return out


def fused_terms(case, args, w):
    """Product terms (A, B) whose sum is w * call(case, args); A and B use f[p].name for
    HapFeat fields and g{p}_name for scaled features."""
    g = lambda p, n: f"g{p}_{n}"  # noqa: E731
    f = lambda p, n: f"f[{p}].{n}"  # noqa: E731
    need = {"dd1": 1.0, "dd2": 1.0, "dz_iii": 1.0, "dz_iij": 0.5, "dz_iji": 0.5, "dz_ijj": 1.0,
            "dz_ijk": 0.5, "pi2_same": 1.0, "pi2_triple": 1.0, "pi2_iikk": 0.5, "pi2_iikl": 0.5,
            "pi2_ijkk": 0.5, "pi2_alldiff": 0.5, "pi2_ijij": 1.0, "pi2_shared": 0.5}[case]
    if w != need:
        raise ValueError(f"weight {w} of {case}{args}: fused form assumes {need}")
    if case == "dd1":
        (i,) = args
        return [(f(i, "DDs"), f(i, "r4"))]
    if case == "dd2":
        i, j = args
        return [(g(i, "Er2"), g(j, "Er2"))]
    if case == "dz_iii":
        (i,) = args
        return [(f(i, "DZs"), f(i, "r4"))]
    if case == "dz_iij":
        i, j = args
        return [(g(i, "aEr3h"), g(j, "br1"))]
    if case == "dz_iji":
        i, j = args
        return [(g(i, "bEr3h"), g(j, "ar1"))]
    if case == "dz_ijj":
        i, j = args
        return [(g(i, "Er2"), g(j, "Sr2"))]
    if case == "dz_ijk":
        i, j, k = args
        return [(g(i, "Er2h"), f"({g(j, 'ar1')} * {g(k, 'br1')})")]
    if case == "pi2_same":
        (i,) = args
        return [(f(i, "PIs"), f(i, "r4"))]
    if case == "pi2_triple":
        t, s_ = args
        return [(g(t, "T1r3h"), g(s_, "pBr1")), (g(t, "T2r3h"), g(s_, "qBr1"))]
    if case == "pi2_iikk":
        i, k = args
        return [(g(i, "fAr2h"), g(k, "fBr2"))]
    if case == "pi2_iikl":
        i, k, l = args
        return [(g(i, "fAr2q"), f"({g(k, 'pBr1')} * {g(l, 'qBr1')} + {g(k, 'qBr1')} * {g(l, 'pBr1')})")]
    if case == "pi2_ijkk":
        i, j, k = args
        return [(g(k, "fBr2q"), f"({g(i, 'pAr1')} * {g(j, 'qAr1')} + {g(i, 'qAr1')} * {g(j, 'pAr1')})")]
    if case == "pi2_alldiff":
        i, j, k, l = args
        return [(f"(0.125 * ({g(i, 'pAr1')} * {g(j, 'qAr1')} + {g(i, 'qAr1')} * {g(j, 'pAr1')}))",
                 f"({g(k, 'pBr1')} * {g(l, 'qBr1')} + {g(k, 'qBr1')} * {g(l, 'pBr1')})")]
    if case == "pi2_shared":
        s_, a, b = args
        return [(g(a, "pAr1"), f"({g(b, 'pBr1')} * {g(s_, 'F1h')} + {g(b, 'qBr1')} * {g(s_, 'F2h')})"),
                (g(a, "qAr1"), f"({g(b, 'pBr1')} * {g(s_, 'F3h')} + {g(b, 'qBr1')} * {g(s_, 'F4h')})")]
    if case == "pi2_ijij":
        i, j = args
        HA = f"({f(i, 'pA')} * {f(j, 'qA')} + {f(i, 'qA')} * {f(j, 'pA')})"
        HB = f"({f(i, 'pB')} * {f(j, 'qB')} + {f(i, 'qB')} * {f(j, 'pB')})"
        X = (f"({f(i, 'c4')} * {f(j, 'c1')} + {f(i, 'c3')} * {f(j, 'c2')} + {f(i, 'c2')} * {f(j, 'c3')}"
             f" + {f(i, 'c1')} * {f(j, 'c4')})")
        body = (f"({HA} * {HB} + {X} * (1 - {f(i, 'ns')} - {f(j, 'ns')})"
                f" - ({f(i, 'E')} * {f(j, 's')} + {f(j, 'E')} * {f(i, 's')}))")
        return [(f"({g(i, 'r2h')} * {g(j, 'r2h')})", body)]
    raise ValueError(case)


def _term_cost(A, B):
    return 1 + sum(t.count("*") + t.count(" + ") + t.count(" - ") for t in (A, B))


# Four populations: the split the tensor-core kernel uses to divide the 105 statistics
# between the two epilogue warps of a TMEM lane quarter, set by register pressure rather than
# cost.  Measured (4 populations of 100-160 haplotypes, 16 bins): the cost-balanced point
# (72) leaves one warp 72 accumulators and spills ~1.1 KB per thread, 4.1e9 pairs/s; 56
# spills ~0.5 KB, 7.9e9 pairs/s; 60: 7.4e9.
FUSED_SPLIT_AT = {4: 56}


def fused_split(P):
    """Split point K of the statistics into two contiguous halves: of about equal cost, or
    FUSED_SPLIT_AT[P]."""
    if P in FUSED_SPLIT_AT:
        return FUSED_SPLIT_AT[P]
    costs = [sum(_term_cost(A, B) for w, c, a in terms for A, B in fused_terms(c, a, w))
             for _, terms in fused_plan(P)]
    tot, run, best = sum(costs), 0, (None, 0)
    for k in range(1, len(costs)):
        run += costs[k - 1]
        d = abs(2 * run - tot)
        if best[0] is None or d < best[0]:
            best = (d, k)
    return best[1]


def _scaled_closure(used):
    """(p, name) scaled features needed by the used set, in definition order."""
    defs = dict(FUSED_SCALED)
    import re
    need = set(used)
    changed = True
    while changed:
        changed = False
        for p, n in list(need):
            for dep in re.findall(r"g\.(\w+)", defs[n]):
                if (p, dep) not in need:
                    need.add((p, dep))
                    changed = True
    order = [n for n, _ in FUSED_SCALED]
    return sorted(need, key=lambda t: (t[0], order.index(t[1])))


def emit_hap_fused(P):
    """hap_fused_P{P}_{part}: part 0 = all statistics, 1 = [0, K), 2 = [K, NS)."""
    import re
    plan_ = fused_plan(P)
    K = fused_split(P)
    ranges = {0: (0, len(plan_)), 1: (0, K), 2: (K, len(plan_))}
    L = [f"// P = {P}, fused path: statistics split at {K} of {len(plan_)}"]
    for part, (lo, hi) in ranges.items():
        lines, used = [], set()
        for si in range(lo, hi):
            name, terms = plan_[si]
            for w, case, args in terms:
                for A, B in fused_terms(case, args, w):
                    for m in re.finditer(r"g(\d)_(\w+)", A + " " + B):
                        used.add((int(m.group(1)), m.group(2)))
                    lines.append(f"    acc[{si - lo}] += {_cexpr(A)} * {_cexpr(B)};  // {name}: {case}{args}")
        defs = dict(FUSED_SCALED)
        L.append("template <typename T>")
        L.append(f"LDK_DEV void hap_fused_P{P}_{part}(const HapFeat<T>* f, T* acc) {{")
        for p, n in _scaled_closure(used):
            e = defs[n].replace("x.", f"f[{p}].")
            e = re.sub(r"g\.(\w+)", lambda m: f"g{p}_{m.group(1)}", e)
            L.append(f"    const T g{p}_{n} = {_cexpr(e)};")
        L.extend(lines)
        L.append("}")
    return "\n".join(L)


def fused_features_ok():
    """Every HapFeat field the fused forms read is computed by hap_features_P*."""
    import re
    for P in (1, 2, 3, 4):
        have = set(hap_features_needed(P)[0]) | {"c1", "c2", "c3", "c4", "ns", "n", "r1", "r2", "r3", "r4"}
        text = " ".join(A + " " + B for _, terms in fused_plan(P) for w, c, a in terms for A, B in fused_terms(c, a, w))
        text += " " + " ".join(e for _, e in FUSED_SCALED)
        used = set(re.findall(r"f\[\d\]\.(\w+)", text))
        scaled_used = {n for p_, n in _scaled_closure(
            {(int(m.group(1)), m.group(2)) for m in re.finditer(r"g(\d)_(\w+)", text)})}
        used |= {d for n, e in FUSED_SCALED if n in scaled_used for d in re.findall(r"x\.(\w+)", e)}
        if not used <= have:
            raise AssertionError(f"P={P}: fused forms read {sorted(used - have)} not computed")
    return True


def numpy_hap_fused(counts_list, n_list=None, part=0):
    """Evaluate the fused forms with NumPy float64 (test helper); columns of the part."""
    import re
    import numpy as np
    P = len(counts_list)
    xs = _numpy_hap_feats(counts_list, n_list, all_features=True)
    env = {}
    for p, x in enumerate(xs):
        for n, e in FUSED_SCALED:
            g = _NS()
            for k, v in env.items():
                if k.startswith(f"g{p}_"):
                    setattr(g, k[len(f"g{p}_"):], v)
            env[f"g{p}_{n}"] = eval(e, {}, {"x": x, "g": g})
    plan_ = fused_plan(P)
    K = fused_split(P)
    lo, hi = {0: (0, len(plan_)), 1: (0, K), 2: (K, len(plan_))}[part]
    out = np.zeros((len(xs[0].c1), hi - lo))
    for si in range(lo, hi):
        for w, case, args in plan_[si][1]:
            for A, B in fused_terms(case, args, w):
                out[:, si - lo] += eval(A, {}, {"f": xs, **env}) * eval(B, {}, {"f": xs, **env})
    return out


def _cexpr(e):
    """Numeric literals as T(...) so float and double instantiations stay exact."""
    import re
    return re.sub(r"(?<![\w.\[])(\d+\.\d+|\d+)(?![\w.\]])", lambda m: f"T({m.group(1)})", e)


HEADER = """// GENERATED by gen_estimators.py -- do not edit by hand.
//
// Straight-line two-locus LD estimators for P = 1..4 populations (haplotype path).
// Statistic order and averaging weights follow moments.LD (pg_gpu ld_pipeline.py:357-457);
// raw-call algebra restates pg_gpu haplotype_kernels.py:69-304 in factored form.
// hap_stats_P* evaluate every distinct raw call (plain kernel, raw-call entry points);
// hap_fused_P* are the statistic-level forms of the tensor-core parse.
#pragma once
"""


def generate(path=None):
    path = path or os.path.join(HERE, "ldk_estimators.cuh")
    parts = [HEADER, '#include "ldk_hap_feat.cuh"', ""]
    for P in (1, 2, 3, 4):
        parts.append(emit_hap(P))
        parts.append("")
    for P in (1, 2, 3, 4):
        parts.append(emit_hap_fused(P))
        parts.append("")
    parts.append('#include "ldk_geno_feat.cuh"')
    for P in (1, 2, 3, 4):
        parts.append(emit_geno(P))
        parts.append("")
    parts.append(emit_raw_dispatch())
    parts.append("")
    parts.append("template <int P> struct HapNStats;")
    for P in (1, 2, 3, 4):
        parts.append(f"template <> struct HapNStats<{P}> {{ static constexpr int value = {len(stat_specs(P))}; }};")
    parts.append("// first statistic of the second half of the fused path's two-way split")
    parts.append("template <int P> struct HapFusedSplit;")
    for P in (1, 2, 3, 4):
        parts.append(f"template <> struct HapFusedSplit<{P}> {{ static constexpr int value = {fused_split(P)}; }};")
    parts.append("""
template <typename T, int P>
LDK_DEV void hap_features(HapFeat<T>& x) {
    if constexpr (P == 1) hap_features_P1<T>(x);
    else if constexpr (P == 2) hap_features_P2<T>(x);
    else if constexpr (P == 3) hap_features_P3<T>(x);
    else hap_features_P4<T>(x);
}
template <typename T, int P, bool PREP = true>
LDK_DEV void geno_features(GenoFeat<T>& x) {
    if constexpr (P == 1) geno_features_P1<T, PREP>(x);
    else if constexpr (P == 2) geno_features_P2<T, PREP>(x);
    else if constexpr (P == 3) geno_features_P3<T, PREP>(x);
    else geno_features_P4<T, PREP>(x);
}
template <typename T, int P, int S = 1>
LDK_DEV void geno_stats(const GenoFeat<T>* f, T* acc) {
    if constexpr (P == 1) geno_stats_P1<T, S>(f, acc);
    else if constexpr (P == 2) geno_stats_P2<T, S>(f, acc);
    else if constexpr (P == 3) geno_stats_P3<T, S>(f, acc);
    else geno_stats_P4<T, S>(f, acc);
}
// Fused-path statistics of part PART (0: all, 1: [0, split), 2: [split, NS)) added into
// acc[0 ..) of that part.
template <typename T, int P, int PART>
LDK_DEV void hap_fused(const HapFeat<T>* f, T* acc) {
#define LDK_FUSED_CASE(PP) \\
    if constexpr (P == PP) { \\
        if constexpr (PART == 0) hap_fused_P##PP##_0<T>(f, acc); \\
        else if constexpr (PART == 1) hap_fused_P##PP##_1<T>(f, acc); \\
        else hap_fused_P##PP##_2<T>(f, acc); \\
    }
    LDK_FUSED_CASE(1)
    LDK_FUSED_CASE(2)
    LDK_FUSED_CASE(3)
    LDK_FUSED_CASE(4)
#undef LDK_FUSED_CASE
}
template <typename T, int P, int S = 1>
LDK_DEV void hap_stats(const HapFeat<T>* f, T* acc) {
    if constexpr (P == 1) hap_stats_P1<T, S>(f, acc);
    else if constexpr (P == 2) hap_stats_P2<T, S>(f, acc);
    else if constexpr (P == 3) hap_stats_P3<T, S>(f, acc);
    else hap_stats_P4<T, S>(f, acc);
}
""")
    text = "\n".join(parts)
    with open(path, "w") as fh:
        fh.write(text)
    return path


# ---------------------------------------------------------------------------
# NumPy evaluation of the same expressions (used by the unit tests)
# ---------------------------------------------------------------------------


class _NS:
    pass


def _numpy_hap_feats(counts_list, n_list=None, all_features=False):
    import numpy as np
    P = len(counts_list)
    feats = [n for n, _ in HAP_FEATURES] if all_features else hap_features_needed(P)[0]
    fs = []
    for p, c in enumerate(counts_list):
        c = np.asarray(c, dtype=np.float64)
        x = _NS()
        x.c1, x.c2, x.c3, x.c4 = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
        x.ns = x.c1 + x.c2 + x.c3 + x.c4
        x.n = x.ns if (n_list is None or n_list[p] is None) else np.asarray(n_list[p], np.float64)
        for name, e in HAP_FEATURES:
            if name in feats:
                setattr(x, name, eval(e, {}, {"x": x}))
        n = x.n
        with np.errstate(divide="ignore", invalid="ignore"):
            d1, d2 = n, n * (n - 1)
            d3, d4 = d2 * (n - 2), d2 * (n - 2) * (n - 3)
            x.r1 = np.where(d1 > 0, 1 / np.where(d1 > 0, d1, 1), 0.0)
            x.r2 = np.where(d2 > 0, 1 / np.where(d2 > 0, d2, 1), 0.0)
            x.r3 = np.where(d3 > 0, 1 / np.where(d3 > 0, d3, 1), 0.0)
            x.r4 = np.where(d4 > 0, 1 / np.where(d4 > 0, d4, 1), 0.0)
        fs.append(x)
    return fs


def numpy_hap_stats(counts_list, n_list=None):
    """Evaluate the generated expressions with NumPy float64 (test helper)."""
    import numpy as np
    fs = _numpy_hap_feats(counts_list, n_list)
    calls, stats = plan(len(counts_list))
    vals = [eval(hap_call_expr(case, args), {}, {"f": fs}) for case, args in calls]
    out = np.zeros((len(fs[0].c1), len(stats)))
    for si, (_, terms) in enumerate(stats):
        for idx, w in terms:
            out[:, si] += w * vals[idx]
    return out


def check():
    """Symbolic check of the factored forms against the reference formulas (sympy)."""
    import sympy as sp
    for poly in _HORNER_POLYS.values():
        e, _, g = _horner_sympy(poly)
        loc = {f"g{i + 1}": g[i] for i in range(9)}
        h = sp.sympify(horner_form(poly).replace("x.g", "g"), locals=loc)
        assert sp.expand(h - e) == 0
    a = sp.symbols("a1:5")
    b = sp.symbols("b1:5")

    def feats(c):
        x = _NS()
        x.c1, x.c2, x.c3, x.c4 = c
        x.ns = sum(c)
        x.n = x.ns
        for name, e in HAP_FEATURES:
            setattr(x, name, eval(e, {}, {"x": x}))
        return x

    X, Y = feats(a), feats(b)
    a1, a2, a3, a4 = a
    b1, b2, b3, b4 = b
    # pi2(i,j,i,j) numerator, haplotype_kernels.py:250-263
    qBa, qAa, pAb, pBb = a2 + a4, a3 + a4, b1 + b2, b1 + b3
    pBa, qAb, qBb, pAa = a1 + a3, b3 + b4, b2 + b4, a1 + a2
    ref_ijij = ((qBa * qAa * pAb * pBb + pBa * qAa * pAb * qBb + pAa * qBa * pBb * qAb + pAa * pBa * qBb * qAb
                 + (-(a2 * a3 * b1) + a4 * b1 - a2 * a4 * b1 - a3 * a4 * b1 - a4 * a4 * b1 - a4 * b1 * b1
                    + a3 * b2 - a1 * a3 * b2 - a3 * a3 * b2 - a1 * a4 * b2 - a3 * a4 * b2 - a3 * b1 * b2
                    - a4 * b1 * b2 - a3 * b2 * b2 + a2 * b3 - a1 * a2 * b3 - a2 * a2 * b3 - a1 * a4 * b3
                    - a2 * a4 * b3 - a2 * b1 * b3 - a4 * b1 * b3 - a1 * b2 * b3 - a4 * b2 * b3 - a2 * b3 * b3
                    + a1 * b4 - a1 * a1 * b4 - a1 * a2 * b4 - a1 * a3 * b4 - a2 * a3 * b4 - a2 * b1 * b4
                    - a3 * b1 * b4 - a1 * b2 * b4 - a3 * b2 * b4 - a1 * b3 * b4 - a2 * b3 * b4
                    - a1 * b4 * b4)) / 4)
    HA = X.pA * Y.qA + X.qA * Y.pA
    HB = X.pB * Y.qB + X.qB * Y.pB
    corr = (X.Q1 * b4 + X.Q2 * b3 + X.Q3 * b2 + X.Q4 * b1
            - (a1 * Y.L1 + a2 * Y.L2 + a3 * Y.L3 + a4 * Y.L4))
    assert sp.expand(ref_ijij - (HA * HB + corr) / 4) == 0
    # fused path: the symmetric pi2(i,j,i,j) correction and F_k = L_k - c_{5-k}
    Xs = a4 * b1 + a3 * b2 + a2 * b3 + a1 * b4
    corr2 = Xs * (1 - X.ns - Y.ns) - (X.E * Y.s + Y.E * X.s)
    assert sp.expand(corr - corr2) == 0
    m1 = X.ns - 1
    for Lk, ck, sig in ((X.L1, a4, 1), (X.L2, a3, -1), (X.L3, a2, -1), (X.L4, a1, 1)):
        assert sp.expand((Lk - ck) - (ck * m1 - sig * X.E)) == 0
    # single-population numerators, haplotype_kernels.py:76, 102-104, 298-301
    c1, c2, c3, c4 = a
    assert sp.expand(X.DDs - (c1 * (c1 - 1) * c4 * (c4 - 1) + c2 * (c2 - 1) * c3 * (c3 - 1)
                              - 2 * c1 * c2 * c3 * c4)) == 0
    diff = c1 * c4 - c2 * c3
    assert sp.expand(X.DZs - (diff * (c3 + c4 - c1 - c2) * (c2 + c4 - c1 - c3) + diff * (c2 + c3 - c1 - c4)
                              + 2 * (c2 * c3 + c1 * c4))) == 0
    assert sp.expand(X.PIs - ((c1 + c2) * (c1 + c3) * (c2 + c4) * (c3 + c4)
                              - c1 * c4 * (-1 + c1 + 3 * c2 + 3 * c3 + c4)
                              - c2 * c3 * (-1 + 3 * c1 + c2 + c3 + 3 * c4))) == 0
    # triple, haplotype_kernels.py:276-286 (t = a, single = b)
    tpA, tqA = a1 + a2, a3 + a4
    spB, sqB = b1 + b3, b2 + b4
    ref_tr = (-(tpA * a4 * spB) - (a2 * tqA * spB) + (tpA * (a2 + a4) * tqA * spB)
              + (tpA * tqA * (-2 * b2 - 2 * b4)) + (tpA * a4 * sqB) + (a2 * tqA * sqB)
              + (tpA * (a1 + a3) * tqA * sqB)) / 2
    assert sp.expand(ref_tr - (spB * X.T1 + sqB * X.T2) / 2) == 0
    # shared, haplotype_kernels.py:225-238 (s = a, a-pop = b, b-pop = c)
    c = sp.symbols("e1:5")
    Z = feats(c)
    s1, s2, s3, s4 = a
    ca1, ca2 = b1, b2
    cb1, cb2, cb3, cb4 = c
    inner = (-1 + s3) * cb1 + s3 * cb2 - cb3 + s3 * cb3 + s3 * cb4 + s1 * Z.qB
    ref_sh = (s4 * s4 * Y.pA * Z.pB + s2 * s2 * Y.qA * Z.pB
              + (-1 + s1 + s3) * (s3 * Y.pA + s1 * Y.qA) * Z.qB
              + s4 * (s1 * Y.qA * Z.pB + ca1 * inner + ca2 * inner)
              + s2 * (s4 * (Y.pA + Y.qA) * Z.pB + s3 * (ca1 * Z.pB + ca2 * Z.pB + Y.qA * Z.qB)
                      + Y.qA * ((-1 + s1) * cb1 - cb3 + s1 * (cb2 + cb3 + cb4)))) / 4
    mine = (Y.pA * (Z.pB * (X.L1 - s4) + Z.qB * (X.L2 - s3))
            + Y.qA * (Z.pB * (X.L3 - s2) + Z.qB * (X.L4 - s1))) / 4
    assert sp.expand(ref_sh - mine) == 0
    return True


if __name__ == "__main__":
    check()
    fused_features_ok()
    print(generate())
