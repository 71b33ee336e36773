"""CPU oracle for the two-locus LD parse -- TEST INFRASTRUCTURE ONLY.

A float64 NumPy restatement of pg_gpu's LD path (pairs within a distance cutoff ->
per-population two-locus counts -> unbiased DD / Dz / pi2 and r^2 estimators ->
distance-bin sums).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / ``--impl reference`` leg may import this module, and only as the
checker or the timed CPU baseline; the product (``pg_gpu_b200``) never calls it.

Every function cites the reference file:line it restates (paths relative to the
pg_gpu checkout).  Arithmetic is float64 throughout, which is what the reference
computes on its multi-population ``PopData`` / ``_PopDataGeno`` path.  (The
reference's own 1- and 2-population haplotype path evaluates the same polynomials in
the int32 dtype of its counts and overflows for large samples; the oracle follows the
float64 form.)

Parity pins (tests/test_oracle_golden.py):
  * moments' own output on the reference's IM example (``tests/golden/im_example.npz``);
  * the reference's Python dispatch and kernel bodies run on the host
    (``tests/golden/ref_*.npz``, made by ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------------------
# statistic names and averaging specs  (ld_pipeline.py:357-457)
# ---------------------------------------------------------------------------


def ld_names(num_pops):
    """moments.LD.Util.ld_names order (ld_pipeline.py:357-376)."""
    names = []
    P = num_pops
    for i in range(P):
        for j in range(i, P):
            names.append(f"DD_{i}_{j}")
    for i in range(P):
        for j in range(P):
            for k in range(j, P):
                names.append(f"Dz_{i}_{j}_{k}")
    for i in range(P):
        for j in range(i, P):
            for k in range(i, P):
                for l in range(k, P):
                    if k == i == l and j != i:
                        continue
                    if i == k and l < j:
                        continue
                    names.append(f"pi2_{i}_{j}_{k}_{l}")
    return names


def het_names(num_pops):
    """ld_pipeline.py:379-385."""
    return [f"H_{i}_{j}" for i in range(num_pops) for j in range(i, num_pops)]


def stat_specs(num_pops):
    """Averaging of raw estimator calls per named statistic (ld_pipeline.py:388-457)."""
    specs = []
    for name in ld_names(num_pops):
        kind, *nums = name.split("_")
        p = tuple(int(x) for x in nums)
        if kind == "DD":
            specs.append((name, [(1.0, "dd", p)]))
        elif kind == "Dz":
            i, j, k = p
            if j == k:
                specs.append((name, [(1.0, "dz", p)]))
            else:
                specs.append((name, [(0.5, "dz", (i, j, k)), (0.5, "dz", (i, k, j))]))
        else:
            i, j, k, l = p
            if i == j and k == l:
                if i == k:
                    calls = [(1.0, p)]
                else:
                    calls = [(0.5, (i, j, k, l)), (0.5, (k, l, i, j))]
            elif i == j:
                calls = [(0.25, q) for q in ((i, j, k, l), (i, j, l, k), (k, l, i, j), (l, k, i, j))]
            elif k == l:
                calls = [(0.25, q) for q in ((i, j, k, l), (j, i, k, l), (k, l, i, j), (k, l, j, i))]
            else:
                calls = [(0.125, q) for q in ((i, j, k, l), (i, j, l, k), (j, i, k, l), (j, i, l, k),
                                               (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i))]
            specs.append((name, [(w, "pi2", q) for w, q in calls]))
    return specs


# ---------------------------------------------------------------------------
# pairs and bins
# ---------------------------------------------------------------------------


def pairs_within_distance(positions, max_dist):
    """All (i, j), i < j, with pos[j] - pos[i] <= max_dist, in anchor order.

    ld_pipeline.py:85-121 (searchsorted on pos + max_dist, side='right').
    """
    pos = np.asarray(positions)
    n = len(pos)
    if n < 2:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    jmax = np.searchsorted(pos, pos + max_dist, side="right")
    per = np.maximum(0, jmax - np.arange(n) - 1)
    tot = int(per.sum())
    ii = np.repeat(np.arange(n, dtype=np.int64), per)
    start = np.cumsum(per) - per
    jj = ii + 1 + (np.arange(tot, dtype=np.int64) - np.repeat(start, per))
    return ii, jj


def bin_index(dist, edges):
    """cp.digitize(d, edges) - 1: bins are right-open [e_b, e_{b+1}) (moments_ld.py:314)."""
    return np.digitize(dist, np.asarray(edges, dtype=np.float64)) - 1


# ---------------------------------------------------------------------------
# two-locus counts
# ---------------------------------------------------------------------------


def hap_counts(hap, idx_i, idx_j, rows=None):
    """[n11, n10, n01, n00] per pair plus n_valid (ld_pipeline.py:130-175).

    ``n_valid`` is None unless the population's rows hold a -1 anywhere (:158).
    """
    h = hap if rows is None else hap[np.asarray(rows)]
    a = h[:, idx_i]
    b = h[:, idx_j]
    has_missing = bool(np.any(h == -1))
    valid = (a >= 0) & (b >= 0)
    n11 = np.sum((a == 1) & (b == 1) & valid, axis=0)
    n10 = np.sum((a == 1) & (b == 0) & valid, axis=0)
    n01 = np.sum((a == 0) & (b == 1) & valid, axis=0)
    n00 = np.sum((a == 0) & (b == 0) & valid, axis=0)
    counts = np.stack([n11, n10, n01, n00], axis=1).astype(np.int64)
    n_valid = np.sum(valid, axis=0).astype(np.int64) if has_missing else None
    return counts, n_valid


def geno_counts(geno, idx_i, idx_j, rows=None):
    """9-cell genotype table, column g_i*3+g_j, plus valid count (ld_pipeline.py:183-263)."""
    g = geno if rows is None else geno[np.asarray(rows)]
    a = g[:, idx_i].astype(np.int64)
    b = g[:, idx_j].astype(np.int64)
    valid = (a >= 0) & (b >= 0)
    combo = np.where(valid, a * 3 + b, -1)
    counts = np.stack([np.sum(combo == c, axis=0) for c in range(9)], axis=1).astype(np.int64)
    n_valid = np.sum(valid, axis=0).astype(np.int64)
    return counts, (n_valid if bool(np.any(g < 0)) else None)


# ---------------------------------------------------------------------------
# haplotype estimators  (ld_pipeline.py:465-482; haplotype_kernels.py:69-640)
# ---------------------------------------------------------------------------


class HapPop:
    """Float64 per-population features of one batch of pairs (ld_pipeline.py:465-482)."""

    def __init__(self, counts, n_valid=None):
        c = np.asarray(counts, dtype=np.float64)
        self.c1, self.c2, self.c3, self.c4 = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
        self.n = (np.asarray(n_valid, dtype=np.float64) if n_valid is not None
                  else self.c1 + self.c2 + self.c3 + self.c4)
        self.D = self.c2 * self.c3 - self.c1 * self.c4
        self.pA = self.c1 + self.c2
        self.qA = self.c3 + self.c4
        self.pB = self.c1 + self.c3
        self.qB = self.c2 + self.c4


def _div(num, den):
    """``(den > 0) ? num / den : 0`` as in every fused haplotype kernel."""
    out = np.zeros_like(den, dtype=np.float64)
    ok = den > 0
    out[ok] = num[ok] / den[ok]
    return out


def _hap_dd(P, p):
    i, j = p
    if i == j:  # haplotype_kernels.py:69-79
        x = P[i]
        a, b, c, d, n = x.c1, x.c2, x.c3, x.c4, x.n
        num = a * (a - 1) * d * (d - 1) + b * (b - 1) * c * (c - 1) - 2 * a * b * c * d
        return _div(num, n * (n - 1) * (n - 2) * (n - 3))
    x, y = P[i], P[j]  # :81-89
    return _div(x.D * y.D, x.n * (x.n - 1) * y.n * (y.n - 1))


def _hap_dz(P, p):
    p1, p2, p3 = p
    if p1 == p2 == p3:  # haplotype_kernels.py:95-107
        x = P[p1]
        a, b, c, d, n = x.c1, x.c2, x.c3, x.c4, x.n
        diff = a * d - b * c
        num = diff * (c + d - a - b) * (b + d - a - c) + diff * (b + c - a - d) + 2 * (b * c + a * d)
        return _div(num, n * (n - 1) * (n - 2) * (n - 3))
    if p1 == p2:  # :109-120, i = p1, j = p3
        x, y = P[p1], P[p3]
        num = (-x.pA + x.qA) * (-x.D) * (-y.c1 + y.c2 - y.c3 + y.c4)
        return _div(num, y.n * x.n * (x.n - 1) * (x.n - 2))
    if p1 == p3:  # :122-133, i = p1, j = p2
        x, y = P[p1], P[p2]
        num = (-x.c1 + x.c2 - x.c3 + x.c4) * (-x.D) * (-y.pA + y.qA)
        return _div(num, y.n * x.n * (x.n - 1) * (x.n - 2))
    if p2 == p3:  # :135-147, i = p1, j = p2
        x, y = P[p1], P[p2]
        num = ((-x.D) * (-y.c1 + y.c2 + y.c3 - y.c4)
               + (-x.D) * (-y.c1 + y.c2 - y.c3 + y.c4) * (-y.pA + y.qA))
        return _div(num, x.n * (x.n - 1) * y.n * (y.n - 1))
    x, y, z = P[p1], P[p2], P[p3]  # :149-160
    num = -(x.D * (y.pA - y.qA) * (z.c1 - z.c2 + z.c3 - z.c4))
    return _div(num, x.n * (x.n - 1) * y.n * z.n)


def pi2_case(p):
    """Case of a raw pi2 call (haplotype_kernels.py:463-486)."""
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


def shared_roles(p):
    """(shared, other-of-first-pair, other-of-second-pair) (haplotype_kernels.py:527-541)."""
    i, j, k, l = p
    if i == k:
        return i, j, l
    if i == l:
        return i, j, k
    if j == k:
        return j, i, l
    if j == l:
        return j, i, k
    return 0, 0, 0


def triple_roles(p):
    """(tripled population, single population) (haplotype_kernels.py:549-556)."""
    cnt = {}
    for q in p:
        cnt[q] = cnt.get(q, 0) + 1
    return ([q for q, c in cnt.items() if c == 3][0], [q for q, c in cnt.items() if c == 1][0])


def _hap_pi2(P, p):
    case = pi2_case(p)
    i, j, k, l = p
    if case == "alldiff":  # haplotype_kernels.py:167-178
        HA = P[i].pA * P[j].qA + P[i].qA * P[j].pA
        HB = P[k].pB * P[l].qB + P[k].qB * P[l].pB
        return _div(HA * HB, 4 * P[i].n * P[j].n * P[k].n * P[l].n)
    if case == "iikk":  # :180-190
        x, y = P[i], P[k]
        return _div(x.pA * x.qA * y.pB * y.qB, x.n * (x.n - 1) * y.n * (y.n - 1))
    if case == "iikl":  # :192-203
        x = P[i]
        HB = P[k].pB * P[l].qB + P[k].qB * P[l].pB
        return _div(x.pA * x.qA * HB, 2 * x.n * (x.n - 1) * P[k].n * P[l].n)
    if case == "ijkk":  # :205-216
        HA = P[i].pA * P[j].qA + P[i].qA * P[j].pA
        z = P[k]
        return _div(z.pB * z.qB * HA, 2 * z.n * (z.n - 1) * P[i].n * P[j].n)
    if case == "shared":  # :218-241
        s, a, b = shared_roles(p)
        S, A, B = P[s], P[a], P[b]
        cs1, cs2, cs3, cs4, ns = S.c1, S.c2, S.c3, S.c4, S.n
        ca1, ca2, cb1, cb2, cb3, cb4 = A.c1, A.c2, B.c1, B.c2, B.c3, B.c4
        inner = (-1 + cs3) * cb1 + cs3 * cb2 - cb3 + cs3 * cb3 + cs3 * cb4 + cs1 * B.qB
        num = (cs4 * cs4 * A.pA * B.pB
               + cs2 * cs2 * A.qA * B.pB
               + (-1 + cs1 + cs3) * (cs3 * A.pA + cs1 * A.qA) * B.qB
               + cs4 * (cs1 * A.qA * B.pB + ca1 * inner + ca2 * inner)
               + cs2 * (cs4 * (A.pA + A.qA) * B.pB
                        + cs3 * (ca1 * B.pB + ca2 * B.pB + A.qA * B.qB)
                        + A.qA * ((-1 + cs1) * cb1 - cb3 + cs1 * (cb2 + cb3 + cb4)))) / 4
        return _div(num, ns * (ns - 1) * A.n * B.n)
    if case == "triple":  # :268-289
        t, s = triple_roles(p)
        T, S = P[t], P[s]
        t1, t2, t3, t4, nt = T.c1, T.c2, T.c3, T.c4, T.n
        tpA, tqA = t1 + t2, t3 + t4
        num = (-(tpA * t4 * S.pB) - (t2 * tqA * S.pB) + (tpA * (t2 + t4) * tqA * S.pB)
               + (tpA * tqA * (-2 * S.c2 - 2 * S.c4)) + (tpA * t4 * S.qB) + (t2 * tqA * S.qB)
               + (tpA * (t1 + t3) * tqA * S.qB)) / 2
        return _div(num, S.n * nt * (nt - 1) * (nt - 2))
    if case == "ijij":  # :243-266
        X, Y = P[i], P[j]
        a1, a2, a3, a4 = X.c1, X.c2, X.c3, X.c4
        b1, b2, b3, b4 = Y.c1, Y.c2, Y.c3, Y.c4
        qBa, qAa, pAb, pBb = a2 + a4, a3 + a4, b1 + b2, b1 + b3
        pBa, qAb, qBb, pAa = a1 + a3, b3 + b4, b2 + b4, a1 + a2
        corr = (-(a2 * a3 * b1) + a4 * b1 - a2 * a4 * b1 - a3 * a4 * b1 - a4 * a4 * b1 - a4 * b1 * b1
                + a3 * b2 - a1 * a3 * b2 - a3 * a3 * b2 - a1 * a4 * b2 - a3 * a4 * b2 - a3 * b1 * b2
                - a4 * b1 * b2 - a3 * b2 * b2
                + a2 * b3 - a1 * a2 * b3 - a2 * a2 * b3 - a1 * a4 * b3 - a2 * a4 * b3 - a2 * b1 * b3
                - a4 * b1 * b3 - a1 * b2 * b3 - a4 * b2 * b3 - a2 * b3 * b3
                + a1 * b4 - a1 * a1 * b4 - a1 * a2 * b4 - a1 * a3 * b4 - a2 * a3 * b4 - a2 * b1 * b4
                - a3 * b1 * b4 - a1 * b2 * b4 - a3 * b2 * b4 - a1 * b3 * b4 - a2 * b3 * b4 - a1 * b4 * b4)
        num = (qBa * qAa * pAb * pBb / 4 + pBa * qAa * pAb * qBb / 4 + pAa * qBa * pBb * qAb / 4
               + pAa * pBa * qBb * qAb / 4 + corr / 4)
        return _div(num, X.n * (X.n - 1) * Y.n * (Y.n - 1))
    x = P[i]  # same: :291-304
    a, b, c, d, n = x.c1, x.c2, x.c3, x.c4, x.n
    num = ((a + b) * (a + c) * (b + d) * (c + d) - a * d * (-1 + a + 3 * b + 3 * c + d)
           - b * c * (-1 + 3 * a + b + c + 3 * d))
    return _div(num, n * (n - 1) * (n - 2) * (n - 3))


_HAP_KIND = {"dd": _hap_dd, "dz": _hap_dz, "pi2": _hap_pi2}


def hap_raw(kind, pops, P):
    """One raw estimator call on per-pop features ``P`` (list of HapPop)."""
    return _HAP_KIND[kind](P, pops)


def assemble(specs, raw):
    """Weighted sums of cached raw calls (haplotype_kernels.py:627-640)."""
    cols = []
    for _, calls in specs:
        cols.append(sum(w * raw(k, q) for w, k, q in calls))
    return np.stack(cols, axis=1)


def hap_stats(counts_list, n_valid_list=None):
    """(N, n_stats) moments-ordered statistics (haplotype_kernels.py:584-640)."""
    Pn = len(counts_list)
    if n_valid_list is None:
        n_valid_list = [None] * Pn
    pops = [HapPop(c, nv) for c, nv in zip(counts_list, n_valid_list)]
    cache = {}

    def raw(k, q):
        if (k, q) not in cache:
            cache[(k, q)] = hap_raw(k, q, pops)
        return cache[(k, q)]

    return assemble(stat_specs(Pn), raw)


def hap_r_squared(counts, n_valid=None):
    """r^2 = D^2 / (pA qA pB qB) in frequencies; NaN if the denominator is 0
    (haplotype_kernels.py:32-42)."""
    c = np.asarray(counts, dtype=np.float64)
    a, b, cc, d = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    n = np.asarray(n_valid, np.float64) if n_valid is not None else a + b + cc + d
    with np.errstate(divide="ignore", invalid="ignore"):
        pA = (a + b) / n
        pB = (a + cc) / n
        D = (a * d - b * cc) / (n * n)
        den = pA * (1.0 - pA) * pB * (1.0 - pB)
        return np.where(den > 0.0, D * D / np.where(den > 0, den, 1.0), np.nan)


def hap_r(counts, n_valid=None):
    """Signed r (haplotype_kernels.py:20-30)."""
    c = np.asarray(counts, dtype=np.float64)
    a, b, cc, d = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    n = np.asarray(n_valid, np.float64) if n_valid is not None else a + b + cc + d
    with np.errstate(divide="ignore", invalid="ignore"):
        pA = (a + b) / n
        pB = (a + cc) / n
        D = (a * d - b * cc) / (n * n)
        den = pA * (1.0 - pA) * pB * (1.0 - pB)
        return np.where(den > 0.0, D / np.sqrt(np.where(den > 0, den, 1.0)), np.nan)


def hap_d_prime(counts, n_valid=None):
    """Lewontin's D' (haplotype_kernels.py:44-62)."""
    c = np.asarray(counts, dtype=np.float64)
    a, b, cc, d = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    n = np.asarray(n_valid, np.float64) if n_valid is not None else a + b + cc + d
    with np.errstate(divide="ignore", invalid="ignore"):
        pA = (a + b) / n
        pB = (a + cc) / n
        qA, qB = 1.0 - pA, 1.0 - pB
        D = (a * d - b * cc) / (n * n)
        dmax = np.where(D >= 0.0, np.minimum(pA * qB, qA * pB), np.minimum(pA * pB, qA * qB))
        return np.where(dmax > 0.0, D / np.where(dmax > 0, dmax, 1.0), np.nan)


# ---------------------------------------------------------------------------
# genotype estimators  (genotype_kernels.py:27-936)
# ---------------------------------------------------------------------------


def to_moments_order(counts9):
    """g1..g9 = n22, n21, n20, n12, n11, n10, n02, n01, n00 (genotype_kernels.py:424-435)."""
    c = np.asarray(counts9, dtype=np.float64)
    return [c[:, 8 - m] for m in range(9)]


class GenoPop:
    """Float64 per-population genotype features (genotype_kernels.py:412-492, 513-554)."""

    def __init__(self, counts9, n_valid=None):
        g = to_moments_order(counts9)
        self.g = g
        g1, g2, g3, g4, g5, g6, g7, g8, g9 = g
        self.n = (np.asarray(n_valid, np.float64) if n_valid is not None
                  else g1 + g2 + g3 + g4 + g5 + g6 + g7 + g8 + g9)
        n = self.n
        self.x_AB = g1 + g2 / 2 + g4 / 2 + g5 / 4
        self.x_Ab = g2 / 2 + g3 + g5 / 4 + g6 / 2
        self.x_aB = g4 / 2 + g5 / 4 + g7 + g8 / 2
        self.x_ab = g5 / 4 + g6 / 2 + g8 / 2 + g9
        self.D = self.x_AB * self.x_ab - self.x_Ab * self.x_aB
        self.pA = g1 + g2 + g3 + g4 / 2 + g5 / 2 + g6 / 2
        self.qA = g4 / 2 + g5 / 2 + g6 / 2 + g7 + g8 + g9
        self.pB = g1 + g2 / 2 + g4 + g5 / 2 + g7 + g8 / 2
        self.qB = g2 / 2 + g3 + g5 / 2 + g6 + g8 / 2 + g9
        nn1 = np.maximum(4 * n * (n - 1), 1)
        self.BL = (4 * self.pA * self.qA - (g4 + g5 + g6)) / nn1
        self.BR = (4 * self.pB * self.qB - (g2 + g5 + g8)) / nn1
        self.C00 = (self.pA * self.pB - self.x_AB) / nn1
        self.C01 = (self.pA * self.qB - self.x_Ab) / nn1
        self.C10 = (self.qA * self.pB - self.x_aB) / nn1
        self.C11 = (self.qA * self.qB - self.x_ab) / nn1
        self.Bsgn = self.x_AB - self.x_Ab - self.x_aB + self.x_ab
        with np.errstate(divide="ignore", invalid="ignore"):
            self.p, self.r = self.pA / n, self.qA / n
            self.q, self.s = self.pB / n, self.qB / n
        P, R, Q, S = self.pA, self.qA, self.pB, self.qB
        L0 = g5 + 2 * g6 + 2 * g8 + 4 * g9
        L1 = g5 + 2 * g6
        M1 = g5 + 2 * g8
        negR3 = 3 * g4 + 3 * g5 + 3 * g6 + 4 * g7 + 4 * g8 + 4 * g9
        negR5 = 5 * g4 + 5 * g5 + 5 * g6 + 8 * g7 + 8 * g8 + 8 * g9
        b5A = -2 * g2 - 4 * g3 + 4 * g4 + g5 - 2 * g6 + 8 * g7 + 4 * g8 + 4
        b6A = -g5 - 2 * g6 - 4 * g7 - 4 * g8 - 4 * g9
        self.AQ3 = -(S * negR3) / 8 + P * S * R / 2 + (R * L0) / 8 + L1 / 8 - (P * L0) / 8
        self.AS3 = -(Q * negR5) / 8 + P * Q * R / 2 + (R * b5A) / 8 + b6A / 8 + (P * L0) / 8
        negL3 = 3 * g2 + 4 * g3 + 3 * g5 + 4 * g6 + 3 * g8 + 4 * g9
        negL5 = 5 * g2 + 8 * g3 + 5 * g5 + 8 * g6 + 5 * g8 + 8 * g9
        b5B = 4 * g2 + 8 * g3 - 2 * g4 + g5 + 4 * g6 - 4 * g7 - 2 * g8 + 4
        b6B = -4 * g3 - g5 - 4 * g6 - 2 * g8 - 4 * g9
        self.BP3 = -(R * negL3) / 8 + Q * S * R / 2 + (S * L0) / 8 + M1 / 8 - (Q * L0) / 8
        self.BR3 = -(P * negL5) / 8 + P * Q * S / 2 + (S * b5B) / 8 + b6B / 8 + (Q * L0) / 8
        # Dz features (genotype_kernels.py:176-197)
        self.A = -g1 + g3 - g4 + g6 - g7 + g9
        self.Bv = -g1 - g2 - g3 + g7 + g8 + g9
        c = -g1 + g3 + g7 - g9
        MA = (2 * g2 * g7 + 4 * g3 * g7 + 2 * g5 * g7 + 4 * g6 * g7 - 2 * g1 * g8 + 2 * g3 * g8
              - 2 * g4 * g8 + 2 * g6 * g8 - 4 * g1 * g9 - 2 * g2 * g9 - 4 * g4 * g9 - 2 * g5 * g9)
        MB = (2 * g3 * g4 + 2 * g3 * g5 - 2 * g1 * g6 - 2 * g2 * g6 + 4 * g3 * g7 + 2 * g6 * g7
              + 4 * g3 * g8 + 2 * g6 * g8 - 4 * g1 * g9 - 4 * g2 * g9 - 2 * g4 * g9 - 2 * g5 * g9)
        self.Wjj = c + self.A * self.Bv
        self.U = self.D * (1 + self.Bv) + 0.25 * MA
        self.V = self.D * (1 + self.A) + 0.25 * MB
        self.ns = g1 + g2 + g3 + g4 + g5 + g6 + g7 + g8 + g9


def geno_dd_single_num(g):
    """16x the polynomial part of genotype DD(i,i) (genotype_kernels.py:43-68)."""
    n1, n2, n3, n4, n5, n6, n7, n8, n9 = g
    return ((n2 * n4 - n2 * n2 * n4 + 4 * n3 * n4 - 4 * n2 * n3 * n4 - 4 * n3 * n3 * n4)
            + (-n2 * n4 * n4 - 4 * n3 * n4 * n4)
            + (n1 * n5 - n1 * n1 * n5 + n3 * n5 + 2 * n1 * n3 * n5 - n3 * n3 * n5
               - 4 * n3 * n4 * n5 - n1 * n5 * n5 - n3 * n5 * n5)
            + (4 * n1 * n6 - 4 * n1 * n1 * n6 + n2 * n6 - 4 * n1 * n2 * n6 - n2 * n2 * n6
               + 2 * n2 * n4 * n6 - 4 * n1 * n5 * n6 - 4 * n1 * n6 * n6 - n2 * n6 * n6)
            + (4 * n2 * n7 - 4 * n2 * n2 * n7
               + 16 * n3 * n7 - 16 * n2 * n3 * n7 - 16 * n3 * n3 * n7
               - 4 * n2 * n4 * n7 - 16 * n3 * n4 * n7
               + n5 * n7 + 2 * n1 * n5 * n7 - 4 * n2 * n5 * n7 - 18 * n3 * n5 * n7 - n5 * n5 * n7
               + 4 * n6 * n7 + 8 * n1 * n6 * n7 - 16 * n3 * n6 * n7 - 4 * n5 * n6 * n7 - 4 * n6 * n6 * n7
               - 4 * n2 * n7 * n7 - 16 * n3 * n7 * n7 - n5 * n7 * n7 - 4 * n6 * n7 * n7)
            + (4 * n1 * n8 - 4 * n1 * n1 * n8 + 4 * n3 * n8 + 8 * n1 * n3 * n8 - 4 * n3 * n3 * n8
               + n4 * n8 - 4 * n1 * n4 * n8 + 2 * n2 * n4 * n8 - n4 * n4 * n8
               - 4 * n1 * n5 * n8 - 4 * n3 * n5 * n8
               + n6 * n8 + 2 * n2 * n6 * n8 - 4 * n3 * n6 * n8 + 2 * n4 * n6 * n8 - n6 * n6 * n8
               - 16 * n3 * n7 * n8 - 4 * n6 * n7 * n8
               - 4 * n1 * n8 * n8 - 4 * n3 * n8 * n8 - n4 * n8 * n8 - n6 * n8 * n8)
            + (16 * n1 * n9 - 16 * n1 * n1 * n9 + 4 * n2 * n9 - 16 * n1 * n2 * n9 - 4 * n2 * n2 * n9
               + 4 * n4 * n9 - 16 * n1 * n4 * n9 + 8 * n3 * n4 * n9 - 4 * n4 * n4 * n9
               + n5 * n9 - 18 * n1 * n5 * n9 - 4 * n2 * n5 * n9 + 2 * n3 * n5 * n9 - 4 * n4 * n5 * n9
               - n5 * n5 * n9
               - 16 * n1 * n6 * n9 - 4 * n2 * n6 * n9
               + 8 * n2 * n7 * n9 + 2 * n5 * n7 * n9
               - 16 * n1 * n8 * n9 - 4 * n4 * n8 * n9
               - 16 * n1 * n9 * n9 - 4 * n2 * n9 * n9 - 4 * n4 * n9 * n9 - n5 * n9 * n9))


def geno_dz_single_quartic(g):
    """Quartic part of genotype Dz(i,i,i) (genotype_kernels.py:249-269)."""
    n1, n2, n3, n4, n5, n6, n7, n8, n9 = g
    return (-(n2 * n4) + 3 * n1 * n2 * n4 + n2 * n2 * n4 + 2 * n3 * n4 + 4 * n1 * n3 * n4 - n2 * n3 * n4
            - 4 * n3 * n3 * n4 + n2 * n4 * n4 + 2 * n3 * n4 * n4 + 2 * n1 * n5 - 3 * n1 * n1 * n5 - n1 * n2 * n5
            + 2 * n3 * n5 + 2 * n1 * n3 * n5 - n2 * n3 * n5 - 3 * n3 * n3 * n5 - n1 * n4 * n5 + n3 * n4 * n5
            + 2 * n1 * n6 - 4 * n1 * n1 * n6 - n2 * n6 - n1 * n2 * n6 + n2 * n2 * n6 + 4 * n1 * n3 * n6
            + 3 * n2 * n3 * n6 - 2 * n1 * n4 * n6 - 2 * n2 * n4 * n6 - 2 * n3 * n4 * n6 + n1 * n5 * n6 - n3 * n5 * n6
            + 2 * n1 * n6 * n6 + n2 * n6 * n6 + 2 * n2 * n7 + 4 * n1 * n2 * n7 + 2 * n2 * n2 * n7 + 8 * n3 * n7
            + 4 * n1 * n3 * n7 - 4 * n3 * n3 * n7 - n2 * n4 * n7 + 2 * n5 * n7 + 2 * n1 * n5 * n7 + n2 * n5 * n7
            + 2 * n3 * n5 * n7 - n4 * n5 * n7 + 2 * n6 * n7 - n2 * n6 * n7 - 2 * n4 * n6 * n7 + n5 * n6 * n7
            + 2 * n6 * n6 * n7 - 4 * n2 * n7 * n7 - 4 * n3 * n7 * n7 - 3 * n5 * n7 * n7 - 4 * n6 * n7 * n7
            + 2 * n1 * n8 - 4 * n1 * n1 * n8 - 2 * n1 * n2 * n8 + 2 * n3 * n8 - 2 * n2 * n3 * n8 - 4 * n3 * n3 * n8
            - n4 * n8 - n1 * n4 * n8 - 2 * n2 * n4 * n8 - n3 * n4 * n8 + n4 * n4 * n8 + n1 * n5 * n8 + n3 * n5 * n8
            - n6 * n8 - n1 * n6 * n8 - 2 * n2 * n6 * n8 - n3 * n6 * n8 - 2 * n4 * n6 * n8 + n6 * n6 * n8
            + 4 * n1 * n7 * n8 - 2 * n2 * n7 * n8 + 3 * n4 * n7 * n8 - n5 * n7 * n8 - n6 * n7 * n8
            + 2 * n1 * n8 * n8 + 2 * n3 * n8 * n8 + n4 * n8 * n8 + n6 * n8 * n8
            + 8 * n1 * n9 - 4 * n1 * n1 * n9 + 2 * n2 * n9 + 2 * n2 * n2 * n9 + 4 * n1 * n3 * n9 + 4 * n2 * n3 * n9
            + 2 * n4 * n9 - n2 * n4 * n9 + 2 * n4 * n4 * n9 + 2 * n5 * n9 + 2 * n1 * n5 * n9 + n2 * n5 * n9
            + 2 * n3 * n5 * n9 + n4 * n5 * n9 - n2 * n6 * n9 - 2 * n4 * n6 * n9 - n5 * n6 * n9
            + 4 * n1 * n7 * n9 + 4 * n3 * n7 * n9 + 4 * n4 * n7 * n9 + 2 * n5 * n7 * n9 + 4 * n6 * n7 * n9
            - 2 * n2 * n8 * n9 + 4 * n3 * n8 * n9 - n4 * n8 * n9 - n5 * n8 * n9 + 3 * n6 * n8 * n9
            - 4 * n1 * n9 * n9 - 4 * n2 * n9 * n9 - 4 * n4 * n9 * n9 - 3 * n5 * n9 * n9)


def geno_pi2_single_corr(g):
    """16x the correction part of genotype pi2(i,i,i,i) (genotype_kernels.py:377-403)."""
    n1, n2, n3, n4, n5, n6, n7, n8, n9 = g
    return (
        (13 * n2 * n4 - 16 * n1 * n2 * n4 - 11 * n2 * n2 * n4 + 16 * n3 * n4 - 28 * n1 * n3 * n4 - 24 * n2 * n3 * n4)
        + (-8 * n3 * n3 * n4 - 11 * n2 * n4 * n4 - 20 * n3 * n4 * n4 - 6 * n5 + 12 * n1 * n5 - 4 * n1 * n1 * n5 + 17 * n2 * n5)
        + (-20 * n1 * n2 * n5 - 11 * n2 * n2 * n5 + 12 * n3 * n5 - 28 * n1 * n3 * n5 - 20 * n2 * n3 * n5 - 4 * n3 * n3 * n5)
        + (17 * n4 * n5 - 20 * n1 * n4 * n5 - 32 * n2 * n4 * n5 - 40 * n3 * n4 * n5 - 11 * n4 * n4 * n5 + 11 * n5 * n5)
        + (-16 * n1 * n5 * n5 - 17 * n2 * n5 * n5 - 16 * n3 * n5 * n5 - 17 * n4 * n5 * n5 - 6 * n5 * n5 * n5 + 16 * n1 * n6 - 8 * n1 * n1 * n6)
        + (13 * n2 * n6 - 24 * n1 * n2 * n6 - 11 * n2 * n2 * n6 - 28 * n1 * n3 * n6 - 16 * n2 * n3 * n6 + 24 * n4 * n6)
        + (-36 * n1 * n4 * n6 - 38 * n2 * n4 * n6 - 36 * n3 * n4 * n6 - 20 * n4 * n4 * n6 + 17 * n5 * n6 - 40 * n1 * n5 * n6)
        + (-32 * n2 * n5 * n6 - 20 * n3 * n5 * n6 - 42 * n4 * n5 * n6 - 17 * n5 * n5 * n6 - 20 * n1 * n6 * n6 - 11 * n2 * n6 * n6)
        + (-20 * n4 * n6 * n6 - 11 * n5 * n6 * n6 + 16 * n2 * n7 - 28 * n1 * n2 * n7 - 20 * n2 * n2 * n7 + 16 * n3 * n7)
        + (-48 * n1 * n3 * n7 - 44 * n2 * n3 * n7 - 16 * n3 * n3 * n7 - 24 * n2 * n4 * n7 - 44 * n3 * n4 * n7)
        + (12 * n5 * n7 - 28 * n1 * n5 * n7 - 40 * n2 * n5 * n7 - 48 * n3 * n5 * n7 - 20 * n4 * n5 * n7 - 16 * n5 * n5 * n7)
        + (16 * n6 * n7 - 48 * n1 * n6 * n7 - 48 * n2 * n6 * n7 - 44 * n3 * n6 * n7 - 36 * n4 * n6 * n7 - 40 * n5 * n6 * n7)
        + (-20 * n6 * n6 * n7 - 8 * n2 * n7 * n7 - 16 * n3 * n7 * n7 - 4 * n5 * n7 * n7 - 8 * n6 * n7 * n7 + 16 * n1 * n8 - 8 * n1 * n1 * n8)
        + (24 * n2 * n8 - 36 * n1 * n2 * n8 - 20 * n2 * n2 * n8 + 16 * n3 * n8 - 48 * n1 * n3 * n8 - 36 * n2 * n3 * n8 - 8 * n3 * n3 * n8)
        + (13 * n4 * n8 - 24 * n1 * n4 * n8 - 38 * n2 * n4 * n8 - 48 * n3 * n4 * n8 - 11 * n4 * n4 * n8 + 17 * n5 * n8 - 40 * n1 * n5 * n8)
        + (-42 * n2 * n5 * n8 - 40 * n3 * n5 * n8 - 32 * n4 * n5 * n8 - 17 * n5 * n5 * n8 + 13 * n6 * n8 - 48 * n1 * n6 * n8)
        + (-38 * n2 * n6 * n8 - 24 * n3 * n6 * n8 - 38 * n4 * n6 * n8 - 32 * n5 * n6 * n8 - 11 * n6 * n6 * n8 - 28 * n1 * n7 * n8)
        + (-36 * n2 * n7 * n8 - 44 * n3 * n7 * n8 - 16 * n4 * n7 * n8 - 20 * n5 * n7 * n8 - 24 * n6 * n7 * n8 - 20 * n1 * n8 * n8)
        + (-20 * n2 * n8 * n8 - 20 * n3 * n8 * n8 - 11 * n4 * n8 * n8 - 11 * n5 * n8 * n8 - 11 * n6 * n8 * n8 + 16 * n1 * n9 - 16 * n1 * n1 * n9)
        + (16 * n2 * n9 - 44 * n1 * n2 * n9 - 20 * n2 * n2 * n9 - 48 * n1 * n3 * n9 - 28 * n2 * n3 * n9 + 16 * n4 * n9)
        + (-44 * n1 * n4 * n9 - 48 * n2 * n4 * n9 - 48 * n3 * n4 * n9 - 20 * n4 * n4 * n9 + 12 * n5 * n9 - 48 * n1 * n5 * n9)
        + (-40 * n2 * n5 * n9 - 28 * n3 * n5 * n9 - 40 * n4 * n5 * n9 - 16 * n5 * n5 * n9 - 44 * n1 * n6 * n9 - 24 * n2 * n6 * n9)
        + (-36 * n4 * n6 * n9 - 20 * n5 * n6 * n9 - 48 * n1 * n7 * n9 - 48 * n2 * n7 * n9 - 48 * n3 * n7 * n9 - 28 * n4 * n7 * n9)
        + (-28 * n5 * n7 * n9 - 28 * n6 * n7 * n9 - 44 * n1 * n8 * n9 - 36 * n2 * n8 * n9 - 28 * n3 * n8 * n9 - 24 * n4 * n8 * n9)
        + (-20 * n5 * n8 * n9 - 16 * n6 * n8 * n9 - 16 * n1 * n9 * n9 - 8 * n2 * n9 * n9 - 8 * n4 * n9 * n9 - 4 * n5 * n9 * n9))


def _ns_den4(x):
    ns = x.ns
    return ns * (ns - 1) * (ns - 2) * (ns - 3)


def _geno_dd(P, p):
    i, j = p
    if i == j:  # genotype_kernels.py:27-71
        x = P[i]
        num = geno_dd_single_num(x.g) / 16 + x.D * x.D
        den = _ns_den4(x)
        out = np.zeros_like(den)
        ok = x.ns >= 4
        out[ok] = 4 * num[ok] / den[ok]
        return out
    x, y = P[i], P[j]  # :73-81
    return _div(4 * x.D * y.D, x.n * (x.n - 1) * y.n * (y.n - 1))


def _raw_div(num, den):
    """Unguarded division, as in the genotype Dz cross-population kernels."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return num / den


def _geno_dz(P, p):
    p1, p2, p3 = p
    if p1 == p2 == p3:  # genotype_kernels.py:235-272
        x = P[p1]
        num = 0.25 * geno_dz_single_quartic(x.g) + x.A * x.Bv * x.D
        den = _ns_den4(x)
        out = np.zeros_like(den)
        ok = x.ns >= 4
        out[ok] = 2 * num[ok] / den[ok]
        return out
    if p1 == p2:  # :208-215 (I = p1, J = p3)
        x, y = P[p1], P[p3]
        return _raw_div(2 * x.U * y.A, y.ns * x.ns * (x.ns - 1) * (x.ns - 2))
    if p1 == p3:  # :217-224 (I = p1, J = p2)
        x, y = P[p1], P[p2]
        return _raw_div(2 * x.V * y.Bv, y.ns * x.ns * (x.ns - 1) * (x.ns - 2))
    if p2 == p3:  # :226-233 (I = p1, J = p2)
        x, y = P[p1], P[p2]
        return _raw_div(2 * x.D * y.Wjj, y.ns * (y.ns - 1) * x.ns * (x.ns - 1))
    x, y, z = P[p1], P[p2], P[p3]  # :199-206
    return _raw_div(2 * x.D * y.Bv * z.A, x.ns * (x.ns - 1) * y.ns * z.ns)


def geno_pi2_case(p):
    """Genotype pi2 case (genotype_kernels.py:738-762): triples split by position."""
    c = pi2_case(p)
    if c == "triple":
        t, _ = triple_roles(p)
        return "triple_iiij" if (p[0] == t and p[1] == t) else "triple_ijii"
    return c


def _geno_pi2(P, p):
    case = geno_pi2_case(p)
    i, j, k, l = p
    if case == "alldiff":  # genotype_kernels.py:279-284
        return 0.25 * (P[i].p * P[j].r + P[i].r * P[j].p) * (P[k].q * P[l].s + P[k].s * P[l].q)
    if case == "iikk":  # :286-291
        return P[i].BL * P[k].BR
    if case == "iikl":  # :293-299
        return P[i].BL * 0.5 * (P[k].q * P[l].s + P[k].s * P[l].q)
    if case == "ijkk":  # :301-307
        return 0.5 * (P[i].p * P[j].r + P[i].r * P[j].p) * P[k].BR
    if case == "shared":  # :309-317
        s, a, b = shared_roles(p)
        S, A, B = P[s], P[a], P[b]
        return A.r * (S.C00 * B.s + S.C01 * B.q) + A.p * (S.C10 * B.s + S.C11 * B.q)
    if case == "triple_iiij":  # :319-328
        t, s = triple_roles(p)
        T, S = P[t], P[s]
        return _div(T.AQ3 * S.pB + T.AS3 * S.qB, T.n * (T.n - 1) * (T.n - 2) * S.n)
    if case == "triple_ijii":  # :330-339
        t, s = triple_roles(p)
        T, S = P[t], P[s]
        return _div(T.BP3 * S.pA + T.BR3 * S.qA, T.n * (T.n - 1) * (T.n - 2) * S.n)
    if case == "ijij":  # :341-362
        X, Y = P[i], P[j]
        Pi, Qi, Ri, Si = X.pA, X.pB, X.qA, X.qB
        Pj, Qj, Rj, Sj = Y.pA, Y.pB, Y.qA, Y.qB
        X01i, X10i, X11i, Bi = X.x_Ab, X.x_aB, X.x_ab, X.Bsgn
        X01j, X10j, X11j, Bj = Y.x_Ab, Y.x_aB, Y.x_ab, Y.Bsgn
        PQi, PRi, PSi, QRi, RSi = Pi * Qi, Pi * Ri, Pi * Si, Qi * Ri, Ri * Si
        PQj, PSj, QRj, RSj = Pj * Qj, Pj * Sj, Qj * Rj, Rj * Sj
        Tc = Ri * (1.0 + X01i - X10i)
        Uc = Si * (1.0 + Ri)
        num = (-0.25 * RSi * Qj - 0.25 * X11i * PQj + 0.25 * RSi * PQj - 0.25 * Ri * PSj
               - 0.25 * PQi * X11j - 0.25 * RSi * X11j + 0.25 * PSi * X11j + 0.25 * QRi * X11j
               - 0.25 * PRi * Sj + 0.25 * Tc * Sj + 0.25 * X11i * PSj + 0.25 * QRi * PSj
               + 0.25 * Uc * Rj - 0.25 * X01i * QRj + 0.25 * PSi * QRj
               - 0.25 * PSi * Rj - 0.25 * Pi * RSj + 0.25 * X01i * RSj + 0.25 * PQi * RSj
               + 0.25 * X11i * Bj + 0.25 * Bi * X11j - 1.0 * X11i * X11j)
        return _div(num, X.n * (X.n - 1) * Y.n * (Y.n - 1))
    x = P[i]  # same: :364-405
    g1, g2, g3, g4, g5, g6, g7, g8, g9 = x.g
    a1 = g1 + g2 + g3 + 0.5 * g4 + 0.5 * g5 + 0.5 * g6
    a2 = g1 + 0.5 * g2 + g4 + 0.5 * g5 + g7 + 0.5 * g8
    a3 = 0.5 * g2 + g3 + 0.5 * g5 + g6 + 0.5 * g8 + g9
    a4 = 0.5 * g4 + 0.5 * g5 + 0.5 * g6 + g7 + g8 + g9
    num = a1 * a2 * a3 * a4 + geno_pi2_single_corr(x.g) / 16
    den = _ns_den4(x)
    out = np.zeros_like(den)
    ok = x.ns >= 4
    out[ok] = num[ok] / den[ok]
    return out


_GENO_KIND = {"dd": _geno_dd, "dz": _geno_dz, "pi2": _geno_pi2}


def geno_raw(kind, pops, P):
    return _GENO_KIND[kind](P, pops)


def geno_stats(counts_list, n_valid_list=None):
    """(N, n_stats) genotype-path statistics (genotype_kernels.py:881-936)."""
    Pn = len(counts_list)
    if n_valid_list is None:
        n_valid_list = [None] * Pn
    pops = [GenoPop(c, nv) for c, nv in zip(counts_list, n_valid_list)]
    cache = {}

    def raw(k, q):
        if (k, q) not in cache:
            cache[(k, q)] = geno_raw(k, q, pops)
        return cache[(k, q)]

    return assemble(stat_specs(Pn), raw)


def geno_dosage_r2(counts9):
    """Pairwise-complete dosage (Rogers-Huff) r^2 from the 9-cell table.

    Equals ``allel.rogers_huff_r`` squared when nothing is missing
    (ld_statistics.py:410-443); NaN where either locus is constant.
    """
    c = np.asarray(counts9, dtype=np.float64)
    a = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2], dtype=np.float64)
    b = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2], dtype=np.float64)
    n = c.sum(axis=1)
    sx, sy = c @ a, c @ b
    sxx, syy, sxy = c @ (a * a), c @ (b * b), c @ (a * b)
    vx = n * sxx - sx * sx
    vy = n * syy - sy * sy
    cov = n * sxy - sx * sy
    den = vx * vy
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(den > 0, cov * cov / np.where(den > 0, den, 1.0), np.nan)


# ---------------------------------------------------------------------------
# the binned parse  (moments_ld.py:248-343; haplotype_matrix.py:1592-1866)
# ---------------------------------------------------------------------------


def bin_sums(data, positions, pop_rows, edges, genotypes=False, chunk=200_000,
             max_dist=None, coords=None, pair_range=None, window_offsets=None,
             snp_block=None, n_blocks=1, anchor_end=None, stat_fn=None):
    """Per-bin sums of the moments-ordered statistics.

    Returns dict: ``sums`` (n_blocks, n_bins, n_stats), ``pairs`` (n_blocks, n_bins)
    pairs per bin, ``r2_sum`` / ``r2_count`` (n_blocks, n_bins) over pairs with finite
    r^2 (first population; dosage r^2 on the genotype path), and ``n_pairs`` (pairs
    generated, incl. dropped).  ``window_offsets`` restricts pairs to SNP windows;
    ``snp_block`` assigns each pair to the bootstrap block of its left SNP.

    ``coords`` (optional, per-SNP f64) replaces positions for binning, as the
    genetic-map path does (moments_ld.py:301-311); the pair cutoff still uses
    positions and ``max_dist``.  ``pair_range`` = (lo, hi) restricts to that slice of
    the anchor-ordered pair list (bounded CPU baselines).  ``anchor_end`` (one per window)
    keeps only the pairs whose left SNP lies before it (a rank's share of a split parse).
    ``stat_fn`` replaces the statistics function (``hap_stats`` signature), e.g. pg_gpu's
    own kernels through ``oracle.ref_kernels.hap_stats``.
    """
    edges = np.asarray(edges, dtype=np.float64)
    nb = len(edges) - 1
    Pn = len(pop_rows)
    n_stats = len(ld_names(Pn))
    max_dist = float(edges[-1]) if max_dist is None else float(max_dist)
    positions = np.asarray(positions)
    if window_offsets is None:
        window_offsets = [0, len(positions)]
    iis, jjs = [], []
    for w, (a, b) in enumerate(zip(window_offsets[:-1], window_offsets[1:])):
        ii, jj = pairs_within_distance(positions[a:b], max_dist)
        if anchor_end is not None:
            keep = ii + a < anchor_end[w]
            ii, jj = ii[keep], jj[keep]
        iis.append(ii + a)
        jjs.append(jj + a)
    ii = np.concatenate(iis) if iis else np.empty(0, np.int64)
    jj = np.concatenate(jjs) if jjs else np.empty(0, np.int64)
    if pair_range is not None:
        ii, jj = ii[pair_range[0]:pair_range[1]], jj[pair_range[0]:pair_range[1]]
    blk_of = (np.zeros(len(positions), np.int64) if snp_block is None
              else np.asarray(snp_block, np.int64))
    out = {"sums": np.zeros((n_blocks, nb, n_stats)), "pairs": np.zeros((n_blocks, nb), np.int64),
           "r2_sum": np.zeros((n_blocks, nb)), "r2_count": np.zeros((n_blocks, nb), np.int64),
           "n_pairs": len(ii)}
    coord = np.asarray(positions if coords is None else coords, dtype=np.float64)
    count_fn = geno_counts if genotypes else hap_counts
    stat_fn = stat_fn or (geno_stats if genotypes else hap_stats)
    for s in range(0, len(ii), chunk):
        ci, cj = ii[s:s + chunk], jj[s:s + chunk]
        d = np.abs(coord[cj] - coord[ci])
        cb = bin_index(d, edges)
        cl, nl = [], []
        for rows in pop_rows:
            c, nv = count_fn(data, ci, cj, rows)
            cl.append(c)
            nl.append(nv)
        st = stat_fn(cl, nl)
        keep = (cb >= 0) & (cb < nb)
        flat = blk_of[ci[keep]] * nb + cb[keep]
        np.add.at(out["sums"].reshape(-1, n_stats), flat, st[keep])
        out["pairs"] += np.bincount(flat, minlength=n_blocks * nb).reshape(n_blocks, nb)
        r2 = geno_dosage_r2(cl[0]) if genotypes else hap_r_squared(cl[0], nl[0])
        r2 = r2[keep]
        fin = np.isfinite(r2)
        np.add.at(out["r2_sum"].reshape(-1), flat[fin], r2[fin])
        out["r2_count"] += np.bincount(flat[fin], minlength=n_blocks * nb).reshape(n_blocks, nb)
    return out


def heterozygosity(data, pop_rows, genotypes=False):
    """H_i_j sums over sites (moments_ld.py:346-388)."""
    alt, ref, nh = [], [], []
    for rows in pop_rows:
        x = np.asarray(data)[np.asarray(rows)]
        if genotypes:
            v = x >= 0
            a = np.where(v, x, 0).astype(np.int64).sum(axis=0).astype(np.float64)
            n = 2.0 * v.sum(axis=0).astype(np.float64)
        else:
            a = np.maximum(x, 0).astype(np.int64).sum(axis=0).astype(np.float64)
            n = np.full_like(a, float(len(rows)))
        alt.append(a)
        ref.append(n - a)
        nh.append(n)
    out = {}
    P = len(pop_rows)
    for i in range(P):
        for j in range(i, P):
            if i == j:
                v = np.sum(2.0 * ref[i] * alt[i] / (nh[i] * (nh[i] - 1)))
            else:
                v = np.sum((ref[i] * alt[j] + alt[i] * ref[j]) / (nh[i] * nh[j]))
            out[f"H_{i}_{j}"] = float(v)
    return out


def biallelic_keep(hap):
    """Sites with both alleles present and nothing >= 2 (haplotype_matrix.py:724-789)."""
    h = np.asarray(hap)
    return (np.sum(h >= 2, axis=0) == 0) & (np.sum(h == 0, axis=0) > 0) & (np.sum(h == 1, axis=0) > 0)


def geno_biallelic_keep(geno, rows_union=None):
    """Genotype-path filter over the union of pops (moments_ld.py:256-278)."""
    g = np.asarray(geno)
    if rows_union is not None:
        g = g[np.asarray(sorted(set(int(r) for r in rows_union)))]
    v = g >= 0
    alt = np.where(v, g, 0).astype(np.int64).sum(axis=0)
    nv = v.sum(axis=0)
    return (alt > 0) & (alt < 2 * nv) & (nv >= 2)


# ---------------------------------------------------------------------------
# all-pairs LD of one SNP set: pairwise r^2, sigma_D^2, r^2 from joint counts, ZnS, Omega,
# windowed r^2 percentiles  (haplotype_matrix.py:1092-1317, ld_statistics.py:249-862)
# ---------------------------------------------------------------------------


def segregating(hap, missing_data="include"):
    """Column indices kept by ``_prepare_segregating`` (ld_statistics.py:249-278):
    with 'exclude' only sites without missing calls, then sites with 0 < dac < n_valid."""
    hap = np.asarray(hap)
    keep = np.arange(hap.shape[1])
    if missing_data == "exclude":
        keep = keep[np.sum(hap < 0, axis=0) == 0]
    sub = hap[:, keep]
    dac = np.maximum(sub, 0).sum(axis=0)
    nv = (sub >= 0).sum(axis=0)
    return keep[(dac > 0) & (dac < nv)]


def _gram_counts(hap):
    """c1..c4 and n (joint valid) for all column pairs (ld_statistics.py:281-299)."""
    v = (hap >= 0).astype(np.float64)
    h = np.where(hap >= 0, hap, 0).astype(np.float64)
    c1 = h.T @ h
    s12 = h.T @ v
    s13 = v.T @ h
    n = v.T @ v
    return c1, s12 - c1, s13 - c1, n - s12 - s13 + c1, n


def pairwise_r2_matrix(hap):
    """``HaplotypeMatrix.pairwise_r2('r2')`` (haplotype_matrix.py:1092-1136, 1171-1175):
    D = p_AB - p_i p_j with p_AB over jointly valid haplotypes and p_i over the site's valid
    haplotypes; r^2 = D^2 / (p_i q_i p_j q_j), 0 where that product is 0; diagonal 0."""
    hap = np.asarray(hap)
    v = (hap >= 0).astype(np.float64)
    h = np.where(hap >= 0, hap, 0).astype(np.float64)
    nv = v.sum(axis=0)
    p = np.where(nv > 0, h.sum(axis=0) / np.where(nv > 0, nv, 1), 0.0)
    jn = v.T @ v
    j11 = h.T @ h
    pab = np.where(jn > 0, j11 / np.where(jn > 0, jn, 1), 0.0)
    D = pab - np.outer(p, p)
    den = np.outer(p * (1 - p), p * (1 - p))
    r2 = np.where(den > 0, D ** 2 / np.where(den > 0, den, 1), 0.0)
    np.fill_diagonal(r2, 0.0)
    return r2


def sigma_d2_matrix(hap):
    """Unbiased sigma_D^2 = D^2 / pi2 numerators per pair (ld_statistics.py:311-344,
    788-810): 0 where n < 4 or the pi2 numerator is 0; diagonal 0.  Also returns the
    valid mask n >= 4 (diagonal False) that ZnS counts."""
    c1, c2, c3, c4, n = _gram_counts(np.asarray(hap))
    dd = c1 * (c1 - 1) * c4 * (c4 - 1) + c2 * (c2 - 1) * c3 * (c3 - 1) - 2 * c1 * c2 * c3 * c4
    s12, s13, s24, s34 = c1 + c2, c1 + c3, c2 + c4, c3 + c4
    pi2 = (s12 * s13 * s24 * s34 - c1 * c4 * (-1 + c1 + 3 * c2 + 3 * c3 + c4)
           - c2 * c3 * (-1 + 3 * c1 + c2 + c3 + 3 * c4))
    valid = n >= 4
    out = np.where(valid & (pi2 != 0), dd / np.where(pi2 != 0, pi2, 1), 0.0)
    np.fill_diagonal(out, 0.0)
    np.fill_diagonal(valid, False)
    return out, valid


def r2_counts_matrix(hap):
    """r^2 from the jointly valid two-locus counts for every pair, the estimator of
    ``ld_statistics.r_squared`` (haplotype_kernels.py:32-42) that ``windowed_r_squared``
    applies to every pair (haplotype_matrix.py:1285-1289): NaN where pA qA pB qB = 0;
    diagonal NaN."""
    c1, c2, c3, c4, n = _gram_counts(np.asarray(hap))
    with np.errstate(divide="ignore", invalid="ignore"):
        D = c1 * c4 - c2 * c3
        den = (c1 + c2) * (c3 + c4) * (c1 + c3) * (c2 + c4)
        r2 = np.where(den > 0, D * D / np.where(den > 0, den, 1), np.nan)
    np.fill_diagonal(r2, np.nan)
    return r2


def zns(hap, estimator="sigma_d2", missing_data="include"):
    """Kelly's ZnS on segregating sites (ld_statistics.py:534-596, 679-718): mean naive
    pairwise r^2 over the m(m-1)/2 pairs, or mean sigma_D^2 over pairs with n >= 4.  With
    the sigma_D^2 estimator the reference replaces ``missing_data`` by its internal
    projection mode (ld_statistics.py:711), so 'exclude' is not applied there."""
    if estimator != "r2":
        missing_data = "include"
    sub = np.asarray(hap)[:, segregating(hap, missing_data)]
    m = sub.shape[1]
    if m < 2:
        return 0.0
    if estimator == "r2":
        r2 = pairwise_r2_matrix(sub)
        return float(r2.sum() / (m * (m - 1)))
    sd, valid = sigma_d2_matrix(sub)
    npairs = int(valid.sum())
    return float(sd.sum() / npairs) if npairs > 0 else 0.0


def omega(hap, estimator="sigma_d2", missing_data="include"):
    """Kim & Nielsen's Omega on segregating sites (ld_statistics.py:761-862): max over
    split points l = 3 .. m-2 of mean within-block / mean cross-block value, upper
    triangle pairs only; 0 if fewer than 5 sites."""
    sub = np.asarray(hap)[:, segregating(hap, missing_data)]
    m = sub.shape[1]
    if m < 5:
        return 0.0
    mat = pairwise_r2_matrix(sub) if estimator == "r2" else sigma_d2_matrix(sub)[0]
    up = np.triu(mat, k=1)
    best = 0.0
    for l in range(3, m - 1):
        left = up[:l, :l].sum()
        cross = up[:l, l:].sum()
        right = up[l:, l:].sum()
        n_within = l * (l - 1) // 2 + (m - l) * (m - l - 1) // 2
        n_cross = l * (m - l)
        if n_within > 0 and n_cross > 0 and cross > 0:
            best = max(best, ((left + right) / n_within) / (cross / n_cross))
    return float(best)


def windowed_r2(hap, positions, bp_bins, percentile=50):
    """``HaplotypeMatrix.windowed_r_squared`` with the 'r2' estimator
    (haplotype_matrix.py:1235-1317): r^2 from joint counts for every pair i < j, binned by
    pos[j] - pos[i] with digitize (right-open), NaN pairs dropped; per-bin percentiles
    (NaN for empty bins) and pair counts."""
    r2 = r2_counts_matrix(hap)
    pos = np.asarray(positions)
    m = len(pos)
    iu, ju = np.triu_indices(m, k=1)
    vals = r2[iu, ju]
    dist = pos[ju] - pos[iu]
    edges = np.asarray(bp_bins)
    nb = len(edges) - 1
    b = np.digitize(dist, edges) - 1
    ok = (b >= 0) & (b < nb) & ~np.isnan(vals)
    pct = np.atleast_1d(percentile)
    res = np.full((nb, len(pct)), np.nan)
    cnt = np.zeros(nb, dtype=int)
    for k in range(nb):
        sel = vals[ok & (b == k)]
        cnt[k] = len(sel)
        if len(sel):
            res[k] = np.percentile(sel, pct)
    return (res[:, 0] if res.shape[1] == 1 else res), cnt


def _geno_cells_all_pairs(geno):
    """Nine-cell counts n_ab (a = g_i, b = g_j, both valid) for all column pairs, as the
    list [n00, n01, ..., n22] of (m, m) arrays (ld_pipeline.py:183-263 column order)."""
    g = np.asarray(geno)
    ind = [(g == a).astype(np.float64) for a in range(3)]
    return [ind[a].T @ ind[b] for a in range(3) for b in range(3)]


def rogers_huff_r(geno):
    """Condensed upper-triangle Rogers-Huff r of dosages without missing calls
    (ld_statistics.py:392-524): cov = g_i . g_j - n mu_i mu_j, r = cov / sqrt(ssd_i ssd_j),
    NaN where either site is constant."""
    g = np.asarray(geno, dtype=np.float64)
    n = g.shape[0]
    mu = g.mean(axis=0)
    ssd = ((g - mu) ** 2).sum(axis=0)
    cov = g.T @ g - n * np.outer(mu, mu)
    den = np.sqrt(np.outer(ssd, ssd))
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den > 0, cov / np.where(den > 0, den, 1), np.nan)
    iu = np.triu_indices(g.shape[1], k=1)
    return r[iu]


def diploid_r2_matrix(geno):
    """Dosage r^2 with missing calls (ld_statistics.py:973-1021): dosages centred on the
    site's valid mean and zeroed where missing, cov = gn_i . gn_j, r^2 = cov^2 / (var_i
    var_j), 0 where that product is 0; diagonal 0."""
    g = np.asarray(geno)
    v = (g >= 0).astype(np.float64)
    gc = np.where(g >= 0, g, 0).astype(np.float64)
    nv = v.sum(axis=0)
    mean = np.where(nv > 0, gc.sum(axis=0) / np.where(nv > 0, nv, 1), 0.0)
    gn = (gc - mean[None, :]) * v
    var = (gn ** 2).sum(axis=0)
    cov = gn.T @ gn
    den = np.sqrt(np.outer(var, var))
    r2 = np.where(den > 0, (cov / np.where(den > 0, den, 1)) ** 2, 0.0)
    np.fill_diagonal(r2, 0.0)
    return r2


def sigma_d2_geno(geno):
    """Condensed upper-triangle unbiased sigma_D^2 of genotype pairs (genotype_kernels.py:
    91-170, ld_statistics_genotype.py:1518-1598): DD numerator over pi2 numerator (their
    denominators cancel), NaN where fewer than 4 individuals or the pi2 numerator <= 0."""
    cells = _geno_cells_all_pairs(geno)
    iu = np.triu_indices(np.asarray(geno).shape[1], k=1)
    c = np.stack([x[iu] for x in cells], axis=1)
    n1, n2, n3, n4, n5, n6, n7, n8, n9 = to_moments_order(c)
    ns = n1 + n2 + n3 + n4 + n5 + n6 + n7 + n8 + n9
    Dg = (-(0.5 * n2 + n3 + 0.25 * n5 + 0.5 * n6) * (0.5 * n4 + 0.25 * n5 + n7 + 0.5 * n8)
          + (n1 + 0.5 * n2 + 0.5 * n4 + 0.25 * n5) * (0.25 * n5 + 0.5 * n6 + 0.5 * n8 + n9))
    g9 = [n1, n2, n3, n4, n5, n6, n7, n8, n9]
    dd = (geno_dd_single_num(g9) / 16.0 + Dg * Dg) * 4.0
    a1 = n1 + n2 + n3 + 0.5 * n4 + 0.5 * n5 + 0.5 * n6
    a2 = n1 + 0.5 * n2 + n4 + 0.5 * n5 + n7 + 0.5 * n8
    a3 = 0.5 * n2 + n3 + 0.5 * n5 + n6 + 0.5 * n8 + n9
    a4 = 0.5 * n4 + 0.5 * n5 + 0.5 * n6 + n7 + n8 + n9
    pi2 = a1 * a2 * a3 * a4 + geno_pi2_single_corr(g9) / 16.0
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.where((ns >= 4) & (pi2 > 0), dd / np.where(pi2 > 0, pi2, 1), np.nan)
    return out


def zns_diploid(geno):
    """ZnS of a GenotypeMatrix (ld_statistics.py:679-735 via _resolve_r2_matrix, :926-972):
    mean off-diagonal dosage r^2."""
    r2 = diploid_r2_matrix(geno)
    m = r2.shape[0]
    return 0.0 if m < 2 else float((r2.sum() - np.trace(r2)) / (m * (m - 1)))


def omega_diploid(geno):
    """Omega of a GenotypeMatrix on its dosage r^2 matrix (ld_statistics.py:761-862)."""
    r2 = diploid_r2_matrix(geno)
    m = r2.shape[0]
    if m < 5:
        return 0.0
    up = np.triu(r2, k=1)
    best = 0.0
    for l in range(3, m - 1):
        left, cross, right = up[:l, :l].sum(), up[:l, l:].sum(), up[l:, l:].sum()
        n_within = l * (l - 1) // 2 + (m - l) * (m - l - 1) // 2
        n_cross = l * (m - l)
        if n_within > 0 and n_cross > 0 and cross > 0:
            best = max(best, ((left + right) / n_within) / (cross / n_cross))
    return float(best)
