"""pg_gpu's ``ld_statistics`` call surface for the two-locus estimators
(``pg_gpu/ld_statistics.py:13-246``) on libldk.

``dd`` / ``dz`` / ``pi2`` accept haplotype counts (N, 4P) (any numeric dtype; evaluated in
float64 -- the reference's own int32 path overflows for large samples) with the
reference's ``populations`` and ``n_valid`` conventions (an (N,) array, an (N, P) array or
a tuple of per-population arrays).  Each call runs one raw-estimator kernel of libldk;
pi2(i,i,k,k) with i != k is, as in ``ld_statistics._pi2_multi``, the average of the two
orientations.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .csrc import gen_estimators as G


def _as_f64(x):
    torch = _lib.require_cuda()
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=torch.float64).contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device="cuda").contiguous()


def _n_valid_matrix(n_valid, counts, P):
    """(N, P) float64 n_valid following ld_statistics._get_pop_data (:1079-1112)."""
    torch = _lib.require_cuda()
    if n_valid is None:
        return None
    N = counts.shape[0]
    cols = []
    for p in range(P):
        if isinstance(n_valid, tuple):
            v = n_valid[p] if p < len(n_valid) and n_valid[p] is not None else counts[:, 4 * p:4 * p + 4].sum(1)
        elif _as_f64(n_valid).dim() == 2:
            v = _as_f64(n_valid)[:, p]
        else:
            v = n_valid
        cols.append(_as_f64(v).reshape(N))
    return torch.stack(cols, dim=1).contiguous()


def _raw(case, args, counts, nv, P):
    torch = _lib.require_cuda()
    lib = _lib.load()
    N = counts.shape[0]
    out = torch.empty(N, dtype=torch.float64, device="cuda")
    a = (ctypes.c_int32 * 4)(*(list(args) + [0] * (4 - len(args))))
    _lib.check(lib.ldk_raw_hap(G.RAW_CASES.index(case), a, P, _lib.ptr(counts), _lib.ptr(nv), N, _lib.ptr(out),
                               _lib.stream_handle()))
    return out


def _prepare(counts, n_valid):
    c = _as_f64(counts)
    if c.dim() != 2 or c.shape[1] % 4:
        raise ValueError("counts must be (N, 4*P)")
    P = c.shape[1] // 4
    return c, _n_valid_matrix(n_valid, c, P), P


def dd(counts, populations=None, n_valid=None):
    """D^2 (ld_statistics.py:13-62)."""
    c, nv, P = _prepare(counts, n_valid)
    if populations is None:
        return _raw("dd1", (0,), c, nv, P)
    i, j = populations
    if i == j:
        return _raw("dd1", (i,), c, nv, P)
    if isinstance(n_valid, tuple):
        # ld_statistics._dd_between reads n_valid[0] and n_valid[1] of a tuple whatever the
        # population indices (:1143-1147)
        nv = nv.clone()
        a = n_valid[0] if n_valid[0] is not None else c[:, 4 * i:4 * i + 4].sum(1)
        b = n_valid[1] if len(n_valid) > 1 and n_valid[1] is not None else c[:, 4 * j:4 * j + 4].sum(1)
        nv[:, i] = _as_f64(a).reshape(-1)
        nv[:, j] = _as_f64(b).reshape(-1)
    return _raw("dd2", (i, j), c, nv, P)


def dz(counts, populations=None, n_valid=None):
    """Dz (ld_statistics.py:65-94)."""
    c, nv, P = _prepare(counts, n_valid)
    pops = (0, 0, 0) if populations is None else tuple(populations)
    case, args = G.canonical("dz", pops)
    return _raw(case, args, c, nv, P)


def pi2(counts, populations=None, n_valid=None):
    """pi2 (ld_statistics.py:97-129, 1296-1617)."""
    c, nv, P = _prepare(counts, n_valid)
    pops = (0, 0, 0, 0) if populations is None else tuple(populations)
    case, args = G.canonical("pi2", pops)
    if case == "pi2_iikk":
        i, k = args
        return 0.5 * (_raw(case, (i, k), c, nv, P) + _raw(case, (k, i), c, nv, P))
    return _raw(case, args, c, nv, P)


def dd_within(counts, n_valid=None):
    return dd(counts, None, n_valid)


def dd_between(counts, pop1_idx, pop2_idx, n_valid=None):
    return dd(counts, (pop1_idx, pop2_idx), n_valid)


def _r_family(which, counts, n_valid):
    torch = _lib.require_cuda()
    lib = _lib.load()
    c = _as_f64(counts).reshape(-1, 4).contiguous()
    nv = None if n_valid is None else _as_f64(n_valid).reshape(-1)
    out = torch.empty(c.shape[0], dtype=torch.float64, device="cuda")
    _lib.check(lib.ldk_r_family(which, _lib.ptr(c), _lib.ptr(nv), c.shape[0], _lib.ptr(out), _lib.stream_handle()))
    return out


def r(counts, n_valid=None):
    """Pearson r per pair; NaN where a locus is monomorphic (ld_statistics.py:153-172)."""
    return _r_family(0, counts, n_valid)


def r_squared(counts, n_valid=None):
    """r^2 per pair; NaN where undefined (ld_statistics.py:194-217)."""
    return _r_family(1, counts, n_valid)


def d_prime(counts, n_valid=None):
    """Lewontin's D' per pair (ld_statistics.py:220-246)."""
    return _r_family(2, counts, n_valid)


def zns(r2_matrix_or_matrix, missing_data="include", estimator="auto"):
    """Kelly's ZnS (ld_statistics.py:679-718): a HaplotypeMatrix goes through the
    all-pairs kernel (no matrix is materialised); a precomputed square r^2 matrix gives
    (sum - trace) / (m (m - 1))."""
    from .haplotype_matrix import HaplotypeMatrix
    from . import ld_matrix
    if isinstance(r2_matrix_or_matrix, HaplotypeMatrix):
        r2_matrix_or_matrix.transfer_to_gpu()
        return ld_matrix.zns(r2_matrix_or_matrix.haplotypes, missing_data, estimator)
    if estimator == "sigma_d2":
        raise ValueError("estimator='sigma_d2' requires a HaplotypeMatrix, not a pre-computed r^2 array")
    if hasattr(r2_matrix_or_matrix, "genotypes"):  # GenotypeMatrix: dosage r^2 (ld_statistics.py:926-972)
        if estimator not in ("auto", "r2", "rogers_huff"):
            raise ValueError(f"Unknown estimator: {estimator!r}")
        r2_matrix_or_matrix.transfer_to_gpu()
        return ld_matrix.zns_diploid(r2_matrix_or_matrix.genotypes, missing_data)
    torch = _lib.require_cuda()
    M = torch.as_tensor(r2_matrix_or_matrix, dtype=torch.float64, device="cuda")
    m = M.shape[0]
    if m < 2:
        return 0.0
    return float(((M.sum() - torch.trace(M)) / (m * (m - 1))).item())


def omega(r2_matrix_or_matrix, missing_data="include", estimator="auto"):
    """Kim & Nielsen's Omega (ld_statistics.py:761-862) of a HaplotypeMatrix (all-pairs
    kernel on its segregating sites) or of a precomputed r^2 matrix."""
    from .haplotype_matrix import HaplotypeMatrix
    from . import ld_matrix
    if isinstance(r2_matrix_or_matrix, HaplotypeMatrix):
        r2_matrix_or_matrix.transfer_to_gpu()
        return ld_matrix.omega(r2_matrix_or_matrix.haplotypes, missing_data, estimator)
    if estimator == "sigma_d2":
        raise ValueError("estimator='sigma_d2' requires a HaplotypeMatrix")
    if hasattr(r2_matrix_or_matrix, "genotypes"):  # GenotypeMatrix: dosage r^2 (ld_statistics.py:926-972)
        if estimator not in ("auto", "r2", "rogers_huff"):
            raise ValueError(f"Unknown estimator: {estimator!r}")
        r2_matrix_or_matrix.transfer_to_gpu()
        return ld_matrix.omega_from_matrix(ld_matrix.diploid_r2_matrix(r2_matrix_or_matrix.genotypes, missing_data))
    return ld_matrix.omega_from_matrix(r2_matrix_or_matrix)


def rogers_huff_r(matrix, tile_size=None):
    """Condensed Rogers-Huff r of a HaplotypeMatrix (paired haplotypes) or GenotypeMatrix
    (ld_statistics.py:492-521); ``tile_size`` is accepted for call compatibility."""
    from . import ld_matrix
    return ld_matrix.rogers_huff_r(matrix)


def rogers_huff_r_squared(matrix, tile_size=None):
    """Squared ``rogers_huff_r`` (ld_statistics.py:524-531)."""
    from . import ld_matrix
    return ld_matrix.rogers_huff_r_squared(matrix)
