"""All-pairs LD of one SNP set on libldk (``ldk_ld_matrix``): pg_gpu's pairwise r^2, the
unbiased sigma_D^2 matrix, r^2 from jointly valid counts, and the statistics built on
them -- Kelly's ZnS, Kim & Nielsen's Omega, windowed r^2 percentiles.

Mirrors ``HaplotypeMatrix.pairwise_r2`` / ``windowed_r_squared``
(``pg_gpu/haplotype_matrix.py:1092-1317``) and ``ld_statistics.zns`` / ``omega``
(``pg_gpu/ld_statistics.py:249-862``) for haplotype input.  Counts come from the INT8
tensor-core Gram pipeline, values are FP64; ZnS needs no matrix (the kernel reduces).
"""
from __future__ import annotations

import numpy as np

from . import _lib

ESTIMATORS = {"r2": 0, "sigma_d2": 1, "r2_counts": 2,                          # haplotypes
              "diploid_r2": 3, "rogers_huff_r": 4, "sigma_d2_geno": 5}           # genotypes


def _hap_tensor(hap, torch):
    if isinstance(hap, torch.Tensor):
        return hap.to(device="cuda", dtype=torch.int8).contiguous()
    return torch.as_tensor(np.ascontiguousarray(hap), dtype=torch.int8, device="cuda")


def ld_matrix(hap, rows=None, estimator="r2", matrix=True, reduce=False, stream=None):
    """All-pairs LD of the SNPs (columns) of ``hap`` over ``rows`` (default: all rows).

    Returns ``(M, sums)``: ``M`` the (n_var, n_var) float64 matrix (or None) and ``sums``
    the float64 tensor [sum over pairs i < j entering ZnS's mean, their count] (or None).
    ``estimator``: haplotypes "r2" (pairwise_r2), "sigma_d2", "r2_counts"; genotypes
    "diploid_r2", "rogers_huff_r", "sigma_d2_geno" (see ``ldk_ld_matrix``)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    X = _hap_tensor(hap, torch)
    n_rows, n_var = X.shape
    r = np.arange(n_rows) if rows is None else np.asarray(rows, dtype=np.int64).ravel()
    if r.size == 0:
        raise ValueError("no rows selected")
    if r.min() < 0 or r.max() >= n_rows:
        raise IndexError("row index out of range")
    R = torch.as_tensor(r.astype(np.int32), device="cuda")
    est = ESTIMATORS[estimator]
    M = torch.empty((n_var, n_var), dtype=torch.float64, device="cuda") if matrix else None
    S = torch.zeros(2, dtype=torch.float64, device="cuda") if reduce else None
    ws_bytes = lib.ldk_ld_matrix_workspace_size(n_var, len(r))
    ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device="cuda")
    _lib.check(lib.ldk_ld_matrix(_lib.ptr(X), n_var, n_var, _lib.ptr(R), len(r), est, _lib.ptr(M),
                                 n_var, _lib.ptr(S), _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream)))
    return M, S


def segregating(hap, missing_data="include"):
    """Column indices (int64 tensor) kept by ``_prepare_segregating``
    (ld_statistics.py:249-278): with 'exclude' only sites without missing calls, then
    sites with 0 < derived count < valid count."""
    torch = _lib.require_cuda()
    X = _hap_tensor(hap, torch)
    keep = torch.arange(X.shape[1], device="cuda")
    if missing_data == "exclude":
        keep = keep[(X < 0).sum(0) == 0]
    sub = X.index_select(1, keep)
    dac = sub.clamp(min=0).to(torch.int64).sum(0)
    nv = (sub >= 0).sum(0)
    return keep[(dac > 0) & (dac < nv)]


def _resolve(estimator):
    """'auto' means sigma_d2 for haplotype input (ld_statistics.py:347-364)."""
    if estimator == "auto":
        return "sigma_d2"
    if estimator not in ("r2", "sigma_d2"):
        raise ValueError(f"Unknown estimator: {estimator!r} (expected 'auto', 'r2' or 'sigma_d2')")
    return estimator


def zns(hap, missing_data="include", estimator="auto"):
    """Kelly's ZnS over segregating sites (ld_statistics.py:534-596, 679-718): mean
    pairwise r^2, or mean sigma_D^2 over pairs with at least 4 jointly valid haplotypes.
    As in the reference, ``missing_data`` applies to the r^2 estimator only (the
    sigma_D^2 path takes the reference's internal projection mode, :711)."""
    torch = _lib.require_cuda()
    est = _resolve(estimator)
    X = _hap_tensor(hap, torch)
    seg = segregating(X, missing_data if est == "r2" else "include")
    m = int(seg.numel())
    if m < 2:
        return 0.0
    _, S = ld_matrix(X.index_select(1, seg), estimator=est, matrix=False, reduce=True)
    total, count = S.tolist()
    if est == "r2":
        return total / (m * (m - 1) / 2)
    return total / count if count > 0 else 0.0


def omega(hap, missing_data="include", estimator="auto"):
    """Kim & Nielsen's Omega over segregating sites (ld_statistics.py:761-862): the
    largest ratio of mean within-block to mean cross-block value over split points
    l = 3 .. m-2, upper-triangle pairs, evaluated with 2-D prefix sums."""
    torch = _lib.require_cuda()
    est = _resolve(estimator)
    X = _hap_tensor(hap, torch)
    seg = segregating(X, missing_data)
    m = int(seg.numel())
    if m < 5:
        return 0.0
    M, _ = ld_matrix(X.index_select(1, seg), estimator=est)
    return omega_from_matrix(M)


def omega_from_matrix(M):
    """Omega of a precomputed (m, m) LD matrix (ld_statistics.py:814-862); 0 below 5 sites."""
    torch = _lib.require_cuda()
    M = torch.as_tensor(M, dtype=torch.float64, device="cuda")
    m = M.shape[0]
    if m < 5:
        return 0.0
    up = torch.triu(M, diagonal=1)
    S = torch.cumsum(torch.cumsum(up, dim=0), dim=1)
    lv = torch.arange(3, m - 1, device="cuda")
    left = S[lv - 1, lv - 1]
    total = S[m - 1, m - 1]
    cross = S[lv - 1, m - 1] - left
    right = total - left - cross
    lf = lv.to(torch.float64)
    n_within = lf * (lf - 1) / 2 + (m - lf) * (m - lf - 1) / 2
    n_cross = lf * (m - lf)
    ok = (n_within > 0) & (n_cross > 0) & (cross > 0)
    mean_within = torch.where(n_within > 0, (left + right) / n_within.clamp(min=1), torch.zeros_like(left))
    mean_cross = torch.where(n_cross > 0, cross / n_cross.clamp(min=1), torch.ones_like(cross))
    vals = torch.where(ok, mean_within / mean_cross, torch.zeros_like(left))
    return float(vals.max().item())


def windowed_r_squared(hap, positions, bp_bins, percentile=50, rows=None):
    """Percentiles of r^2 (jointly valid counts) over all pairs per distance bin and the
    pair counts (haplotype_matrix.py:1235-1317): bins right-open as ``digitize``, pairs
    with undefined r^2 dropped, NaN for empty bins; one column per percentile (squeezed
    for a single percentile)."""
    torch = _lib.require_cuda()
    X = _hap_tensor(hap, torch)
    m = X.shape[1]
    M, _ = ld_matrix(X, rows=rows, estimator="r2_counts")
    pos = torch.as_tensor(np.asarray(positions, dtype=np.float64), device="cuda")
    iu = torch.triu_indices(m, m, offset=1, device="cuda")
    vals = M[iu[0], iu[1]]
    dist = pos[iu[1]] - pos[iu[0]]
    edges = torch.as_tensor(np.asarray(bp_bins, dtype=np.float64), device="cuda")
    nb = len(bp_bins) - 1
    b = torch.bucketize(dist, edges, right=True) - 1
    ok = (b >= 0) & (b < nb) & ~torch.isnan(vals)
    vals, b = vals[ok], b[ok]
    pct = np.atleast_1d(np.asarray(percentile, dtype=np.float64))
    q = torch.as_tensor(pct / 100.0, device="cuda")
    res = np.full((nb, len(pct)), np.nan)
    cnt = torch.bincount(b, minlength=nb).cpu().numpy().astype(int)
    for k in range(nb):
        if cnt[k]:
            res[k] = torch.quantile(vals[b == k], q).cpu().numpy()
    return (res[:, 0] if res.shape[1] == 1 else res), cnt


# ---------------------------------------------------------------------------
# genotype input (ld_statistics.py:371-531, 973-1021; ld_statistics_genotype.py:1518-1598)
# ---------------------------------------------------------------------------


def dosages(matrix):
    """(n_individuals, n_variants) int8 dosages of a GenotypeMatrix, or of a HaplotypeMatrix
    with adjacent haplotypes paired (ld_statistics.py:371-409); missing calls raise, as in
    the reference's Rogers-Huff and sigma_D^2 genotype functions."""
    torch = _lib.require_cuda()
    from .genotype_matrix import GenotypeMatrix
    from .haplotype_matrix import HaplotypeMatrix
    if isinstance(matrix, HaplotypeMatrix):
        matrix.transfer_to_gpu()
        hap = matrix.haplotypes
        if bool((hap < 0).any()):
            raise ValueError("input HaplotypeMatrix contains missing values (-1); drop or impute missing sites first")
        if hap.shape[0] % 2:
            raise ValueError(f"HaplotypeMatrix has an odd number of haplotypes ({hap.shape[0]}); cannot pair into diploids")
        return (hap[0::2] + hap[1::2]).to(torch.int8).contiguous()
    if isinstance(matrix, GenotypeMatrix):
        matrix.transfer_to_gpu()
        g = matrix.genotypes
        if bool((g < 0).any()):
            raise ValueError("input GenotypeMatrix contains missing values (-1); drop or impute missing sites first")
        return g.to(torch.int8).contiguous()
    raise TypeError(f"expected HaplotypeMatrix or GenotypeMatrix; got {type(matrix).__name__}")


def _condensed(M):
    torch = _lib.require_cuda()
    m = M.shape[0]
    iu = torch.triu_indices(m, m, offset=1, device=M.device)
    return M[iu[0], iu[1]]


def rogers_huff_r(matrix):
    """Condensed (upper triangle, row-major pair order) Rogers-Huff r of the dosages
    (ld_statistics.py:492-521); NaN where a site is constant."""
    return _condensed(ld_matrix(dosages(matrix), estimator="rogers_huff_r")[0])


def rogers_huff_r_squared(matrix):
    """``rogers_huff_r(matrix) ** 2`` (ld_statistics.py:524-531)."""
    return rogers_huff_r(matrix) ** 2


def sigma_d2_geno(matrix, idx_i=None, idx_j=None):
    """Unbiased sigma_D^2 of genotype pairs (ld_statistics_genotype.py:1518-1598): all pairs
    i < j in condensed order, or the given pairs; NaN where pi2 is not positive or fewer
    than 4 individuals."""
    torch = _lib.require_cuda()
    M = ld_matrix(dosages(matrix), estimator="sigma_d2_geno")[0]
    if idx_i is None and idx_j is None:
        return _condensed(M)
    if idx_i is None or idx_j is None:
        raise ValueError("idx_i and idx_j must be provided together")
    ii = torch.as_tensor(np.asarray(idx_i), dtype=torch.int64, device="cuda")
    jj = torch.as_tensor(np.asarray(idx_j), dtype=torch.int64, device="cuda")
    if ii.shape != jj.shape:
        raise ValueError("idx_i and idx_j must have the same shape")
    return M[ii, jj]


def diploid_r2_matrix(geno, missing_data="include"):
    """Dosage r^2 matrix of a genotype array with missing calls allowed
    (ld_statistics.py:973-1021; 'exclude' first drops sites with a missing call)."""
    torch = _lib.require_cuda()
    X = _hap_tensor(geno, torch)
    if missing_data == "exclude":
        X = X[:, (X < 0).sum(0) == 0].contiguous()
    return ld_matrix(X, estimator="diploid_r2")[0]


def zns_diploid(geno, missing_data="include"):
    """ZnS of a genotype array: mean off-diagonal dosage r^2 (ld_statistics.py:720-735)."""
    torch = _lib.require_cuda()
    X = _hap_tensor(geno, torch)
    if missing_data == "exclude":
        X = X[:, (X < 0).sum(0) == 0].contiguous()
    m = X.shape[1]
    if m < 2:
        return 0.0
    _, S = ld_matrix(X, estimator="diploid_r2", matrix=False, reduce=True)
    return S[0].item() / (m * (m - 1) / 2)
