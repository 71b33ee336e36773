"""pg_gpu's ``ld_pipeline`` call surface (``pg_gpu/ld_pipeline.py``) on libldk.

Pair generation, per-pair two-locus counts, moments statistic names / averaging specs
and the batched statistics, with the reference's signatures and return conventions.
Arrays are torch CUDA tensors (numpy inputs are copied to the device); counting and
estimators run in libldk, pair enumeration uses device tensor ops.
"""
from __future__ import annotations

import numpy as np

from . import _lib

# ---------------------------------------------------------------------------
# memory estimation and pairs  (ld_pipeline.py:16-122)
# ---------------------------------------------------------------------------


def estimate_ld_chunk_size(n_haplotypes_per_pop, available_memory_bytes=None, num_pops=2):
    """Pairs per chunk for the per-pair-list API (same model as ld_pipeline.py:16-49)."""
    if available_memory_bytes is None:
        torch = _lib.require_cuda()
        available_memory_bytes = int(torch.cuda.mem_get_info()[0] * 0.5)
    bytes_per_pair = (4 * n_haplotypes_per_pop * num_pops + 150 * num_pops) * 3
    chunk = available_memory_bytes // bytes_per_pair
    return max(100_000, min(chunk, 10_000_000))


def _device_tensor(x, dtype):
    torch = _lib.require_cuda()
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")


def iter_pairs_within_distance(positions, max_dist, chunk_size):
    """Yield (idx_i, idx_j) int32 CUDA tensors of all pairs i < j with
    pos[j] - pos[i] <= max_dist, in anchor order, in chunks of about ``chunk_size``
    pairs (ld_pipeline.py:57-122: whole anchors per chunk)."""
    torch = _lib.require_cuda()
    pos = _device_tensor(positions, torch.float64)
    n = pos.numel()
    if n < 2:
        return
    jmax = torch.searchsorted(pos, pos + float(max_dist), right=True)
    per = torch.clamp(jmax - torch.arange(n, device=pos.device) - 1, min=0)
    cum = torch.cumsum(per, 0)
    total = int(cum[-1].item())
    if total == 0:
        return
    chunk_size = max(1, int(chunk_size))
    n_chunks = (total + chunk_size - 1) // chunk_size
    targets = torch.clamp(torch.arange(1, n_chunks + 1, device=pos.device) * chunk_size, max=total)
    v_his = (torch.searchsorted(cum, targets, right=False) + 1).clamp(max=n).cpu().tolist()
    v_lo = 0
    for v_hi in v_his:
        if v_hi <= v_lo:
            continue
        counts = per[v_lo:v_hi]
        npairs = int(counts.sum().item())
        if npairs == 0:
            v_lo = v_hi
            continue
        anchors = torch.arange(v_lo, v_hi, device=pos.device)
        idx_i = torch.repeat_interleave(anchors, counts)
        start = torch.cumsum(counts, 0) - counts
        within = torch.arange(npairs, device=pos.device) - torch.repeat_interleave(start, counts)
        yield idx_i.to(torch.int32), (idx_i + 1 + within).to(torch.int32)
        v_lo = v_hi


# ---------------------------------------------------------------------------
# per-pair counts  (ld_pipeline.py:130-263)
# ---------------------------------------------------------------------------


def _rows_and_missing(mat, pop_indices, missing_pred):
    torch = _lib.require_cuda()
    if pop_indices is None:
        rows = torch.arange(mat.shape[0], dtype=torch.int32, device="cuda")
        sub = mat
    else:
        rows = _device_tensor(np.asarray(pop_indices) if not isinstance(pop_indices, torch.Tensor)
                              else pop_indices, torch.int32)
        sub = mat.index_select(0, rows.long())
    return rows, bool(missing_pred(sub).any().item())


def compute_counts_for_pairs(haplotypes, idx_i, idx_j, pop_indices=None):
    """[n11, n10, n01, n00] (N, 4) int32 and n_valid (N,) int32 -- None when the
    population has no missing entry (ld_pipeline.py:130-175)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    X = _device_tensor(haplotypes, torch.int8)
    I = _device_tensor(idx_i, torch.int32)
    J = _device_tensor(idx_j, torch.int32)
    rows, has_missing = _rows_and_missing(X, pop_indices, lambda s: s == -1)
    n = I.numel()
    counts = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    nv = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(lib.ldk_counts_hap(_lib.ptr(X), X.shape[1], X.shape[1], _lib.ptr(rows), rows.numel(), _lib.ptr(I),
                                  _lib.ptr(J), n, _lib.ptr(counts), _lib.ptr(nv), _lib.stream_handle()))
    return counts, (nv if has_missing else None)


def compute_genotype_counts_for_pairs(genotypes, idx_i, idx_j, pop_indices=None):
    """Nine-cell counts (N, 9) int32 in column order g_i*3 + g_j and n_valid (None without
    missing data) (ld_pipeline.py:183-263)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    X = _device_tensor(genotypes, torch.int8)
    I = _device_tensor(idx_i, torch.int32)
    J = _device_tensor(idx_j, torch.int32)
    rows, has_missing = _rows_and_missing(X, pop_indices, lambda s: s < 0)
    n = I.numel()
    counts = torch.empty((n, 9), dtype=torch.int32, device="cuda")
    nv = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(lib.ldk_counts_geno(_lib.ptr(X), X.shape[1], X.shape[1], _lib.ptr(rows), rows.numel(),
                                   _lib.ptr(I), _lib.ptr(J), n, _lib.ptr(counts), _lib.ptr(nv),
                                   _lib.stream_handle()))
    return counts, (nv if has_missing else None)


# ---------------------------------------------------------------------------
# batched statistics  (ld_pipeline.py:271-349, haplotype_kernels.py:584-640,
# genotype_kernels.py:881-936)
# ---------------------------------------------------------------------------


def compute_multi_pop_statistics_batch(counts_per_pop, n_valid_per_pop=None, genotypes=False):
    """(N, n_stats) float64 moments-ordered statistics of P populations."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    P = len(counts_per_pop)
    width = 9 if genotypes else 4
    C = torch.stack([_device_tensor(c, torch.int32).reshape(-1, width) for c in counts_per_pop]).contiguous()
    n = C.shape[1]
    NV = None
    if n_valid_per_pop is not None and any(v is not None for v in n_valid_per_pop):
        NV = torch.stack([_device_tensor(v, torch.int32) if v is not None else C[p].sum(dim=1, dtype=torch.int32)
                          for p, v in enumerate(n_valid_per_pop)]).contiguous()
    out = torch.empty((n, len(ld_names(P))), dtype=torch.float64, device="cuda")
    _lib.check(lib.ldk_stats(int(bool(genotypes)), P, _lib.ptr(C), _lib.ptr(NV), n, _lib.ptr(out),
                             _lib.stream_handle()))
    return out


def compute_two_pop_statistics_batch(counts_pop1, counts_pop2, n_valid1, n_valid2, ld_statistics=None):
    """The 15 two-population statistics (ld_pipeline.py:271-322)."""
    return compute_multi_pop_statistics_batch([counts_pop1, counts_pop2], [n_valid1, n_valid2])


def compute_single_pop_statistics_batch(counts, n_valid, ld_statistics=None):
    """[DD, Dz, pi2] of one population (ld_pipeline.py:330-349)."""
    return compute_multi_pop_statistics_batch([counts], [n_valid])


def compute_multi_pop_statistics_batch_hap(counts_per_pop, n_valid_per_pop, ld_statistics_module=None,
                                           stat_specs=None):
    """Drop-in for haplotype_kernels.compute_multi_pop_statistics_batch_hap (:584-640)."""
    _check_specs(len(counts_per_pop), stat_specs)
    return compute_multi_pop_statistics_batch(counts_per_pop, n_valid_per_pop)


def compute_multi_pop_statistics_batch_geno(counts_per_pop, n_valid_per_pop, _=None, stat_specs=None):
    """Drop-in for genotype_kernels.compute_multi_pop_statistics_batch_geno (:881-936)."""
    _check_specs(len(counts_per_pop), stat_specs)
    return compute_multi_pop_statistics_batch(counts_per_pop, n_valid_per_pop, genotypes=True)


def _check_specs(P, stat_specs):
    if stat_specs is not None and [s[0] for s in stat_specs] != ld_names(P):
        raise ValueError("libldk evaluates moments' statistic set for P populations; custom specs differ")


# ---------------------------------------------------------------------------
# names and averaging specs  (ld_pipeline.py:357-457)
# ---------------------------------------------------------------------------


def ld_names(num_pops):
    """moments.LD.Util.ld_names order."""
    names = []
    for i in range(num_pops):
        for j in range(i, num_pops):
            names.append(f"DD_{i}_{j}")
    for i in range(num_pops):
        for j in range(num_pops):
            for k in range(j, num_pops):
                names.append(f"Dz_{i}_{j}_{k}")
    for i in range(num_pops):
        for j in range(i, num_pops):
            for k in range(i, num_pops):
                for l in range(k, num_pops):
                    if k == i == l and j != i:
                        continue
                    if i == k and l < j:
                        continue
                    names.append(f"pi2_{i}_{j}_{k}_{l}")
    return names


def het_names(num_pops):
    return [f"H_{i}_{j}" for i in range(num_pops) for j in range(i, num_pops)]


def generate_stat_specs(num_pops):
    """(name, [(weight, kind, pops), ...]) -- moments' _call_sgc averaging."""
    from .csrc import gen_estimators as G
    return [(name, [(w, k, tuple(q)) for (w, k, q) in calls]) for name, calls in G.stat_specs(num_pops)]
