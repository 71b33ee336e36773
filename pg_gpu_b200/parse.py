"""The binned two-locus LD parse on the GPU (``ldk_parse``).

``ld_parse`` takes a haplotype (or genotype) matrix in pg_gpu's layout, population row
lists, positions and bin edges, and returns per-bin (optionally per-bootstrap-block)
float64 sums of the moments-ordered statistics, pair counts, and the sum and count of
finite r^2.  Two counting/estimator methods:

* ``"plain"`` -- per-pair byte counting + FP64 estimators (the reference's design);
* ``"tc"``    -- INT8 tcgen05 Gram-product counts + FP64 estimators and bin sums;
* ``"auto"``  -- ``"tc"``, or ``"plain"`` for the shapes the tensor-core kernel cannot stage
  (its per-bin sums must fit in shared memory beside the pipeline -- four genotype
  populations with more than 36 bins do not -- and each 64-SNP (genotypes: 128-SNP) row
  block may span at most two (four) bootstrap blocks).  Both are GPU kernels.

``Pipeline`` runs a stream of same-shape parses from pinned host memory with the copies
overlapped with the parses.  ``pack_codes`` stores a matrix in two bits per entry
(``ldk_parse_t.x_format = LDK_X_PACKED2``), a quarter of the bytes to copy to the GPU;
``Parser(..., packed=True)`` parses it (tensor-core method).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

METHODS = {"plain": _lib.METHOD_PLAIN, "tc": _lib.METHOD_TC, "auto": _lib.METHOD_TC}


def n_stats(P: int) -> int:
    return {1: 3, 2: 15, 3: 45, 4: 105}[P]


@dataclass
class ParseResult:
    sums: "object"        # (n_blocks, n_bins, n_stats) float64, device
    r2_sums: "object"     # (n_blocks, n_bins) float64
    pairs: "object"       # (n_blocks, n_bins) int64 (uint64 bit pattern)
    r2_counts: "object"   # (n_blocks, n_bins) int64

    def numpy(self):
        return {k: getattr(self, k).cpu().numpy() for k in ("sums", "r2_sums", "pairs", "r2_counts")}


def tc_blocks_fit(snp_block, window_offsets, n_var, genotypes=False) -> bool:
    """Whether every tensor-core row block (``_lib.tc_row_blocks``: SNPs counted from each
    window start) covers at most the bootstrap blocks the kernel stages per row block,
    counted from its first SNP's block -- the kernel's condition (LDK_DEVERR_BLOCK_SPAN
    otherwise)."""
    rows, slots = _lib.tc_row_blocks(genotypes)
    b = snp_block.cpu().numpy() if hasattr(snp_block, "cpu") else np.asarray(snp_block)
    b = b.astype(np.int64).ravel()
    wo = [0, n_var] if window_offsets is None else [int(x) for x in window_offsets]
    for a, e in zip(wo[:-1], wo[1:]):
        seg = b[a:e]
        if seg.size == 0:
            continue
        starts = np.arange(0, seg.size, rows)
        first = seg[starts]
        if np.any(np.maximum.reduceat(seg, starts) - first >= slots) or np.any(np.minimum.reduceat(seg, starts) < first):
            return False
    return True


def pack_codes(data):
    """(n_rows, n_var) int8 codes in {-1, 0, 1, 2} -> (n_rows, ceil(n_var / 4)) uint8: each
    entry as code + 1 in two bits, SNP v in bits 2 (v % 4) of byte v / 4 (LDK_X_PACKED2)."""
    x = np.asarray(data)
    if x.ndim != 2:
        raise ValueError("data must be (n_rows, n_var)")
    if x.size and (x.min() < -1 or x.max() > 2):
        raise ValueError("codes must lie in {-1, 0, 1, 2}")
    n_rows, n_var = x.shape
    c = np.zeros((n_rows, (n_var + 3) // 4 * 4), np.uint8)
    c[:, :n_var] = (x.astype(np.int16) + 1).astype(np.uint8)
    c = c.reshape(n_rows, -1, 4)
    return np.ascontiguousarray(c[..., 0] | (c[..., 1] << 2) | (c[..., 2] << 4) | (c[..., 3] << 6))


def unpack_codes(packed, n_var):
    """Inverse of ``pack_codes``."""
    p = np.asarray(packed, dtype=np.uint8)
    c = np.stack([(p >> s) & 3 for s in (0, 2, 4, 6)], axis=-1).reshape(p.shape[0], -1)
    return (c[:, :n_var].astype(np.int16) - 1).astype(np.int8)


def _dev(x, dtype, torch, device):
    if isinstance(x, torch.Tensor):
        t = x.to(device=device, dtype=dtype)
    else:
        t = torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)
    return t.contiguous()


class Parser:
    """Reusable parse of one input shape: holds the descriptor, workspace and outputs so
    that repeated calls allocate nothing (the CUDA library itself never allocates)."""

    def __init__(self, data, positions, pop_rows, edges, *, genotypes=False, method="auto", max_dist=None,
                 coords=None, window_offsets=None, snp_block=None, n_blocks=1, anchor_end=None, packed=False,
                 device=None):
        torch = _lib.require_cuda()
        lib = _lib.load()
        device = torch.device(device or "cuda")
        self.torch = torch
        self.lib = lib
        if packed:  # pack_codes output: the SNP count comes from the positions
            self.X = _dev(data.view(torch.int8) if isinstance(data, torch.Tensor) else np.asarray(data).view(np.int8),
                          torch.int8, torch, device)
            if self.X.dim() != 2:
                raise ValueError("packed data must be (n_rows, ceil(n_var / 4))")
            n_rows, n_var = self.X.shape[0], len(positions)
            if self.X.shape[1] < (n_var + 3) // 4:
                raise ValueError("packed data holds fewer SNPs than the positions")
        else:
            self.X = _dev(data, torch.int8, torch, device)
            if self.X.dim() != 2:
                raise ValueError("data must be (n_rows, n_var)")
            n_rows, n_var = self.X.shape
        P = len(pop_rows)
        if not 1 <= P <= _lib.MAX_POPS:
            raise ValueError("1-4 populations supported")
        rows = [np.asarray(r, dtype=np.int64).ravel() for r in pop_rows]
        for r in rows:
            if r.size and (r.min() < 0 or r.max() >= n_rows):
                raise IndexError("population row index out of range")
        self.rows = _dev(np.concatenate(rows).astype(np.int32), torch.int32, torch, device)
        self.pos = _dev(np.asarray(positions, dtype=np.float64) if not isinstance(positions, torch.Tensor)
                        else positions, torch.float64, torch, device)
        if self.pos.numel() != n_var:
            raise ValueError("positions must have n_var entries")
        self.coord = None if coords is None else _dev(coords, torch.float64, torch, device)
        edges = np.asarray(edges, dtype=np.float64)
        nb = len(edges) - 1
        if not 1 <= nb <= _lib.MAX_BINS:
            raise ValueError("1-64 bins supported")
        self.n_bins = nb
        self.P = P
        self.n_blocks = int(n_blocks)
        self.block = None if snp_block is None else _dev(np.asarray(snp_block, np.int32)
                                                         if not isinstance(snp_block, torch.Tensor) else snp_block,
                                                         torch.int32, torch, device)
        d = _lib.ParseDesc()
        d.X = _lib.ptr(self.X)
        d.ld_x = self.X.shape[1]
        d.x_format = _lib.X_PACKED2 if packed else _lib.X_INT8
        d.n_rows = n_rows
        d.n_var = n_var
        d.genotypes = int(bool(genotypes))
        d.n_pops = P
        d.pop_rows = _lib.ptr(self.rows)
        off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
        for k in range(_lib.MAX_POPS + 1):
            d.pop_offsets[k] = int(off[min(k, P)])
        d.pos = _lib.ptr(self.pos)
        d.coord = _lib.ptr(self.coord)
        d.max_dist = float(edges[-1] if max_dist is None else max_dist)
        d.n_bins = nb
        for k in range(nb + 1):
            d.edges[k] = float(edges[k])
        if window_offsets is not None:
            wo = np.asarray(window_offsets, dtype=np.int64)
            self._win = (ctypes.c_int64 * len(wo))(*wo.tolist())
            d.window_offsets = ctypes.cast(self._win, ctypes.c_void_p)
            d.n_windows = len(wo) - 1
        else:
            d.window_offsets = None
            d.n_windows = 1
        if anchor_end is not None:
            ae = np.asarray(anchor_end, dtype=np.int64).ravel()
            if ae.size != d.n_windows:
                raise ValueError("anchor_end needs one entry per window")
            self._anc = (ctypes.c_int64 * len(ae))(*ae.tolist())
            d.anchor_end = ctypes.cast(self._anc, ctypes.c_void_p)
        else:
            d.anchor_end = None
        d.snp_block = _lib.ptr(self.block)
        d.n_blocks = self.n_blocks
        if method not in METHODS:
            raise ValueError(f"method must be one of {sorted(METHODS)}")
        d.method = METHODS[method]
        self.auto = method == "auto"
        if self.auto and snp_block is not None and not tc_blocks_fit(snp_block, window_offsets, n_var, genotypes):
            d.method = _lib.METHOD_PLAIN  # bootstrap blocks too small for the tensor-core staging
        self.desc = d
        ws = lib.ldk_parse_workspace_size(ctypes.byref(d))
        if ws == 0:
            # validation failed: run ldk_parse to surface the message
            _lib.check(lib.ldk_parse(ctypes.byref(d), None, None, 0, None))
        self.workspace = torch.empty(int(ws), dtype=torch.uint8, device=device)
        NS = n_stats(P)
        self.out = ParseResult(
            sums=torch.zeros((self.n_blocks, nb, NS), dtype=torch.float64, device=device),
            r2_sums=torch.zeros((self.n_blocks, nb), dtype=torch.float64, device=device),
            pairs=torch.zeros((self.n_blocks, nb), dtype=torch.int64, device=device),
            r2_counts=torch.zeros((self.n_blocks, nb), dtype=torch.int64, device=device))
        o = _lib.ParseOut()
        o.sums = _lib.ptr(self.out.sums)
        o.r2_sums = _lib.ptr(self.out.r2_sums)
        o.pairs = _lib.ptr(self.out.pairs)
        o.r2_counts = _lib.ptr(self.out.r2_counts)
        self._o = o

    def _to_plain(self, rc) -> bool:
        """With method "auto": on the tensor-core kernel's "unsupported shape" answer,
        switch this parse to the plain FP64 kernel (new workspace size) and say so."""
        if not (self.auto and rc == _lib.LDK_ERR_UNSUPPORTED and self.desc.method != _lib.METHOD_PLAIN):
            return False
        self.desc.method = _lib.METHOD_PLAIN
        ws = self.lib.ldk_parse_workspace_size(ctypes.byref(self.desc))
        if ws > self.workspace.numel():
            self.workspace = self.torch.empty(int(ws), dtype=self.torch.uint8, device=self.workspace.device)
        return True

    @property
    def method(self) -> str:
        """The kernel this parse runs: "tc" or "plain"."""
        return {_lib.METHOD_PLAIN: "plain", _lib.METHOD_TC: "tc"}[self.desc.method]

    def run(self, stream=None) -> ParseResult:
        while True:
            rc = self.lib.ldk_parse(ctypes.byref(self.desc), ctypes.byref(self._o), _lib.ptr(self.workspace),
                                    self.workspace.numel(), _lib.stream_handle(stream))
            if not self._to_plain(rc):
                break
        _lib.check(rc)
        return self.out

    def reproducible(self) -> bool:
        """Whether repeated runs give identical bits (``ldk_parse_reproducible``)."""
        r = self.lib.ldk_parse_reproducible(ctypes.byref(self.desc))
        if r < 0:
            _lib.check(r)
        return bool(r)

    def tile_width(self):
        """Partner SNPs per tile this parse uses now (tuned or default); 0 for "plain"."""
        w = self.lib.ldk_tile_width(ctypes.byref(self.desc))
        if w < 0:
            _lib.check(w)
        return w

    # -- the split form: plan once, enqueue device work only, read the status later
    def setup(self, stream=None):
        """Write the plan (window offsets, row blocks) into the workspace; synchronises."""
        while True:
            rc = self.lib.ldk_parse_setup(ctypes.byref(self.desc), _lib.ptr(self.workspace),
                                          self.workspace.numel(), _lib.stream_handle(stream))
            if not self._to_plain(rc):
                break
        _lib.check(rc)

    def enqueue(self, stream=None) -> ParseResult:
        """Enqueue one parse (device work only; capturable).  Needs ``setup()`` first."""
        _lib.check(self.lib.ldk_parse_enqueue(ctypes.byref(self.desc), ctypes.byref(self._o),
                                              _lib.ptr(self.workspace), self.workspace.numel(),
                                              _lib.stream_handle(stream)))
        return self.out

    def status(self, stream=None):
        """Synchronise and raise LdkError if the last enqueued parse set a device error."""
        _lib.check(self.lib.ldk_parse_status(_lib.ptr(self.workspace), _lib.stream_handle(stream)))

    def graph(self, after=None):
        """A CUDA graph of one parse (and of ``after(out)``, torch work on the outputs
        whose result is returned beside the graph).  Replaying it re-reads the input
        tensors (``self.X``, ``self.pos``, ...) in place; call ``status()`` after replays."""
        torch = self.torch
        self.setup()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):  # warm-up outside the capture
            out = self.enqueue()
            if after is not None:
                after(out)
        torch.cuda.current_stream().wait_stream(side)
        self.status()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            out = self.enqueue()
            extra = after(out) if after is not None else None
        return g, extra


class Pipeline:
    """A stream of same-shape parses fed from pinned host memory, with the host-to-device
    copy of each batch and the device-to-host copy of each result overlapped with the
    parses of the neighbouring batches.

    ``make_slot()`` builds one slot and returns ``(parser, inputs, after)``: a ``Parser``;
    a dict naming the device tensors a step reads (the parser's ``X``, ``pos``, ``block``
    and any tensor ``after`` reads), which ``submit`` fills from host tensors of the same
    names; and ``after(out)``, torch work on the parse outputs captured into the slot's
    CUDA graph (e.g. bootstrap replicates via ``block_combine``), returning a tuple of
    device tensors, or None.  Every slot has its own inputs, workspace, outputs and graph,
    so batch k + 1 is copied in while batch k is parsed and batch k - 1 copied out (three
    streams ordered by events).

    Every parse clears its slot's device status word, so after each replay the word is
    OR-ed into a per-batch device word (on the parse stream, before the slot's next
    batch can clear it); ``status()`` checks every batch submitted since the last check.

    ``submit(host_inputs, host_outputs)`` enqueues one batch: ``host_outputs`` receives
    ``(sums, pairs, *after(...))`` of that batch, each a pinned host tensor of the matching
    shape; they are valid after ``drain()``.  The caller must not reuse a batch's host
    tensors before then (or before the batch ``slots`` places later has been submitted
    and drained)."""

    def __init__(self, make_slot, slots: int = 2):
        torch = _lib.require_cuda()
        self.torch = torch
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.slots = []
        for _ in range(slots):
            parser, inputs, after = make_slot()
            graph, extra = parser.graph(after=after)
            extra = () if extra is None else tuple(extra)
            self.slots.append((parser, dict(inputs), graph, (parser.out.sums, parser.out.pairs) + extra))
        self.h2d, self.compute, self.d2h = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        self.ready = [torch.cuda.Event() for _ in range(slots)]
        self.parsed = [torch.cuda.Event() for _ in range(slots)]
        self.free = [torch.cuda.Event() for _ in range(slots)]
        self.k = 0
        self._batch_status = []  # (batch index, slot, device int32 copy of that batch's status word)

    def submit(self, host_inputs: dict, host_outputs) -> None:
        torch = self.torch
        s = self.k % len(self.slots)
        parser, inputs, graph, outs = self.slots[s]
        caller = torch.cuda.current_stream()
        if set(host_inputs) != set(k for k, v in inputs.items() if v is not None):
            raise KeyError(f"host inputs {sorted(host_inputs)} do not match the slot's {sorted(inputs)}")
        if len(host_outputs) != len(outs):
            raise ValueError(f"{len(outs)} host outputs expected")
        for st in (self.h2d, self.compute, self.d2h):
            st.wait_stream(caller)  # work the caller enqueued first (e.g. a start event)
        with torch.cuda.stream(self.h2d):
            self.h2d.wait_event(self.free[s])  # the slot's previous batch is parsed and copied out
            for name, h in host_inputs.items():
                inputs[name].copy_(h, non_blocking=True)
            self.ready[s].record(self.h2d)
        with torch.cuda.stream(self.compute):
            self.compute.wait_event(self.ready[s])
            graph.replay()
            # the status word sits at the start of the workspace; keep this batch's copy
            self._batch_status.append((self.k, s, parser.workspace[:4].view(torch.int32).clone()))
            self.parsed[s].record(self.compute)
        with torch.cuda.stream(self.d2h):
            self.d2h.wait_event(self.parsed[s])
            for h, d in zip(host_outputs, outs):
                h.copy_(d, non_blocking=True)
            self.free[s].record(self.d2h)
        self.k += 1

    def drain(self) -> None:
        """Make the caller's stream wait for every submitted batch; the host outputs are
        valid once that stream is synchronised (``status()`` checks the device status)."""
        caller = self.torch.cuda.current_stream()
        for st in (self.h2d, self.compute, self.d2h):
            caller.wait_stream(st)

    def status(self) -> None:
        """Synchronise and raise LdkError if any batch submitted since the last call set a
        device error (the library decodes the word; the message names the batch)."""
        self.torch.cuda.synchronize()
        pending, self._batch_status = self._batch_status, []
        for k, s, word in pending:
            if int(word.item()) != 0:
                parser = self.slots[s][0]
                # hand the batch's word back to the library, which turns it into its message
                parser.workspace[:4].view(self.torch.int32).copy_(word)
                try:
                    parser.status()
                except _lib.LdkError as e:
                    raise _lib.LdkError(e.code, f"batch {k}: {e.args[0]}") from None


def ld_parse(data, positions, pop_rows, edges, **kw) -> ParseResult:
    """One-shot parse; see ``Parser`` for the arguments."""
    return Parser(data, positions, pop_rows, edges, **kw).run()


def block_combine(block_sums, weights, stream=None):
    """out[r] = sum_b weights[r, b] * block_sums[b] on the GPU (bootstrap replicates,
    window totals).  ``block_sums`` (n_blocks, ...) float64, ``weights`` (R, n_blocks)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    bs = block_sums.contiguous()
    nb = bs.shape[0]
    k = int(bs.numel() // max(nb, 1))
    w = _dev(weights, torch.int32, torch, bs.device)
    if w.dim() != 2 or w.shape[1] != nb:
        raise ValueError("weights must be (n_rep, n_blocks)")
    out = torch.empty((w.shape[0],) + tuple(bs.shape[1:]), dtype=torch.float64, device=bs.device)
    _lib.check(lib.ldk_block_combine(_lib.ptr(bs), nb, k, _lib.ptr(w), w.shape[0], _lib.ptr(out),
                                     _lib.stream_handle(stream)))
    return out
