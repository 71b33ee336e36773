"""ctypes binding of ``libldk.so`` (the C ABI in ``include/ldk.h``).

There is no CPU fallback: every compute call goes through the CUDA library, and a
missing library or a missing GPU raises immediately.  Device buffers are torch CUDA
tensors; torch is used for allocation, streams and host/device copies only.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libldk.so")

LDK_OK = 0
LDK_ERR_ARG = -1
LDK_ERR_CUDA = -2
LDK_ERR_ARCH = -3
LDK_ERR_WORKSPACE = -4
LDK_ERR_DEVICE = -5
LDK_ERR_UNSUPPORTED = -6
MAX_POPS = 4
NOALLOC_SCRATCH_BYTES = 64 << 20
MAX_BINS = 64
METHOD_PLAIN = 0
METHOD_TC = 1
X_INT8 = 0
X_PACKED2 = 1

c_i8p = ctypes.c_void_p
c_vp = ctypes.c_void_p


class LdkError(RuntimeError):
    """A libldk entry point returned a negative status."""

    def __init__(self, code, msg):
        super().__init__(f"libldk error {code}: {msg}")
        self.code = code


class ParseDesc(ctypes.Structure):
    """Mirror of ``ldk_parse_t``."""
    _fields_ = [
        ("X", c_vp), ("ld_x", ctypes.c_int64), ("n_rows", ctypes.c_int64), ("n_var", ctypes.c_int64),
        ("genotypes", ctypes.c_int32), ("n_pops", ctypes.c_int32), ("pop_rows", c_vp),
        ("pop_offsets", ctypes.c_int32 * (MAX_POPS + 1)), ("pos", c_vp), ("coord", c_vp),
        ("max_dist", ctypes.c_double), ("n_bins", ctypes.c_int32),
        ("edges", ctypes.c_double * (MAX_BINS + 1)), ("window_offsets", c_vp), ("n_windows", ctypes.c_int32),
        ("snp_block", c_vp), ("n_blocks", ctypes.c_int32), ("method", ctypes.c_int32),
        ("anchor_end", c_vp), ("x_format", ctypes.c_int32),
    ]


class ParseOut(ctypes.Structure):
    """Mirror of ``ldk_parse_out_t``."""
    _fields_ = [("sums", c_vp), ("r2_sums", c_vp), ("pairs", c_vp), ("r2_counts", c_vp)]


EXPORTS = {
    "ldk_version": (ctypes.c_int, []),
    "ldk_last_error": (ctypes.c_char_p, []),
    "ldk_n_stats": (ctypes.c_int, [ctypes.c_int]),
    "ldk_counts_hap": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, ctypes.c_int32, c_vp, c_vp,
                                      ctypes.c_int64, c_vp, c_vp, c_vp]),
    "ldk_counts_geno": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, ctypes.c_int32, c_vp, c_vp,
                                       ctypes.c_int64, c_vp, c_vp, c_vp]),
    "ldk_stats": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp]),
    "ldk_raw_hap": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.c_int, c_vp, c_vp,
                                   ctypes.c_int64, c_vp, c_vp]),
    "ldk_r_family": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp]),
    "ldk_parse_workspace_size": (ctypes.c_size_t, [ctypes.POINTER(ParseDesc)]),
    "ldk_parse": (ctypes.c_int, [ctypes.POINTER(ParseDesc), ctypes.POINTER(ParseOut), c_vp, ctypes.c_size_t,
                                 c_vp]),
    "ldk_parse_noalloc": (ctypes.c_int, [ctypes.POINTER(ParseDesc), ctypes.POINTER(ParseOut), c_vp]),
    "ldk_parse_setup": (ctypes.c_int, [ctypes.POINTER(ParseDesc), c_vp, ctypes.c_size_t, c_vp]),
    "ldk_parse_enqueue": (ctypes.c_int, [ctypes.POINTER(ParseDesc), ctypes.POINTER(ParseOut), c_vp,
                                         ctypes.c_size_t, c_vp]),
    "ldk_parse_status": (ctypes.c_int, [c_vp, c_vp]),
    "ldk_autotune": (ctypes.c_int, [ctypes.c_int]),
    "ldk_ld_matrix_workspace_size": (ctypes.c_size_t, [ctypes.c_int64, ctypes.c_int32]),
    "ldk_ld_matrix": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, ctypes.c_int32, ctypes.c_int, c_vp,
                                     ctypes.c_int64, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "ldk_tile_width": (ctypes.c_int, [ctypes.POINTER(ParseDesc)]),
    "ldk_autotune_load": (ctypes.c_int, [ctypes.c_char_p]),
    "ldk_autotune_save": (ctypes.c_int, [ctypes.c_char_p]),
    "ldk_autotune_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "ldk_autotune_clear": (ctypes.c_int, []),
    "ldk_parse_reproducible": (ctypes.c_int, [ctypes.POINTER(ParseDesc)]),
    "ldk_tc_row_blocks": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    "ldk_profile": (ctypes.c_int, [ctypes.c_int]),
    "ldk_profile_last_kernel_ms": (ctypes.c_double, []),
    "ldk_block_combine": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, ctypes.c_int64, c_vp,
                                         c_vp]),
    "ldk_probe_peaks": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), c_vp]),
}

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libldk and declare its signatures (no GPU needed to load)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m pg_gpu_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != LDK_OK:
        msg = load().ldk_last_error()
        raise LdkError(rc, msg.decode() if msg else "")


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pg_gpu_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")
    return torch


def stream_handle(stream=None):
    torch = require_cuda()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def probe_peaks(stream=None):
    """Measured INT8 tensor-core ops/s (MAC = 2) and FP64 FMA/s of the current device
    (``ldk_probe_peaks``)."""
    require_cuda()
    i8, f64 = ctypes.c_double(), ctypes.c_double()
    check(load().ldk_probe_peaks(ctypes.byref(i8), ctypes.byref(f64), stream_handle(stream)))
    return i8.value, f64.value


def autotune(enable=True):
    """Turn tile autotuning of the tensor-core parse on or off (``ldk_autotune``)."""
    check(load().ldk_autotune(int(bool(enable))))


def autotune_load(path):
    """Merge a saved tuning table (JSON) into the process table; returns its entries."""
    n = load().ldk_autotune_load(os.fsencode(path))
    if n < 0:
        check(n)
    return n


def autotune_save(path):
    """Write the process tuning table as JSON; returns the entries written."""
    n = load().ldk_autotune_save(os.fsencode(path))
    if n < 0:
        check(n)
    return n


def autotune_count():
    """(entries in the tuning table, tunings this process ran)."""
    t = ctypes.c_int()
    n = load().ldk_autotune_count(ctypes.byref(t))
    return n, t.value


def autotune_clear():
    check(load().ldk_autotune_clear())


def tc_row_blocks(genotypes: bool):
    """(SNPs per tensor-core row block, bootstrap blocks one row block may cover) of the
    haplotype or genotype path (``ldk_tc_row_blocks``; no GPU needed)."""
    rows, blocks = ctypes.c_int32(), ctypes.c_int32()
    check(load().ldk_tc_row_blocks(int(bool(genotypes)), ctypes.byref(rows), ctypes.byref(blocks)))
    return rows.value, blocks.value
