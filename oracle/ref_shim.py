"""Run the reference's LD modules on the CPU through a NumPy-backed ``cupy`` stand-in.

Test infrastructure only (golden-vector generation in this container; never shipped,
never on a product path).  The reference (pg_gpu) is pure Python + CuPy; CuPy is not
installed here.  Its LD modules only use CuPy's NumPy-compatible array API plus
``cp.RawKernel`` and ``cp.cuda.Device().mem_info``, so a module that re-exports NumPy and
routes ``RawKernel`` launches to the host-compiled kernels of ``oracle/_ref`` (built by
``oracle/build_ref.py``) lets the reference's own code run unmodified.

The LD modules are imported as members of a bare ``pg_gpu`` package object so that
``pg_gpu/__init__.py`` (which needs scikit-allel, tskit and zarr) is not executed.
"""
from __future__ import annotations

import ctypes
import hashlib
import importlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")


class RecordedKernel:
    """RawKernel stand-in that only remembers its source (used while building)."""

    def __init__(self, code, name, options=(), **_):
        self.code = code
        self.name = name

    def __call__(self, *a, **k):
        raise RuntimeError("recording shim cannot launch kernels")


class _HostLib:
    lib = None
    table = None

    @classmethod
    def load(cls):
        if cls.lib is None:
            so = os.path.join(REF_OUT, "libpgref.so")
            if not os.path.exists(so):
                raise FileNotFoundError(
                    f"{so} missing: run `python oracle/build_ref.py` first")
            cls.lib = ctypes.CDLL(so)
            with open(os.path.join(REF_OUT, "kernels.json")) as f:
                cls.table = json.load(f)
        return cls.lib, cls.table


class HostKernel:
    """RawKernel stand-in that runs the reference kernel body serially on the host."""

    def __init__(self, code, name, options=(), **_):
        lib, table = _HostLib.load()
        key = hashlib.sha1(code.encode()).hexdigest()[:16]
        if key not in table:
            raise KeyError("reference kernel changed since oracle/_ref was built")
        ent = table[key]
        self.fn = getattr(lib, ent["symbol"])
        self.fn.restype = None
        self.params = ent["params"]
        self.code = code

    def __call__(self, grid, block, args, **_):
        n_threads = int(np.prod(grid)) * int(np.prod(block))
        if len(args) != len(self.params):
            raise TypeError("argument count mismatch")
        cargs = []
        keep = []
        for a, t in zip(args, self.params):
            if t == "ptr":
                if not isinstance(a, np.ndarray) or not a.flags.c_contiguous:
                    raise TypeError("kernel pointer argument must be a C-contiguous array")
                keep.append(a)
                cargs.append(ctypes.c_void_p(a.ctypes.data))
            elif t == "i64":
                cargs.append(ctypes.c_longlong(int(a)))
            else:
                cargs.append(ctypes.c_int(int(a)))
        cargs.append(ctypes.c_longlong(n_threads))
        self.fn(*cargs)


def make_cupy_shim(record_only: bool) -> types.ModuleType:
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.ndarray = np.ndarray
    cp.asnumpy = np.asarray
    cp.RawKernel = RecordedKernel if record_only else HostKernel

    class _Device:
        mem_info = (8 << 30, 16 << 30)

    cuda = types.ModuleType("cupy.cuda")
    cuda.Device = lambda *a, **k: _Device()
    cp.cuda = cuda
    return cp


def import_reference_modules(reference: str, names, record_only: bool = False):
    """Import ``pg_gpu.<name>`` for each name from the reference checkout."""
    for key in [k for k in sys.modules if k == "pg_gpu" or k.startswith("pg_gpu.")]:
        del sys.modules[key]
    sys.modules["cupy"] = make_cupy_shim(record_only)
    pkg = types.ModuleType("pg_gpu")
    pkg.__path__ = [os.path.join(reference, "pg_gpu")]
    sys.modules["pg_gpu"] = pkg
    out = {}
    for n in names:
        out[n] = importlib.import_module(f"pg_gpu.{n}")
    return out
