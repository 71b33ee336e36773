"""Build recipe for ``oracle/_ref``: the reference's own LD kernels, compiled for the host.

Test infrastructure only.  pg_gpu ships its LD kernels as CUDA C strings inside
Python modules (``pg_gpu/haplotype_kernels.py``, ``pg_gpu/genotype_kernels.py``,
``pg_gpu/ld_pipeline.py:183-217``).  Their bodies are plain scalar C, so this recipe
reads those strings from the reference checkout where they lie, wraps each one in a
serial host loop ("thread" t = 0..n-1), and compiles the lot with g++ into
``oracle/_ref/libpgref.so``.  ``oracle/ref_shim.py`` then routes the reference's
``cp.RawKernel`` launches to these host functions, so the reference's own Python
dispatch (``compute_multi_pop_statistics_batch_hap/_geno``, ``r_squared`` ...) runs on
the CPU and produces golden vectors.  Nothing from the reference is copied into the
repository: the generated C++ and the library live only under ``oracle/_ref/``
(git-ignored).

Usage: ``python oracle/build_ref.py [--reference /path/to/pg_gpu-checkout]``.  Without
``--reference`` the checkout is taken from the environment variable ``PG_GPU_REFERENCE``,
else from this machine's read-only checkout below.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
DEFAULT_REFERENCE = os.environ.get("PG_GPU_REFERENCE", "/root/reference")

# modules whose RawKernel strings are on the LD path
KERNEL_MODULES = ("ld_pipeline", "haplotype_kernels", "genotype_kernels")

_PRELUDE = r"""
#include <cmath>
#include <cstdint>
using std::sqrt;
struct ref_dim3 { unsigned int x, y, z; };
static thread_local ref_dim3 threadIdx = {0, 0, 0};
static thread_local ref_dim3 blockIdx = {0, 0, 0};
static thread_local ref_dim3 blockDim = {256, 1, 1};
#define __global__
#define __restrict__ __restrict
static inline void ref_set_thread(long long t) {
    blockIdx.x = (unsigned int)(t / 256); threadIdx.x = (unsigned int)(t % 256);
}
"""


def code_key(code: str) -> str:
    return hashlib.sha1(code.encode()).hexdigest()[:16]


def _parse_params(code: str):
    m = re.search(r"void\s+k\s*\((.*?)\)\s*\{", code, re.S)
    if not m:
        raise ValueError("kernel signature not found")
    params = []
    for raw in m.group(1).split(","):
        p = " ".join(raw.replace("\n", " ").split())
        name = re.findall(r"[A-Za-z_][A-Za-z0-9_]*", p)[-1]
        ptr = "*" in p
        if ptr:
            ctype = "ptr"
        elif "long long" in p:
            ctype = "i64"
        elif "int" in p:
            ctype = "i32"
        else:
            raise ValueError(f"unsupported parameter {p!r}")
        params.append({"decl": p, "name": name, "ctype": ctype})
    return params


def collect_kernels(reference: str):
    """Import the reference LD modules under the recording shim; return kernels."""
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle import ref_shim  # noqa: E402

    mods = ref_shim.import_reference_modules(reference, KERNEL_MODULES, record_only=True)
    kernels = []
    for modname, mod in mods.items():
        for attr, val in sorted(vars(mod).items()):
            if isinstance(val, ref_shim.RecordedKernel):
                kernels.append({"module": modname, "attr": attr, "code": val.code,
                                "key": code_key(val.code)})
    return kernels


def available(reference: str | None = None) -> bool:
    """Whether the pg_gpu checkout this recipe reads is present."""
    return os.path.isdir(os.path.join(reference or DEFAULT_REFERENCE, "pg_gpu"))


def build(reference: str | None = None, verbose: bool = False) -> str:
    reference = reference or DEFAULT_REFERENCE
    if not os.path.isdir(os.path.join(reference, "pg_gpu")):
        raise FileNotFoundError(f"reference checkout not found at {reference}")
    os.makedirs(REF_OUT, exist_ok=True)
    kernels = collect_kernels(reference)
    parts = [_PRELUDE]
    table = {}
    for kern in kernels:
        sym = f"{kern['module']}__{kern['attr'].strip('_')}"
        params = _parse_params(kern["code"])
        body = kern["code"].replace('extern "C"', "")
        body = re.sub(r"void\s+k\s*\(", f"static void kbody_{sym}(", body, count=1)
        decls = ", ".join(p["decl"] for p in params)
        names = ", ".join(p["name"] for p in params)
        parts.append(body)
        parts.append(
            f'extern "C" void run_{sym}({decls}, long long n_threads) {{\n'
            f"    for (long long t = 0; t < n_threads; ++t) {{ ref_set_thread(t); kbody_{sym}({names}); }}\n"
            "}\n")
        table[kern["key"]] = {"symbol": f"run_{sym}", "module": kern["module"],
                              "attr": kern["attr"], "params": [p["ctype"] for p in params]}
    src = os.path.join(REF_OUT, "pgref_kernels.cpp")
    with open(src, "w") as f:
        f.write("\n".join(parts))
    lib = os.path.join(REF_OUT, "libpgref.so")
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off",
           "-o", lib, src]
    subprocess.run(cmd, check=True)
    with open(os.path.join(REF_OUT, "kernels.json"), "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    if verbose:
        print(f"built {lib} with {len(table)} reference kernels")
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    args = ap.parse_args()
    build(args.reference, verbose=True)


if __name__ == "__main__":
    main()
