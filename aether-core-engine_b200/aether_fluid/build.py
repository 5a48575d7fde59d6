"""Builds libaether_fluid.so (sm_100a) in-tree with nvcc.

Every translation unit is compiled for `sm_100a` only; the FP64 units get
`-fmad=false` so that their f64 arithmetic rounds exactly like the reference's
un-fused Rust expressions.  The shared library links the CUDA runtime
statically, so loading it needs only the driver.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(ROOT, "libaether_fluid.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-extended-lambda"]
# Units whose f64 arithmetic must not be contracted into FMAs.
NO_FMA = {"afl_kernels_f64.cu", "afl_poisson_f64.cu", "afl_poisson_resident.cu",
          "afl_poisson_stream.cu", "afl_ensemble_f64.cu", "afl_ensemble_persist.cu",
          "afl_adjoint_kernels.cu", "afl_medium.cu"}
SOURCES = [
    "afl_kernels_f64.cu",
    "afl_kernels_f32.cu",
    "afl_poisson_f64.cu",
    "afl_poisson_mixed.cu",
    "afl_poisson_resident.cu",
    "afl_poisson_stream.cu",
    "afl_solver.cu",
    "afl_noalloc.cu",
    "afl_ensemble_f64.cu",
    "afl_ensemble_f32.cu",
    "afl_ensemble_persist.cu",
    "afl_ensemble.cu",
    "afl_adjoint_kernels.cu",
    "afl_adjoint.cu",
    "afl_medium.cu",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")
    return path


def _deps() -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(os.path.dirname(ROOT), "include", "aether_fluid.h")
    ]


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps())


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    if not _stale(obj, src):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, "-c", os.path.join(CSRC, src), "-o", obj]
    if src in NO_FMA:
        cmd.insert(-4, "-fmad=false")
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            if f.endswith(".o"):
                os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if force or not os.path.exists(LIB) or any(
        os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs
    ):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
