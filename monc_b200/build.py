"""Build libmoncgpu.so in-tree for sm_100a with nvcc.

Each translation unit is compiled separately (so the FP64 dynamical-core kernels can be built
with --fmad=false) and linked into monc_b200/libmoncgpu.so.  Objects go to monc_b200/_build/.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmoncgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

# (source, extra flags)
UNITS = [
    ("grid.cpp", []),
    ("checkpoint.cpp", []),
    ("api.cu", []),
    ("dycore_f64.cu", ["--fmad=false"]),
    ("dycore_f64_fast.cu", []),
    ("dycore_f32.cu", ["--fmad=false"]),
    ("dycore_f32_fast.cu", []),
    ("fft.cu", []),
    ("iter.cu", []),
    ("tlad.cu", []),
    ("adjoint.cu", []),
    ("slab.cu", []),
    ("cfl.cu", []),
    ("forcing.cu", []),
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "monc_gpu.h"))
    objs = []
    for src, extra in UNITS:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers) and not ptxas_v:
            continue
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
        if ptxas_v and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
