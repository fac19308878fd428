"""Build recipe of the native library libfornax_b200.so (in-tree, sm_100a).

    python -m fornaxamr_b200.build

compiles fornaxamr_b200/csrc/*.cu and *.cpp with nvcc for sm_100a only and
links them into fornaxamr_b200/libfornax_b200.so.  --fmad=false keeps every
double multiply and add separately rounded, the arithmetic contract under
which the kernels reproduce the reference CPU path bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfornax_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]
SOURCES = ["fx_kernels.cu", "fx_runtime.cu", "fx_plan.cpp", "fx_noalloc.cu", "fx_adjoint.cu", "fx_amr.cu",
           "fx_amr_host.cpp", "fx_transport.cpp"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "fornax_b200.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers + [__file__]):
            continue
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
