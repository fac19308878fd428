"""Build recipe of the native library libfornax_b200.so (in-tree, sm_100a).

    python -m fornaxamr_b200.build

compiles fornaxamr_b200/csrc/*.cu and *.cpp with nvcc for sm_100a only and
links them into fornaxamr_b200/libfornax_b200.so (2 ghost layers, 20^3 block
arrays) and, with FX_NG=4, fornaxamr_b200/libfornax_b200_ng4.so (4 layers,
24^3, the layout WENO-Z7 needs).  --fmad=false keeps every
double multiply and add separately rounded, the arithmetic contract under
which the kernels reproduce the reference CPU path bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

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


# the 2-ghost-layer build (20^3 block arrays, the reference's default
# PRJ_NGHOST) and the 4-layer build that WENO-Z7 needs (24^3)
LIBS = {2: LIB, 4: os.path.join(HERE, "libfornax_b200_ng4.so")}


def _build_one(ng: int, verbose: bool, ptxas_info: bool) -> str:
    out_dir = BUILD if ng == 2 else os.path.join(BUILD, f"ng{ng}")
    os.makedirs(out_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "fornax_b200.h"))
    jobs, objs = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(out_dir, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers + [__file__]):
            continue
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + [f"-DFX_NG={ng}", "-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        jobs.append(cmd)
    # FX_BUILD_JOBS bounds the parallel compiles (each nvcc of the kernel
    # sources takes a few GB of host memory)
    workers = int(os.environ.get("FX_BUILD_JOBS", "0")) or (os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), workers))) as pool:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        for r in pool.map(lambda c: subprocess.run(c, check=True), jobs):
            pass
    lib = LIBS[ng]
    if _stale(lib, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Builds both libraries; returns the 2-layer one's path."""
    for ng in (2, 4):
        _build_one(ng, verbose, ptxas_info)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
