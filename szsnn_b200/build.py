"""Build libszsnn_cuda.so (the C-ABI library) in-tree with nvcc for sm_100a.

Usage: python -m szsnn_b200.build   (or szsnn_b200.build.build())

Every translation unit is compiled with -fmad=false -ftz=true -prec-div=true so
that the fp32 neuron rules are bit-identical to an IEEE CPU evaluation of the
same expressions with flush-to-zero (the reference builds its kernels with
-cl-denorms-are-zero, szsnn1.1/src/Simulation.ipp:14).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libszsnn_cuda.so")
REF_HOST = os.path.join(HERE, "szsnn_ref_host")  # C++ host on the drop-in kernel seam (csrc/ref_host.cpp)

SOURCES = [
    "context.cu",
    "ref_kernels.cu",
    "net.cu",
    "bptt.cu",
    "probe.cu",
    "layout.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-ftz=true", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libszsnn_cuda.so")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "szsnn_cuda.h"))
    objs = []
    missing = [s for s in SOURCES if not os.path.exists(os.path.join(CSRC, s))]
    if missing:
        raise FileNotFoundError(f"listed sources missing from {CSRC}: {', '.join(missing)}")
    srcs = list(SOURCES)
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc, *ARCH, *NVFLAGS, "-c", src, "-o", obj, "-I", os.path.join(ROOT, "include")]
            if ptxas_verbose and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    host_src = os.path.join(CSRC, "ref_host.cpp")
    if force or _stale(REF_HOST, [host_src, LIB, os.path.join(ROOT, "include", "szsnn_cuda.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), host_src,
               "-L", HERE, "-lszsnn_cuda", "-Wl,-rpath,$ORIGIN", "-o", REF_HOST]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
