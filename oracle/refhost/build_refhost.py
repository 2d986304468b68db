"""Build the reference's own host code against the szsnn compat layer --
TEST INFRASTRUCTURE ONLY.

  python -m oracle.refhost.build_refhost <reference root> [--force]

Compiles, where they lie under <reference root>/szsnn1.1/src, the reference's
host sources that Simulation<float> needs (GroupData, SynapseIndex, the
queues, SpikeBuffer, the timer, exception, data buffers, kernel wrapper,
device manager and utils; the model traits, whose header defines its
statics (so it enters one translation unit only), and the template sources NeuronData,
SynapseData, CurrentData, NetworkGraph and Simulation come in through their
headers) together with:

  * szsnn_b200/compat/: the OpenCL C++ value types over the C ABI (CL/cl.hpp),
    std-backed stand-ins for the Boost parts the host uses, and Context.cpp,
    which replaces the reference's Context.cpp (the one file that talks to
    OpenCL);
  * szsnn_b200/compat/szsnn_locales.h, force-included so the production
    layout constants replace the debugging ones the reference's locales.h
    leaves active;
  * oracle/refhost/refhost_main.cpp, the driver,

linked against szsnn_b200/libszsnn_cuda.so.  Two binaries go to oracle/_ref/
(git-ignored): refhost (partitions of 1024 neurons) and refhost_small (256).
Nothing from the reference is copied into the repository.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
OUT = os.path.join(ORACLE, "_ref")
COMPAT = os.path.join(ROOT, "szsnn_b200", "compat")
LIBDIR = os.path.join(ROOT, "szsnn_b200")

REF_SOURCES = ["GroupData.cpp", "SynapseIndex.cpp", "GlobalQueue.cpp", "LocalQueue.cpp", "SpikeBuffer.cpp",
               "SzsnnTimer.cpp", "SzsnnException.cpp", "DataBuffer.cpp", "MemoryBuffer.cpp", "KernelWrapper.cpp",
               "DeviceManager.cpp", "utils.cpp"]
VARIANTS = {"refhost": 1024, "refhost_small": 256}


def binary(name: str = "refhost") -> str:
    return os.path.join(OUT, name)


def build_refhost(ref_root: str, force: bool = False, verbose: bool = False) -> list[str]:
    src_dir = os.path.join(ref_root, "szsnn1.1", "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference host sources not found under {src_dir}")
    os.makedirs(OUT, exist_ok=True)
    lib = os.path.join(LIBDIR, "libszsnn_cuda.so")
    if not os.path.exists(lib):
        raise FileNotFoundError(f"{lib} is not built (python -m szsnn_b200.build)")
    ours = [os.path.join(COMPAT, "Context.cpp"), os.path.join(HERE, "refhost_main.cpp")]
    srcs = [os.path.join(src_dir, s) for s in REF_SOURCES] + ours
    deps = srcs + [lib] + [os.path.join(dp, f) for dp, _, fs in os.walk(COMPAT) for f in fs]
    outs = []
    for name, mps in VARIANTS.items():
        out = binary(name)
        outs.append(out)
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-w", f"-DSZSNN_MPS={mps}",
               "-include", os.path.join(COMPAT, "szsnn_locales.h"),
               "-I", COMPAT, "-I", os.path.join(ROOT, "include"), "-I", src_dir,
               "-I", os.path.join(src_dir, "models"),
               *srcs, "-L", LIBDIR, "-lszsnn_cuda", f"-Wl,-rpath,{LIBDIR}", "-Wl,-rpath,$ORIGIN/../../szsnn_b200",
               "-o", out]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return outs


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "--force"]
    root = args[0] if args else os.environ.get("SZSNN_REFERENCE")
    if not root:
        sys.exit("usage: build_refhost.py <reference root> [--force]  (or set SZSNN_REFERENCE)")
    for p in build_refhost(root, force="--force" in sys.argv, verbose=True):
        print(p)
