"""Build the CPU oracle -- TEST INFRASTRUCTURE ONLY.

  oracle/_build/liboracle.so   plain-C restatement (always)
  oracle/_ref/libclemu_*.so    the reference's own .cl kernels under the CPU
                               work-group emulator (only where the reference
                               sources are present; see clemu/build_clemu.py)
  oracle/_ref/refhost*         the reference's own host (Simulation, layout
                               builders) on the szsnn C ABI through
                               szsnn_b200/compat (see refhost/build_refhost.py)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle(force: bool = False) -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "liboracle.so")
    srcs = [os.path.join(HERE, f) for f in ("oracle.c", "oracle_step.inc", "oracle.h", "philox.h")]
    if force or not os.path.exists(lib) or any(os.path.getmtime(s) > os.path.getmtime(lib) for s in srcs):
        cmd = ["gcc", "-O2", "-std=gnu11", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-msse2",
               "-shared", "-fPIC", "-o", lib, os.path.join(HERE, "oracle.c"), "-lm"]
        subprocess.run(cmd, check=True)
    return lib


def build_all(ref_root: str | None = None, force: bool = False) -> None:
    """The C restatement always; the reference's kernels under the emulator
    when a reference checkout is given (argument or SZSNN_REFERENCE)."""
    build_oracle(force)
    from .clemu.build_clemu import build_clemu, cl_dir, reference_root
    ref_root = ref_root or reference_root()
    if ref_root and os.path.isdir(cl_dir(ref_root)):
        build_clemu(ref_root, force)
        from .refhost.build_refhost import build_refhost
        build_refhost(ref_root, force)


if __name__ == "__main__":
    # usage: python -m oracle.build [<reference root>] [--force]
    args = [a for a in sys.argv[1:] if a != "--force"]
    build_all(args[0] if args else None, force="--force" in sys.argv)
