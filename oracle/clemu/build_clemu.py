"""Build "Oracle B": the reference's own OpenCL kernels compiled for the CPU.

TEST INFRASTRUCTURE ONLY.  Reads the kernel sources where they lie in the
reference tree (szsnn1.1/src/cl/{gather,scatter,IF_curr_exp_update,
Izhikevich_update,Const_rate_update}_kernel.cl), rewrites only what C++ cannot
parse, and compiles them with the fiber emulator (clemu_rt.cpp) into
oracle/_ref/libclemu_<variant>.so.  Generated sources go to oracle/_ref/gen/
(git-ignored); nothing from the reference is committed.

What the reference's Context does before building a kernel
(szsnn1.1/src/Context.cpp:244-274): prepend locales.h and pass -D flags.  Here
the prepended constants are the variant's values (the production values are
the ones commented in locales.h:19,34,38,46) and the flags are those of
Simulation.ipp:13-38 with FLOAT_TYPE=float (neuron_model_traits.hpp:42-43).
The input kernel is built with -DSZSNN_KERNEL_OUTPUT_SPIKES (the
SZSNN_NO_INPUT_TO_OUTPUT == 0 configuration, Simulation.ipp:31-35), because
with the shipped value 1 input spikes never reach scatter.

Rewrites (text only, kernel arithmetic untouched):
  * `__local T x[..];` statements -> `static thread_local T x[..];` (shared by
    the fibers of one work-group); other `__local`, `__global`, `__kernel`
    qualifiers dropped; `__constant` -> `static const`;
  * `(short2) (a, b)` vector literals -> `make_short2(a, b)`;
  * floating literals get an `f` suffix (-cl-single-precision-constant);
  * the kernel's own `#define NULL 0` is dropped (C++ already defines NULL);
  * scatter only: a barrier at the top of the serial per-spike loop
    (scatter_kernel.cl:121-127).  Work-item 0 overwrites the shared `delayBits`
    for the next spike with no barrier after the other work-items read it for
    the current one; on the reference's target GPUs the MAX_SYNAPTIC_DELAY (64)
    delay lanes run in one lockstep 64-wide wavefront, which orders the read
    before the overwrite.  Fibers are not lockstep, so the barrier restores the
    order that hardware gives.
Compiled with -ffp-contract=off; FTZ/DAZ is switched on per launch
(-cl-denorms-are-zero, Simulation.ipp:14).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")


def reference_root() -> str | None:
    """The reference checkout to read the kernel sources from: the
    SZSNN_REFERENCE environment variable, or None (the prebuilt libraries in
    oracle/_ref/ are then used as they are)."""
    return os.environ.get("SZSNN_REFERENCE") or None


def cl_dir(ref_root: str) -> str:
    return os.path.join(ref_root, "szsnn1.1", "src", "cl")

VARIANTS = {
    # name: (MAX_PARTITION_SIZE, WARP_SIZE, NEURONS_PER_WI, MAX_SYNAPTIC_DELAY)
    "prod": (1024, 32, 4, 64),
    "small": (256, 32, 4, 64),
}

KERNELS = {
    "gather": ("gather_kernel.cl", "gather", False),
    "scatter": ("scatter_kernel.cl", "scatter", False),
    "if_curr_exp": ("IF_curr_exp_update_kernel.cl", "IF_curr_exp_update", True),
    "izhikevich": ("Izhikevich_update_kernel.cl", "Izhikevich_update", True),
    "const_rate": ("Const_rate_update_kernel.cl", "Const_rate_update", True),
}

UPDATE_WRAPPER = """
extern "C" int clemu_{name}(unsigned long cycle, unsigned lpc, const void* ps, const void* params, void* vars,
    unsigned iic, void* ic, void* cur, unsigned iif, void* ifd, void* fc, void* fd, void* fo, unsigned poff,
    unsigned gpc)
{{
    clemu_ftz_scope ftz_;
    return clemu::launch(lpc, THREADS_PER_GROUP, [&] {{
        {kernel}(cycle, lpc, (const unsigned*)ps, (const float*)params, (float*)vars, iic, (float*)ic,
                 (float*)cur, iif, (unsigned*)ifd, (unsigned*)fc, (unsigned*)fd, (unsigned*)fo, poff, gpc);
    }});
}}
"""

GATHER_WRAPPER = """
extern "C" int clemu_gather(unsigned long cycle, unsigned pc, const void* ps, void* cur, unsigned long pitch,
    void* gqc, void* gqb, const void* targets, const void* weights)
{
    clemu_ftz_scope ftz_;
    return clemu::launch(pc, THREADS_PER_GROUP, [&] {
        gather(cycle, pc, (const uint*)ps, (float*)cur, pitch, (uint*)gqc, (uint*)gqb, (const uint*)targets,
               (const float*)weights);
    });
}
"""

SCATTER_WRAPPER = """
extern "C" int clemu_scatter(unsigned long cycle, unsigned pc, void* fc, void* fd, unsigned gpitch,
    unsigned gstep, const void* gptrs, const void* gmat, unsigned long pitch, void* gqc, void* gqb, void* lqc,
    void* lqe, const void* dbits)
{
    clemu_ftz_scope ftz_;
    return clemu::launch(pc, THREADS_PER_GROUP, [&] {
        scatter(cycle, pc, (uint*)fc, (uint*)fd, gpitch, gstep, (const uint2*)gptrs, (const uint2*)gmat, pitch,
                (uint*)gqc, (uint*)gqb, (uint*)lqc, (short2*)lqe, (const ulong*)dbits);
    });
}
"""

_LOCAL_DECL = re.compile(r"^(\s*)__local\s+([^;*=()]*?\w+\s*(?:\[[^\]]*\])?)\s*;", re.M)
_FLOAT_LIT = re.compile(r"(?<![\w.])(\d+\.\d*|\.\d+)([eE][+-]?\d+)?(?![\w.])")
_SHORT2 = re.compile(r"\(short2\)\s*\(([^()]*)\)")


_SCATTER_SPIKE_LOOP = "        uint neuron = l_fired[spike];"


def rewrite(src: str, kernel: str = "") -> str:
    if kernel == "scatter":
        if src.count(_SCATTER_SPIKE_LOOP) != 1:
            raise RuntimeError("scatter kernel: per-spike loop anchor not found")
        src = src.replace(_SCATTER_SPIKE_LOOP, "        barrier(CLK_LOCAL_MEM_FENCE);\n" + _SCATTER_SPIKE_LOOP)
    src = re.sub(r"^\s*#define\s+NULL\s+0\s*$", "", src, flags=re.M)
    src = re.sub(r"^\s*#pragma\s+OPENCL.*$", "", src, flags=re.M)
    src = _LOCAL_DECL.sub(lambda m: f"{m.group(1)}static thread_local {m.group(2)};", src)
    src = src.replace("__local", "").replace("__global", "").replace("__kernel", "")
    src = src.replace("__constant", "static const")
    src = _SHORT2.sub(lambda m: f"make_short2({m.group(1)})", src)
    src = _FLOAT_LIT.sub(lambda m: m.group(0) + "f", src)
    return src


def constants(mps: int, warp: int, npw: int, delay: int) -> str:
    return f"""
#define MAX_CONNECTIONS_PER_NEURON (1<<10)
#define MAX_PARTITION_SIZE {mps}
#define MAX_PARTITION_COUNT (1<<10)
#define MAX_INPUTS_SIZE MAX_PARTITION_SIZE
#define MAX_NETWORK_SIZE MAX_PARTITION_COUNT * MAX_PARTITION_SIZE
#define BIT_VECTOR_WORD_SIZE 32
#define BIT_VECTOR_BYTE_PITCH ((MAX_PARTITION_SIZE)/8)
#define BIT_VECTOR_WORD_PITCH ((MAX_PARTITION_SIZE)/(BIT_VECTOR_WORD_SIZE))
#define WARP_SIZE {warp}
#define BUNDLE_SIZE WARP_SIZE
#define NEURONS_PER_WI {npw}
#define THREADS_PER_GROUP ((MAX_PARTITION_SIZE)/(NEURONS_PER_WI))
#define WARPS_PER_GROUP (THREADS_PER_GROUP / WARP_SIZE)
#define MIN_SYNAPTIC_DELAY 1
#define MAX_SYNAPTIC_DELAY {delay}
#define FLOAT_TYPE float
"""


PRELUDE = """#include <xmmintrin.h>
#include <pmmintrin.h>
#include "clemu_rt.hpp"
// FTZ/DAZ for one launch; the caller's MXCSR is restored on return
struct clemu_ftz_scope {
    unsigned saved;
    clemu_ftz_scope() : saved(_mm_getcsr()) {
        _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
        _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
    }
    ~clemu_ftz_scope() { _mm_setcsr(saved); }
};
"""


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(d) > os.path.getmtime(target) for d in deps)


def build_variant(name: str, force: bool = False, ref_root: str | None = None) -> str:
    """Build oracle/_ref/libclemu_<name>.so from the kernel sources under
    `ref_root` (default: reference_root()).  Without a reference checkout an
    existing library is returned as it is; a missing one is an error."""
    mps, warp, npw, delay = VARIANTS[name]
    lib = os.path.join(OUT, f"libclemu_{name}.so")
    ref_root = ref_root or reference_root()
    if ref_root is None:
        if os.path.exists(lib):
            return lib
        raise FileNotFoundError(f"{lib} is not built and no reference checkout is given "
                                "(set SZSNN_REFERENCE to the reference's root directory)")
    CL_DIR = cl_dir(ref_root)
    gen = os.path.join(OUT, "gen", name)
    os.makedirs(gen, exist_ok=True)
    deps = [os.path.join(HERE, "clemu_rt.cpp"), os.path.join(HERE, "clemu_rt.hpp"), os.path.abspath(__file__)]
    deps += [os.path.join(CL_DIR, f) for f, _, _ in KERNELS.values()]
    if not force and not _stale(lib, deps):
        return lib
    objs_src = [os.path.join(HERE, "clemu_rt.cpp")]
    for key, (fname, kname, is_update) in KERNELS.items():
        with open(os.path.join(CL_DIR, fname), encoding="latin-1") as f:
            body = rewrite(f.read(), key)
        flags = "#define SZSNN_KERNEL_OUTPUT_SPIKES 1\n" if is_update else ""
        if is_update:
            wrapper = UPDATE_WRAPPER.format(name=key, kernel=kname)
        elif key == "gather":
            wrapper = GATHER_WRAPPER
        else:
            wrapper = SCATTER_WRAPPER
        text = (PRELUDE + constants(mps, warp, npw, delay) + flags + "namespace {\n" + body + "\n}  // namespace\n"
                + wrapper)
        path = os.path.join(gen, f"{key}.cpp")
        with open(path, "w") as f:
            f.write(text)
        objs_src.append(path)
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-w",
           "-I", HERE, "-o", lib, *objs_src]
    subprocess.run(cmd, check=True)
    return lib


def build_clemu(ref_root: str, force: bool = False) -> list[str]:
    if not os.path.isdir(cl_dir(ref_root)):
        raise FileNotFoundError(f"reference kernel sources not found under {cl_dir(ref_root)}")
    return [build_variant(v, force, ref_root) for v in VARIANTS]


if __name__ == "__main__":
    # usage: python -m oracle.clemu.build_clemu <reference root> [--force]
    args = [a for a in sys.argv[1:] if a != "--force"]
    root = args[0] if args else reference_root()
    if not root:
        sys.exit("usage: build_clemu.py <reference root> [--force]  (or set SZSNN_REFERENCE)")
    for p in build_clemu(root, force="--force" in sys.argv):
        print(p)
