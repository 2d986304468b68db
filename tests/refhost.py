"""Driver of oracle/_ref/refhost: the reference's own host code (NetworkGraph,
the layout builders, Simulation<float>) built against szsnn_b200/compat.

write_spec() writes the network and per-step firing input in the driver's
format (oracle/refhost/refhost_main.cpp); run() executes `refhost layout`
(host only) or `refhost run` (the drop-in kernels through the C ABI) and
returns its output records as numpy arrays.
"""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
DTYPES = {"partition_sizes": np.uint32, "neuron_params": np.float32, "neuron_vars": np.float32,
          "input_params": np.float32, "input_vars": np.float32, "targets": np.uint32, "weights": np.float32,
          "delay_bits": np.uint64, "group_ptrs": np.uint32, "group_matrix": np.uint32,
          "pitch_step_maxbundles": np.uint64, "fired_counts": np.uint32, "fired_ids": np.uint32}


def binary(small: bool = False) -> str:
    return os.path.join(REF_DIR, "refhost_small" if small else "refhost")


def available(small: bool = False) -> bool:
    return os.path.exists(binary(small))


def write_spec(path, model: int, params, vars_, rates, src, tgt, w, user_delay, forced):
    """model 0 IF_curr_exp (9 params, 4 vars) or 1 Izhikevich (4, 2);
    src >= n_neurons names input (src - n_neurons); forced: one id list (or
    None) per step, in the reference's global ids."""
    params = np.ascontiguousarray(params, np.float32)
    vars_ = np.ascontiguousarray(vars_, np.float32)
    rates = np.ascontiguousarray(rates, np.float32)
    n = params.shape[0]
    with open(path, "wb") as f:
        f.write(b"SZRH")
        f.write(struct.pack("<IIIIIQ", 1, model, n, len(rates), len(forced), len(src)))
        f.write(params.tobytes())
        f.write(vars_.tobytes())
        f.write(rates.tobytes())
        for a, dt in ((src, np.uint32), (tgt, np.uint32), (w, np.float32), (user_delay, np.uint32)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
        for ids in forced:
            ids = np.zeros(0, np.uint32) if ids is None else np.ascontiguousarray(ids, np.uint32)
            f.write(struct.pack("<I", len(ids)))
            f.write(ids.tobytes())


def read_records(path) -> dict:
    out = {}
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            (nl,) = struct.unpack("<I", h)
            name = f.read(nl).decode()
            es, count = struct.unpack("<IQ", f.read(12))
            buf = f.read(es * count)
            out[name] = np.frombuffer(buf, DTYPES.get(name, np.uint8)).copy()
    return out


def run(mode: str, spec_path, out_path, small: bool = False, timeout: int = 600) -> dict:
    r = subprocess.run([binary(small), mode, str(spec_path), str(out_path)], capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"refhost {mode} failed ({r.returncode}): {r.stderr[-2000:]}")
    return read_records(out_path)


def group_entries(ptrs: np.ndarray, matrix: np.ndarray) -> dict:
    """(source partition, neuron, delay) slot -> sorted (target partition,
    bundle) pairs, from groupPtrs / groupMatrix as uint32 pairs: the content
    of the scatter tables independent of the order of groupMatrix rows."""
    p = ptrs.reshape(-1, 2)
    m = matrix.reshape(-1, 2)
    out = {}
    for slot in np.nonzero(p[:, 1])[0]:
        begin, cnt = int(p[slot, 0]), int(p[slot, 1])
        out[int(slot)] = sorted(map(tuple, m[begin:begin + cnt].tolist()))
    return out
