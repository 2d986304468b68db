"""CPU oracle for the SZSNN simulation step -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm import this package, as the checker.  The product (szsnn_b200/) never does.

  liboracle.so  ("Oracle A")  plain-C restatement of the reference step
                (oracle.c / oracle_step.inc), fp32 and fp64, float or
                fixed-point accumulation, multithreaded for timing
  clemu         ("Oracle B")  the reference's own OpenCL kernel sources
                (szsnn1.1/src/cl/*.cl) compiled for the CPU under a work-group
                emulator, built by oracle/clemu/build_clemu.py into oracle/_ref/
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

ACC_FLOAT, ACC_FIXED = 0, 1
MAX_POPS = 16


class OrcPop(C.Structure):
    _fields_ = [("model", C.c_int32), ("flags", C.c_uint32), ("begin", C.c_int64), ("end", C.c_int64),
                ("p", C.c_float * 12), ("pn", C.c_void_p), ("seed", C.c_uint64)]


class OrcNet(C.Structure):
    _fields_ = [("n_neurons", C.c_int64), ("n_sources", C.c_int64), ("max_delay", C.c_int32),
                ("n_pops", C.c_int32), ("pops", OrcPop * MAX_POPS), ("row_ptr", C.c_void_p),
                ("tgt", C.c_void_p), ("w", C.c_void_p)]


class OrcGenBlock(C.Structure):
    _fields_ = [("src_begin", C.c_int64), ("src_count", C.c_int64), ("tgt_begin", C.c_int64),
                ("tgt_count", C.c_int64), ("fanout", C.c_int32), ("exclude_self", C.c_int32),
                ("w_lo", C.c_float), ("w_hi", C.c_float), ("w_sign", C.c_float), ("d_lo", C.c_int32),
                ("d_hi", C.c_int32), ("stream", C.c_uint32), ("syn_offset", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from .build import build_oracle
            build_oracle()
        h = C.CDLL(LIB_PATH)
        P, I64, I = C.c_void_p, C.c_int64, C.c_int
        h.orc_run_f32.restype = C.c_uint64
        h.orc_run_f32.argtypes = [P, P, P, I64, I64, P, P, P, I, I, P, P]
        h.orc_run_f64.restype = C.c_uint64
        h.orc_run_f64.argtypes = [P, P, P, I64, I64, P, P, P, I]
        h.orc_gen_fixed_fanout.restype = None
        h.orc_gen_fixed_fanout.argtypes = [P, C.c_uint64, C.c_int32, P, P, P]
        h.orc_philox4x32.restype = None
        h.orc_philox4x32.argtypes = [P, P, P]
        _lib = h
    return _lib


def philox4x32(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def generate(blocks, seed: int, n_units: int, max_delay: int):
    """Fixed fan-out network, same algorithm as szsnn_net_generate.

    blocks: objects with the GenBlock fields; returns (row_ptr, tgt, w)."""
    total = sum(b.src_count * b.fanout for b in blocks)
    row_ptr = np.zeros(n_units * max_delay + 1, np.uint64)
    tgt = np.zeros(total, np.int32)
    w = np.zeros(total, np.float32)
    off = 0
    row = 0
    for b in blocks:
        row_ptr[row * max_delay: b.src_begin * max_delay] = off  # rows without synapses
        cb = OrcGenBlock(b.src_begin, b.src_count, b.tgt_begin, b.tgt_count, b.fanout,
                         1 if b.exclude_self else 0, b.w_lo, b.w_hi, b.w_sign, b.d_lo, b.d_hi, b.stream, off)
        lib().orc_gen_fixed_fanout(C.byref(cb), seed, max_delay, row_ptr.ctypes.data, tgt.ctypes.data,
                                   w.ctypes.data)
        off += b.src_count * b.fanout
        row = b.src_begin + b.src_count
    row_ptr[row * max_delay:] = off
    return row_ptr, tgt, w


class OracleNet:
    """Oracle A over a delay-bucketed CSR (the native network form).

    pops: objects with model/begin/end/params/per_unit/seed/flags (szsnn_b200.Pop
    has exactly these fields)."""

    def __init__(self, n_neurons: int, n_sources: int, max_delay: int, pops, csr, state=None,
                 dtype=np.float32):
        self.N, self.P, self.D = n_neurons, n_sources, max_delay
        self.U = n_neurons + n_sources
        self.W = (self.U + 31) // 32
        self.dtype = np.dtype(dtype)
        self._keep = []
        net = OrcNet()
        net.n_neurons, net.n_sources, net.max_delay, net.n_pops = n_neurons, n_sources, max_delay, len(pops)
        for i, p in enumerate(pops):
            op = OrcPop()
            op.model, op.flags, op.begin, op.end = p.model, getattr(p, "flags", 0), p.begin, p.end
            pv = np.zeros(12, np.float32)
            pv[: len(p.params)] = np.asarray(p.params, np.float32)
            for k in range(12):
                op.p[k] = float(pv[k])
            if getattr(p, "per_unit", None) is not None:
                a = np.zeros((12, p.end - p.begin), np.float32)
                pu = np.asarray(p.per_unit, np.float32)
                a[: pu.shape[0]] = pu
                a = np.ascontiguousarray(a)
                self._keep.append(a)
                op.pn = a.ctypes.data
            op.seed = getattr(p, "seed", 0)
            net.pops[i] = op
        rp = np.ascontiguousarray(csr[0], np.uint64)
        tg = np.ascontiguousarray(csr[1], np.int32)
        ww = np.ascontiguousarray(csr[2], np.float32)
        self._keep += [rp, tg, ww]
        net.row_ptr, net.tgt, net.w = rp.ctypes.data, tg.ctypes.data, ww.ctypes.data
        self.net = net
        self.state = [np.zeros(self.U, self.dtype) for _ in range(4)]
        if state is not None:
            for k in range(4):
                if state[k] is not None:
                    self.state[k] = np.array(state[k], dtype=self.dtype)
        self.hist = np.zeros(self.D * self.W, np.uint32)
        self.t = 0

    def run(self, steps: int, forced_words=None, current=None, acc_mode: int = ACC_FLOAT, nthreads: int = 1,
            want_inputs: bool = False):
        """Returns (raster [steps][W] uint32, events[, (in_exc, in_inh) of the last step])."""
        raster = np.zeros((steps, self.W), np.uint32)
        fz = None if forced_words is None else np.ascontiguousarray(forced_words, np.uint32)
        cu = None if current is None else np.ascontiguousarray(current, np.float32)
        st = (C.c_void_p * 4)(*[s.ctypes.data for s in self.state])
        ie = np.zeros(max(self.N, 1), np.float32)
        ii = np.zeros(max(self.N, 1), np.float32)
        if self.dtype == np.float32:
            ev = lib().orc_run_f32(C.byref(self.net), st, self.hist.ctypes.data, self.t, steps,
                                   None if cu is None else cu.ctypes.data, None if fz is None else fz.ctypes.data,
                                   raster.ctypes.data, acc_mode, nthreads,
                                   ie.ctypes.data if want_inputs else None, ii.ctypes.data if want_inputs else None)
        else:
            ev = lib().orc_run_f64(C.byref(self.net), st, self.hist.ctypes.data, self.t, steps,
                                   None if cu is None else cu.ctypes.data, None if fz is None else fz.ctypes.data,
                                   raster.ctypes.data, nthreads)
        self.t += steps
        if want_inputs:
            return raster, int(ev), (ie[: self.N], ii[: self.N])
        return raster, int(ev)
