"""Oracle B backend: the reference's own OpenCL kernels on host cores.

TEST INFRASTRUCTURE ONLY.  `ClemuBackend` offers the kernel-backend interface
szsnn_b200.RefSimulation drives (buffer / write / read / gather / update /
scatter), over numpy buffers and the emulator-built reference kernels in
oracle/_ref/libclemu_<variant>.so, so one driver feeds the reference kernels
and the CUDA drop-in kernels with the same arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build_clemu import OUT, VARIANTS, build_variant

_libs = {}


def lib(variant: str = "prod"):
    if variant not in _libs:
        path = os.path.join(OUT, f"libclemu_{variant}.so")
        if not os.path.exists(path):
            build_variant(variant)
        h = C.CDLL(path)
        P, U32, U64 = C.c_void_p, C.c_uint32, C.c_ulong
        upd = [U64, U32, P, P, P, U32, P, P, U32, P, P, P, P, U32, U32]
        for k in ("if_curr_exp", "izhikevich", "const_rate"):
            f = getattr(h, "clemu_" + k)
            f.restype, f.argtypes = C.c_int, upd
        h.clemu_gather.restype = C.c_int
        h.clemu_gather.argtypes = [U64, U32, P, P, U64, P, P, P, P]
        h.clemu_scatter.restype = C.c_int
        h.clemu_scatter.argtypes = [U64, U32, P, P, U32, U32, P, P, U64, P, P, P, P, P]
        _libs[variant] = h
    return _libs[variant]


def available(variant: str = "prod") -> bool:
    try:
        lib(variant)
        return True
    except Exception:
        return False


class HostBuffer:
    def __init__(self, arr: np.ndarray):
        self.arr = np.ascontiguousarray(arr).copy()
        if self.arr.nbytes == 0:
            self.arr = np.zeros(16, np.uint8)
        self.ptr = self.arr.ctypes.data


class ClemuBackend:
    def __init__(self, variant: str = "prod"):
        self.variant = variant
        self.consts = VARIANTS[variant]
        self.h = lib(variant)

    def buffer(self, arr):
        return HostBuffer(arr)

    def write(self, buf: HostBuffer, arr) -> None:
        a = np.ascontiguousarray(arr)
        buf.arr.view(np.uint8)[: a.nbytes] = a.view(np.uint8).reshape(-1)

    def read(self, buf: HostBuffer, dtype, count: int) -> np.ndarray:
        return buf.arr.view(np.uint8).view(dtype)[:count].copy()

    def sync(self) -> None:
        pass

    @staticmethod
    def _a(x):
        return x.ptr if hasattr(x, "ptr") else x

    def update(self, model: str, *args) -> None:
        fn = {"IF_curr_exp": self.h.clemu_if_curr_exp, "Izhikevich": self.h.clemu_izhikevich,
              "Const_rate": self.h.clemu_const_rate}[model]
        if fn(*[self._a(a) for a in args]) != 0:
            raise RuntimeError("clemu: divergent barrier in " + model)

    def gather(self, *args) -> None:
        if self.h.clemu_gather(*[self._a(a) for a in args]) != 0:
            raise RuntimeError("clemu: divergent barrier in gather")

    def scatter(self, *args) -> None:
        if self.h.clemu_scatter(*[self._a(a) for a in args]) != 0:
            raise RuntimeError("clemu: divergent barrier in scatter")
