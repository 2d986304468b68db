"""Context and device buffers -- the Python face of szsnn::Context.

Mirrors the reference's Context (szsnn1.1/src/Context.hpp:77-303): setup picks
the device and creates the one in-order queue (here a CUDA stream),
createBuffer / writeBuffer / readBuffer move data, and every failure raises
(the reference throws SzsnnException on any CL status, utils.h:144-155).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class DeviceBuffer:
    """A device allocation owned by a Context (DataBuffer's cl::Buffer half)."""

    def __init__(self, ctx: "Context", nbytes: int):
        self.ctx = ctx
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        L.check(L.lib().szsnn_alloc(ctx.h, C.c_size_t(max(self.nbytes, 1)), C.byref(p)), ctx.h, "alloc")
        self.ptr = p.value

    def write(self, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr)
        if a.nbytes > self.nbytes:
            raise ValueError(f"write of {a.nbytes} bytes into a {self.nbytes}-byte buffer")
        L.check(L.lib().szsnn_h2d(self.ctx.h, self.ptr, a.ctypes.data, a.nbytes), self.ctx.h, "h2d")

    def read(self, dtype, count: int | None = None) -> np.ndarray:
        dt = np.dtype(dtype)
        n = self.nbytes // dt.itemsize if count is None else int(count)
        out = np.empty(n, dtype=dt)
        if out.nbytes > self.nbytes:
            raise ValueError("read beyond the buffer")
        L.check(L.lib().szsnn_d2h(self.ctx.h, out.ctypes.data, self.ptr, out.nbytes), self.ctx.h, "d2h")
        return out

    def zero(self) -> None:
        L.check(L.lib().szsnn_memset(self.ctx.h, self.ptr, 0, self.nbytes), self.ctx.h, "memset")

    def free(self) -> None:
        if self.ptr is not None and self.ctx.h is not None:
            L.check(L.lib().szsnn_free(self.ctx.h, self.ptr), self.ctx.h, "free")
        self.ptr = None


class Context:
    """One device, one stream, the layout constants of the reference build."""

    def __init__(self, device: int = 0, max_partition_size: int = 1024, threads_per_group: int = 256,
                 warp_size: int = 32, max_synaptic_delay: int = 64):
        self.consts = L.LayoutConsts(max_partition_size, threads_per_group, warp_size, max_synaptic_delay)
        h = C.c_void_p()
        L.check(L.lib().szsnn_ctx_create(device, C.byref(self.consts), C.byref(h)), None, "ctx_create")
        self.h = h.value
        self.device = device

    # --- Context::createBuffer / writeBuffer / readBuffer
    def buffer(self, nbytes: int) -> DeviceBuffer:
        return DeviceBuffer(self, nbytes)

    def upload(self, arr: np.ndarray) -> DeviceBuffer:
        a = np.ascontiguousarray(arr)
        b = DeviceBuffer(self, a.nbytes)
        b.write(a)
        return b

    def sync(self) -> None:
        L.check(L.lib().szsnn_sync(self.h), self.h, "sync")

    def probe_peaks(self, n_targets: int = 1_000_000) -> dict:
        """Measured on-chip ceilings of this device (szsnn_probe_peaks): the
        L2-resident copy bandwidth and the random fp32 reduction rate into
        2 * n_targets floats."""
        p = L.Peaks()
        L.check(L.lib().szsnn_probe_peaks(self.h, int(n_targets), C.byref(p)), self.h, "probe_peaks")
        return {"l2_copy_gbs": p.l2_copy_gbs, "l2_copy_bytes": p.l2_copy_bytes, "red_per_s": p.red_per_s,
                "red_targets": p.red_targets}

    def device_error(self) -> tuple[int, int]:
        code, info = C.c_uint32(), C.c_uint32()
        L.check(L.lib().szsnn_device_error(self.h, C.byref(code), C.byref(info)), self.h, "device_error")
        return code.value, info.value

    def clear_device_error(self) -> None:
        L.check(L.lib().szsnn_clear_device_error(self.h), self.h)

    def set_option(self, option: int, value: int) -> None:
        L.check(L.lib().szsnn_set_option(self.h, option, value), self.h, "set_option")

    def set_stream(self, stream_ptr: int) -> None:
        L.check(L.lib().szsnn_set_stream(self.h, C.c_void_p(stream_ptr)), self.h, "set_stream")

    @property
    def stream(self) -> int:
        return L.lib().szsnn_get_stream(self.h) or 0

    def close(self) -> None:
        if self.h is not None:
            L.lib().szsnn_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
