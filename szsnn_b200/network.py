"""Native network path: delay-bucketed CSR, device spike ring, CUDA graphs.

A Network is the B200 form of Simulation + NetworkGraph for networks beyond
the reference layout's limits (<= 64 delay steps, <= 256 partitions, bundles
padded to 32 slots -- GroupData.cpp:94-228, scatter_kernel.cl:82,291).
Units are neurons 0..N-1 followed by sources N..N+P-1; a spike emitted at
step t over a synapse of delay m (m = user delay + 1, NetworkGraph.ipp:431)
is integrated by the update of step t + m, exactly as the reference's
scatter/gather double buffer delivers it (scatter_kernel.cl:154,207,325;
gather_kernel.cl:55-58).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class Pop:
    model: int
    begin: int
    end: int
    params: np.ndarray = field(default_factory=lambda: np.zeros(12, np.float32))
    per_unit: np.ndarray | None = None   # [12][end-begin] fp32, overrides params
    seed: int = 0
    flags: int = 0

    def to_c(self, keep: list) -> L.PopDesc:
        p = L.PopDesc()
        p.model, p.flags, p.begin, p.end = self.model, self.flags, self.begin, self.end
        pv = np.zeros(12, np.float32)
        pv[: len(self.params)] = np.asarray(self.params, np.float32)
        for i in range(12):
            p.p[i] = float(pv[i])
        if self.per_unit is not None:
            a = np.zeros((12, self.end - self.begin), np.float32)
            pu = np.asarray(self.per_unit, np.float32)
            a[: pu.shape[0]] = pu
            a = np.ascontiguousarray(a)
            keep.append(a)
            p.pn_host = a.ctypes.data
        p.seed = self.seed
        return p


@dataclass
class GenBlock:
    """Fixed fan-out generator block (see szsnn_gen_block)."""
    src_begin: int
    src_count: int
    tgt_begin: int
    tgt_count: int
    fanout: int
    w_lo: float
    w_hi: float
    w_sign: float = 1.0
    d_lo: int = 1
    d_hi: int = 1
    exclude_self: bool = False
    stream: int = 0

    def to_c(self, syn_offset: int) -> L.GenBlock:
        return L.GenBlock(self.src_begin, self.src_count, self.tgt_begin, self.tgt_count, self.fanout,
                          1 if self.exclude_self else 0, self.w_lo, self.w_hi, self.w_sign, self.d_lo, self.d_hi,
                          self.stream, syn_offset)


def csr_from_synapses(n_units: int, max_delay: int, src, tgt, w, delay):
    """Bucket a synapse list into (row_ptr, tgt, w): rows by source, stably by delay."""
    src = np.asarray(src, np.int64)
    delay = np.asarray(delay, np.int64)
    if len(src) and (delay.min() < 1 or delay.max() > max_delay):
        raise ValueError("delays must be in 1..max_delay")
    key = src * max_delay + (delay - 1)
    order = np.argsort(key, kind="stable")
    counts = np.bincount(key, minlength=n_units * max_delay) if len(src) else np.zeros(n_units * max_delay, np.int64)
    row_ptr = np.zeros(n_units * max_delay + 1, np.uint64)
    row_ptr[1:] = np.cumsum(counts, dtype=np.uint64)
    return row_ptr, np.asarray(tgt, np.int32)[order].copy(), np.asarray(w, np.float32)[order].copy()


class Network:
    def __init__(self, ctx, n_neurons: int, n_sources: int, max_delay: int, pops: list[Pop], csr=None,
                 state=None, acc_mode: int = L.ACC_FLOAT, graph_chunk: int = 100, n_synapses: int | None = None,
                 groups=None, n_groups: int = 0):
        self.ctx = ctx
        self.lib = L.lib()
        self.N, self.P, self.D = int(n_neurons), int(n_sources), int(max_delay)
        self.U = self.N + self.P
        self.words = (self.U + 31) // 32
        self.pops = pops
        d = L.NetDesc()
        d.n_neurons, d.n_sources, d.max_delay, d.n_pops = self.N, self.P, self.D, len(pops)
        keep = []
        pop_arr = (L.PopDesc * max(len(pops), 1))()
        for i, p in enumerate(pops):
            pop_arr[i] = p.to_c(keep)
        keep.append(pop_arr)
        d.pops = C.cast(pop_arr, C.c_void_p)
        if groups is not None:
            g = np.ascontiguousarray(groups, np.int32)
            if len(g) != self.U:
                raise ValueError("groups must have one entry per unit")
            keep.append(g)
            d.group_host = g.ctypes.data
            d.n_groups = int(n_groups or (g.max() + 1))
        self.n_groups = int(d.n_groups)
        if csr is not None:
            rp, tg, ww = (np.ascontiguousarray(csr[0], np.uint64), np.ascontiguousarray(csr[1], np.int32),
                          np.ascontiguousarray(csr[2], np.float32))
            keep += [rp, tg, ww]
            d.n_synapses = len(tg)
            d.row_ptr_host, d.tgt_host, d.w_host = rp.ctypes.data, tg.ctypes.data, ww.ctypes.data
        else:
            d.n_synapses = int(n_synapses or 0)
        if state is not None:
            for k in range(4):
                if state[k] is not None:
                    a = np.ascontiguousarray(state[k], np.float32)
                    if len(a) != self.U:
                        raise ValueError("state slots must have n_neurons + n_sources entries")
                    keep.append(a)
                    d.state_host[k] = a.ctypes.data
        d.acc_mode = acc_mode
        d.graph_chunk = graph_chunk
        h = C.c_void_p()
        L.check(self.lib.szsnn_net_create(ctx.h, C.byref(d), C.byref(h)), ctx.h, "net_create")
        self.h = h.value
        self.n_synapses = int(d.n_synapses)
        self.graph_chunk = graph_chunk  # steps per CUDA graph (0: the library's default of 100)
        if not self.graph_chunk:
            self.graph_chunk = 100

    def generate(self, blocks: list[GenBlock], seed: int) -> None:
        off = 0
        arr = (L.GenBlock * max(len(blocks), 1))()
        for i, b in enumerate(blocks):
            arr[i] = b.to_c(off)
            off += b.src_count * b.fanout
        L.check(self.lib.szsnn_net_generate(self.h, arr, len(blocks), seed), self.ctx.h, "net_generate")
        self.n_synapses = off

    # Simulation::stepAndFired(fInput) (Simulation.ipp:517-530)
    def step(self, forced_words=None, current=None, fired=True) -> np.ndarray | None:
        fw = None if forced_words is None else np.ascontiguousarray(forced_words, np.uint32)
        cu = None if current is None else np.ascontiguousarray(current, np.float32)
        out = np.zeros(self.words, np.uint32) if fired else None
        L.check(self.lib.szsnn_net_step(self.h, None if fw is None else fw.ctypes.data,
                                        None if cu is None else cu.ctypes.data,
                                        None if out is None else out.ctypes.data), self.ctx.h, "net_step")
        return out

    def set_owned(self, n_lo: int, n_hi: int, s_lo: int, s_hi: int) -> None:
        """Update only neurons [n_lo, n_hi) and sources [s_lo, s_hi) (one shard)."""
        L.check(self.lib.szsnn_net_set_owned(self.h, n_lo, n_hi, s_lo, s_hi), self.ctx.h, "set_owned")

    def inject_spikes(self, words) -> None:
        """Spike words of the step just done from units other shards update
        (szsnn_net_inject_spikes)."""
        w = np.ascontiguousarray(words, np.uint32)
        if w.shape != (self.words,):
            raise ValueError("inject_spikes takes one step's words")
        L.check(self.lib.szsnn_net_inject_spikes(self.h, w.ctypes.data), self.ctx.h, "inject_spikes")

    def run(self, steps: int, forced_words=None, raster=True, out=None) -> np.ndarray | None:
        """`steps` steps from the host: forced-spike words [steps, words] in,
        raster words [steps, words] out.  Page-locked arrays (`out`, or
        `forced_words`) are copied by DMA directly; pageable ones go through the
        library's pinned bounce buffers."""
        fw = None if forced_words is None else np.ascontiguousarray(forced_words, np.uint32)
        if out is not None:
            if out.dtype != np.uint32 or out.shape != (steps, self.words) or not out.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous uint32 array of shape (steps, words)")
        elif raster:
            out = np.zeros((steps, self.words), np.uint32)
        L.check(self.lib.szsnn_net_run(self.h, steps, None if fw is None else fw.ctypes.data,
                                       None if out is None else out.ctypes.data), self.ctx.h, "net_run")
        return out

    def run_device(self, steps: int, forced_ptr=None, current_ptr=None, raster_ptr=None) -> None:
        L.check(self.lib.szsnn_net_run_device(self.h, steps, forced_ptr, current_ptr, raster_ptr), self.ctx.h,
                "net_run_device")

    def set_monitor(self, ids, slots=(0,), capacity: int = 1000) -> None:
        """Record state slots `slots` of units `ids` after every step, on the
        device, for up to `capacity` steps between reads (ids=[] turns it off)."""
        ids = np.ascontiguousarray(ids, np.int32)
        mask = 0
        for k in slots:
            if not 0 <= int(k) <= 3:
                raise ValueError("state slots are 0..3")
            mask |= 1 << int(k)
        self._mon = (len(ids), bin(mask).count("1"), int(capacity)) if len(ids) else None
        L.check(self.lib.szsnn_net_set_monitor(self.h, ids.ctypes.data if len(ids) else None, len(ids), mask,
                                               int(capacity)), self.ctx.h, "set_monitor")

    def monitor_read(self) -> tuple[np.ndarray, int]:
        """(trace [steps, slots, units] fp32 since set_monitor or the last read,
        steps not recorded because they ran past the capacity); recording then
        restarts at the current step."""
        if getattr(self, "_mon", None) is None:
            raise ValueError("no monitor is set")
        n, ns, cap = self._mon
        out = np.zeros((cap, ns, n), np.float32)
        steps, dropped = C.c_int64(), C.c_int64()
        L.check(self.lib.szsnn_net_monitor_read(self.h, out.ctypes.data, cap, C.byref(steps), C.byref(dropped)),
                self.ctx.h, "monitor_read")
        return out[: steps.value].copy(), int(dropped.value)

    def device_ms(self) -> float:
        """Device time (CUDA events on the net's stream) of the last run / run_device."""
        t = C.c_double()
        L.check(L.lib().szsnn_net_timing(self.h, None, None, C.byref(t)), self.ctx.h, "net timing")
        return float(t.value)

    def profile(self, steps: int) -> tuple[float, float, float]:
        """(propagate ms, update ms) summed over `steps` replays of the current
        step on scratch state, and the events one propagate launch delivers."""
        p, u, ev = C.c_double(), C.c_double(), C.c_double()
        L.check(self.lib.szsnn_net_profile(self.h, steps, C.byref(p), C.byref(u), C.byref(ev)), self.ctx.h,
                "profile")
        return p.value, u.value, ev.value

    def profile_step(self, steps: int) -> dict:
        """Device ms of `steps` replays each of the delivery launch, the update
        launch and the whole step (overlapped: the fused launch), on scratch
        state, and the events one delivery launch delivers."""
        p, u, st, ev = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        L.check(self.lib.szsnn_net_profile_step(self.h, steps, C.byref(p), C.byref(u), C.byref(st), C.byref(ev)),
                self.ctx.h, "profile_step")
        return {"propagate_ms": p.value, "update_ms": u.value, "step_ms": st.value, "events_per_launch": ev.value}

    def set_tuning(self, mode: int = 0, group: int = 0, blocks: int = -1, update_block: int = 0) -> None:
        L.check(self.lib.szsnn_net_set_tuning(self.h, mode, group, blocks, update_block), self.ctx.h, "set_tuning")

    def set_update_tiles(self, mode: int, blocks_per_sm: int = 0) -> None:
        """0: a block per update tile each step; 1: persistent warp tiles with
        `blocks_per_sm` update blocks per SM (0: the default of 2); 2:
        persistent block tiles (`blocks_per_sm`, 0: as many as stay resident)."""
        L.check(self.lib.szsnn_net_set_update_tiles(self.h, mode, blocks_per_sm), self.ctx.h, "set_update_tiles")

    def set_update_units(self, units_per_thread: int) -> None:
        """Units per update thread (0: automatic)."""
        L.check(self.lib.szsnn_net_set_update_units(self.h, units_per_thread), self.ctx.h, "set_update_units")

    def set_resident(self, on: bool, update_warps: int = 0, blocks: int = 0) -> None:
        """Resident stepping: each run chunk is one cooperative launch that
        keeps the neurons' state in shared memory across its steps
        (`update_warps` of each block's 32 warps update, 0: 16; `blocks`, 0:
        one per SM).  Raises SzsnnError with the reason when the network does
        not qualify."""
        L.check(self.lib.szsnn_net_set_resident(self.h, 1 if on else 0, update_warps, blocks), self.ctx.h,
                "set_resident")

    overlap = True

    def set_overlap(self, on: bool) -> None:
        """Overlapped step order (default) or the classic propagate-then-update order."""
        L.check(self.lib.szsnn_net_set_overlap(self.h, 1 if on else 0), self.ctx.h, "set_overlap")
        self.overlap = bool(on)

    def stats(self) -> dict:
        s = L.NetStats()
        L.check(self.lib.szsnn_net_stats_get(self.h, C.byref(s)), self.ctx.h, "stats")
        return dict(steps_done=s.steps_done, events=s.events, spikes=s.spikes,
                    graph_launches=s.graph_launches, kernel_launches=s.kernel_launches)

    def group_spikes(self, reset: bool = False) -> np.ndarray:
        out = np.zeros(self.n_groups, np.uint64)
        L.check(self.lib.szsnn_net_group_spikes(self.h, out.ctypes.data, 1 if reset else 0), self.ctx.h,
                "group_spikes")
        return out

    def get_state(self, slot: int) -> np.ndarray:
        out = np.zeros(self.U, np.float32)
        L.check(self.lib.szsnn_net_get_state(self.h, slot, out.ctypes.data), self.ctx.h, "get_state")
        return out

    def set_state(self, slot: int, values) -> None:
        a = np.ascontiguousarray(values, np.float32)
        if len(a) != self.U:
            raise ValueError("state slot length must be n_neurons + n_sources")
        L.check(self.lib.szsnn_net_set_state(self.h, slot, a.ctypes.data), self.ctx.h, "set_state")

    def checkpoint(self) -> bytes:
        n = C.c_uint64()
        L.check(self.lib.szsnn_net_checkpoint_size(self.h, C.byref(n)), self.ctx.h)
        buf = np.zeros(n.value, np.uint8)
        L.check(self.lib.szsnn_net_checkpoint(self.h, buf.ctypes.data, n.value), self.ctx.h, "checkpoint")
        return buf.tobytes()

    def restore(self, blob: bytes) -> None:
        a = np.frombuffer(blob, np.uint8).copy()
        L.check(self.lib.szsnn_net_restore(self.h, a.ctypes.data, len(a)), self.ctx.h, "restore")

    def synapses(self):
        rp = np.zeros(self.U * self.D + 1, np.uint64)
        tg = np.zeros(self.n_synapses, np.int32)
        ww = np.zeros(self.n_synapses, np.float32)
        L.check(self.lib.szsnn_net_get_synapses(self.h, rp.ctypes.data, tg.ctypes.data, ww.ctypes.data),
                self.ctx.h, "get_synapses")
        return rp, tg, ww

    def last_inputs(self):
        e = np.zeros(self.N, np.float32)
        i = np.zeros(self.N, np.float32)
        L.check(self.lib.szsnn_net_last_inputs(self.h, e.ctypes.data, i.ctypes.data), self.ctx.h)
        return e, i

    def check_finite(self) -> bool:
        f = C.c_int()
        L.check(self.lib.szsnn_net_check_finite(self.h, C.byref(f)), self.ctx.h)
        return bool(f.value)

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.ctx.h is not None:
            self.lib.szsnn_net_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def words_to_ids(words: np.ndarray, n_units: int) -> np.ndarray:
    bits = np.unpackbits(np.ascontiguousarray(words, np.uint32).view(np.uint8), bitorder="little")
    return np.nonzero(bits[:n_units])[0]


def ids_to_words(ids, n_units: int) -> np.ndarray:
    w = np.zeros((n_units + 31) // 32, np.uint32)
    ids = np.asarray(ids, np.int64)
    np.bitwise_or.at(w, ids // 32, (np.uint32(1) << (ids % 32).astype(np.uint32)))
    return w
