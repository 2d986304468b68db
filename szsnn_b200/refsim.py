"""Reference-layout simulation driver: szsnn::Simulation<float> over the drop-in kernels.

Mirrors Simulation (szsnn1.1/src/Simulation.hpp:38-132, Simulation.ipp):
  constructor   -> layout built by szsnn_layout_build (NeuronData / SynapseData /
                   GroupData / queues / spikes / currents, Simulation.ipp:108-118)
                   and uploaded (prepareGPUMemory, :130-138)
  step(fInput)  -> gather, setFiringInput, update (+ input kernel), scatter with
                   the cycle argument = steps done (Simulation.ipp:471-496)
  stepAndFired  -> step + firedOutput bitvector read back and converted to
                   sorted global ids (SpikeBuffer::getOutput, SpikeBuffer.cpp:136-165)

The kernels come from a backend object.  `CudaRefBackend` runs the sm_100a
drop-in kernels of libszsnn_cuda.so; tests pass the reference's own OpenCL
kernels compiled for the CPU through the same interface, so one driver feeds
both with identical buffers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .models import PARAM_COUNT, VAR_COUNT

MODEL_IDS = {"IF_curr_exp": L.IF_CURR_EXP, "Izhikevich": L.IZHIKEVICH}


class CudaRefBackend:
    """Drop-in kernels of libszsnn_cuda.so on device buffers of a Context."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.lib = L.lib()

    def buffer(self, arr: np.ndarray):
        a = np.ascontiguousarray(arr)
        return self.ctx.upload(a) if a.nbytes else self.ctx.buffer(16)

    def write(self, buf, arr: np.ndarray) -> None:
        buf.write(arr)

    def read(self, buf, dtype, count: int) -> np.ndarray:
        return buf.read(dtype, count)

    def sync(self) -> None:
        self.ctx.sync()

    def update(self, model: str, *args) -> None:
        fn = {"IF_curr_exp": self.lib.szsnn_update_if_curr_exp,
              "Izhikevich": self.lib.szsnn_update_izhikevich,
              "Const_rate": self.lib.szsnn_update_const_rate}[model]
        L.check(fn(self.ctx.h, *[_arg(a) for a in args]), self.ctx.h, model + "_update")

    def gather(self, *args) -> None:
        L.check(self.lib.szsnn_gather(self.ctx.h, *[_arg(a) for a in args]), self.ctx.h, "gather")

    def scatter(self, *args) -> None:
        L.check(self.lib.szsnn_scatter(self.ctx.h, *[_arg(a) for a in args]), self.ctx.h, "scatter")


def _arg(a):
    return a.ptr if hasattr(a, "ptr") else a


def build_layout(consts: L.LayoutConsts, n_neurons: int, neuron_params: np.ndarray, neuron_vars: np.ndarray,
                 src, tgt, weight, delay1, n_inputs: int = 0, input_params=None, input_vars=None,
                 add_phony: bool = True):
    """Host layout (no GPU needed).  Returns (info, {array id: np.ndarray})."""
    lib = L.lib()
    npar = np.ascontiguousarray(neuron_params, dtype=np.float32)
    nvar = np.ascontiguousarray(neuron_vars, dtype=np.float32)
    ipar = np.ascontiguousarray(input_params if input_params is not None else np.zeros((n_inputs, 1)), dtype=np.float32)
    ivar = np.ascontiguousarray(input_vars if input_vars is not None else np.zeros((n_inputs, 1)), dtype=np.float32)
    s = np.ascontiguousarray(src, dtype=np.uint32)
    t = np.ascontiguousarray(tgt, dtype=np.uint32)
    w = np.ascontiguousarray(weight, dtype=np.float32)
    d1 = np.ascontiguousarray(delay1, dtype=np.uint32)
    desc = L.LayoutDesc(n_neurons, n_inputs, npar.shape[1], nvar.shape[1], ipar.shape[1] if n_inputs else 0,
                        ivar.shape[1] if n_inputs else 0, npar.ctypes.data, nvar.ctypes.data,
                        ipar.ctypes.data if n_inputs else None, ivar.ctypes.data if n_inputs else None,
                        len(s), s.ctypes.data, t.ctypes.data, w.ctypes.data, d1.ctypes.data, 1 if add_phony else 0)
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = lib.szsnn_layout_build(C.byref(consts), C.byref(desc), C.byref(h), err, 512)
    if rc:
        raise L.SzsnnError(rc, "layout: " + err.value.decode())
    info = L.LayoutInfo()
    lib.szsnn_layout_info_get(h, C.byref(info))
    dtypes = {L.L_PARTITION_SIZES: np.uint32, L.L_NEURON_PARAMS: np.float32, L.L_NEURON_VARS: np.float32,
              L.L_INPUT_PARAMS: np.float32, L.L_INPUT_VARS: np.float32, L.L_TARGETS: np.uint32,
              L.L_WEIGHTS: np.float32, L.L_DELAY_BITS: np.uint64, L.L_GROUP_PTRS: np.uint32,
              L.L_GROUP_MATRIX: np.uint32, L.L_GQ_COUNTER: np.uint32, L.L_GQ_BUNDLES: np.uint32,
              L.L_LQ_COUNTER: np.uint32, L.L_LQ_ENTRIES: np.int16, L.L_FIRED: np.uint32,
              L.L_FIRED_COUNT: np.uint32, L.L_FIRED_INPUT: np.uint32, L.L_FIRED_OUTPUT: np.uint32,
              L.L_INPUT_CURRENT: np.float32, L.L_CURRENT: np.float32}
    arrays = {}
    for k in range(L.L_COUNT):
        nb = int(info.bytes[k])
        a = np.zeros(nb // np.dtype(dtypes[k]).itemsize, dtype=dtypes[k])
        lib.szsnn_layout_array(h, k, a.ctypes.data if nb else None, nb)
        arrays[k] = a
    lib.szsnn_layout_free(h)
    return info, arrays


class RefSimulation:
    """Simulation<float> on the reference layout with a pluggable kernel backend."""

    def __init__(self, backend, consts: L.LayoutConsts, model: str, neuron_params: np.ndarray,
                 neuron_vars: np.ndarray, src, tgt, weight, delay1, input_params=None, input_vars=None,
                 add_phony: bool = True):
        if model not in MODEL_IDS:
            raise ValueError(f"unknown neuron model {model}")
        mid = MODEL_IDS[model]
        neuron_params = np.asarray(neuron_params, dtype=np.float32)
        neuron_vars = np.asarray(neuron_vars, dtype=np.float32)
        if neuron_params.shape[1] != PARAM_COUNT[mid] or neuron_vars.shape[1] != VAR_COUNT[mid]:
            raise ValueError("parameter / variable count does not match the model traits")
        ctx_consts = getattr(getattr(backend, "ctx", None), "consts", None)
        if ctx_consts is not None and tuple(ctx_consts.__getattribute__(f) for f, _ in consts._fields_) != \
                tuple(consts.__getattribute__(f) for f, _ in consts._fields_):
            # the drop-in kernels size their indexing by the context's constants
            raise ValueError("layout constants differ from the context's: create the Context with the same "
                             "max_partition_size / threads_per_group / warp_size / max_synaptic_delay")
        self.model = model
        self.backend = backend
        self.consts = consts
        self.n_neurons = neuron_params.shape[0]
        self.n_inputs = 0 if input_params is None else len(input_params)
        self.info, arr = build_layout(consts, self.n_neurons, neuron_params, neuron_vars, src, tgt, weight, delay1,
                                      self.n_inputs, input_params, input_vars, add_phony)
        self.arrays_host = arr
        self.mps = consts.max_partition_size
        self.bvwp = self.mps // 32
        self.pn = self.info.neuron_partitions
        self.ptot = self.info.total_partitions
        self.buf = {k: backend.buffer(a) for k, a in arr.items()}
        self.cycle = 0
        self.is_input_set = 0

    # SpikeBuffer::setInput (SpikeBuffer.cpp:97-129): an empty list leaves the
    # previous input in force; setInput() with no list clears the flag.
    def _set_firing_input(self, fired_input):
        if fired_input is None:
            self.is_input_set = 0
            return
        ids = np.asarray(fired_input, dtype=np.int64)
        if ids.size == 0:
            return
        part = ids // self.mps
        if np.any(part >= self.ptot):
            raise ValueError("forced spike for a neuron outside the network")
        vec = np.zeros(self.ptot * self.bvwp, dtype=np.uint32)
        loc = ids % self.mps
        np.bitwise_or.at(vec, part * self.bvwp + loc // 32, (np.uint32(1) << (loc % 32).astype(np.uint32)))
        self.backend.write(self.buf[L.L_FIRED_INPUT], vec)
        self.is_input_set = 1

    def step(self, fired_input=None, input_current=None) -> None:
        b, B = self.backend, self.buf
        c = self.cycle
        # prefire: gather (Simulation.ipp:402-420)
        b.gather(c, self.ptot, B[L.L_PARTITION_SIZES], B[L.L_CURRENT], self.info.gq_pitch, B[L.L_GQ_COUNTER],
                 B[L.L_GQ_BUNDLES], B[L.L_TARGETS], B[L.L_WEIGHTS])
        self._set_firing_input(fired_input)
        iic = 0
        if input_current is not None:  # kernel args 5/6, left at 0 by the reference host (:465)
            cur = np.zeros(self.ptot * self.mps, dtype=np.float32)
            ic = np.asarray(input_current, dtype=np.float32)
            ids = np.arange(len(ic))
            cur[(ids // self.mps) * self.mps + ids % self.mps] = ic
            b.write(B[L.L_INPUT_CURRENT], cur)
            iic = 1
        # fire: update + input kernels (:423-441)
        b.update(self.model, c, self.pn, B[L.L_PARTITION_SIZES], B[L.L_NEURON_PARAMS], B[L.L_NEURON_VARS], iic,
                 B[L.L_INPUT_CURRENT], B[L.L_CURRENT], self.is_input_set, B[L.L_FIRED_INPUT], B[L.L_FIRED_COUNT],
                 B[L.L_FIRED], B[L.L_FIRED_OUTPUT], 0, self.ptot)
        if self.n_inputs:
            b.update("Const_rate", c, 1, B[L.L_PARTITION_SIZES], B[L.L_INPUT_PARAMS], B[L.L_INPUT_VARS], iic,
                     B[L.L_INPUT_CURRENT], B[L.L_CURRENT], self.is_input_set, B[L.L_FIRED_INPUT],
                     B[L.L_FIRED_COUNT], B[L.L_FIRED], B[L.L_FIRED_OUTPUT], self.pn, self.ptot)
        # postfire: scatter (:444-460)
        b.scatter(c, self.ptot, B[L.L_FIRED_COUNT], B[L.L_FIRED], self.info.group_pitch, self.info.group_step,
                  B[L.L_GROUP_PTRS], B[L.L_GROUP_MATRIX], self.info.gq_pitch, B[L.L_GQ_COUNTER], B[L.L_GQ_BUNDLES],
                  B[L.L_LQ_COUNTER], B[L.L_LQ_ENTRIES], B[L.L_DELAY_BITS])
        self.cycle += 1

    def fired_output_words(self) -> np.ndarray:
        """firedOutput of the neuron partitions, [Pn][MPS/32] uint32."""
        return self.backend.read(self.buf[L.L_FIRED_OUTPUT], np.uint32, self.pn * self.bvwp).reshape(self.pn, self.bvwp)

    def step_and_fired(self, fired_input=None, input_current=None) -> np.ndarray:
        self.step(fired_input, input_current)
        words = self.fired_output_words()
        # bitvectorToSparse (SpikeBuffer.cpp:144-165)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").reshape(self.pn, self.mps)
        p, n = np.nonzero(bits)
        return (p * self.mps + n).astype(np.int64)

    def neuron_vars(self) -> np.ndarray:
        """Neuron variables as [var_count][n_neurons]."""
        vc = VAR_COUNT[MODEL_IDS[self.model]]
        raw = self.backend.read(self.buf[L.L_NEURON_VARS], np.float32, vc * self.pn * self.mps)
        raw = raw.reshape(vc, self.pn * self.mps)
        ids = np.arange(self.n_neurons)
        return raw[:, (ids // self.mps) * self.mps + ids % self.mps]

    def currents(self) -> np.ndarray:
        """g_current as [2][n_neurons] (exc, inh) -- the last gather's output."""
        raw = self.backend.read(self.buf[L.L_CURRENT], np.float32, 2 * self.ptot * self.mps).reshape(2, self.ptot * self.mps)
        ids = np.arange(self.n_neurons)
        return raw[:, (ids // self.mps) * self.mps + ids % self.mps]

    def sync(self) -> None:
        self.backend.sync()
