"""ctypes binding of libszsnn_cuda.so (declarations in include/szsnn_cuda.h).

The library is the product: there is no Python or CPU fallback.  Loading fails
loudly when the shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libszsnn_cuda.so")

SZSNN_OK = 0
ERR_NAMES = {1: "ARG", 2: "CUDA", 3: "NOMEM", 4: "LIMIT", 5: "DEVICE", 6: "TIMEOUT", 7: "STATE"}

IF_CURR_EXP, IF_COND_EXP, IZHIKEVICH, POISSON, CONST_RATE = 0, 1, 2, 3, 4
MAX_POPS = 65536
POP_IZH_HALF_STEPS = 1
ACC_FLOAT, ACC_FIXED = 0, 1

OPT_OUTPUT_SPARSE_INPUT, OPT_FIRED_OUTPUT_PARTS, OPT_IZH_HALF_STEPS = 1, 2, 3

(L_PARTITION_SIZES, L_NEURON_PARAMS, L_NEURON_VARS, L_INPUT_PARAMS, L_INPUT_VARS, L_TARGETS,
 L_WEIGHTS, L_DELAY_BITS, L_GROUP_PTRS, L_GROUP_MATRIX, L_GQ_COUNTER, L_GQ_BUNDLES, L_LQ_COUNTER,
 L_LQ_ENTRIES, L_FIRED, L_FIRED_COUNT, L_FIRED_INPUT, L_FIRED_OUTPUT, L_INPUT_CURRENT,
 L_CURRENT, L_COUNT) = range(21)


class SzsnnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"szsnn error {code} ({ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class LayoutConsts(C.Structure):
    _fields_ = [("max_partition_size", C.c_uint32), ("threads_per_group", C.c_uint32),
                ("warp_size", C.c_uint32), ("max_synaptic_delay", C.c_uint32)]


class LayoutDesc(C.Structure):
    _fields_ = [("n_neurons", C.c_uint32), ("n_inputs", C.c_uint32),
                ("neuron_param_count", C.c_uint32), ("neuron_var_count", C.c_uint32),
                ("input_param_count", C.c_uint32), ("input_var_count", C.c_uint32),
                ("neuron_params", C.c_void_p), ("neuron_vars", C.c_void_p),
                ("input_params", C.c_void_p), ("input_vars", C.c_void_p),
                ("n_synapses", C.c_uint64), ("src", C.c_void_p), ("tgt", C.c_void_p),
                ("weight", C.c_void_p), ("delay1", C.c_void_p), ("add_phony_synapse", C.c_uint32)]


class LayoutInfo(C.Structure):
    _fields_ = [("neuron_partitions", C.c_uint32), ("input_partitions", C.c_uint32),
                ("total_partitions", C.c_uint32), ("group_pitch", C.c_uint32),
                ("group_step", C.c_uint32), ("gq_pitch", C.c_uint64), ("bundles", C.c_uint64),
                ("bytes", C.c_uint64 * L_COUNT)]


class PopDesc(C.Structure):
    _fields_ = [("model", C.c_int32), ("flags", C.c_uint32), ("begin", C.c_int64), ("end", C.c_int64),
                ("p", C.c_float * 12), ("pn_host", C.c_void_p), ("seed", C.c_uint64)]


class NetDesc(C.Structure):
    _fields_ = [("n_neurons", C.c_int64), ("n_sources", C.c_int64), ("max_delay", C.c_int32),
                ("n_pops", C.c_int32), ("pops", C.c_void_p), ("n_synapses", C.c_uint64),
                ("row_ptr_host", C.c_void_p), ("tgt_host", C.c_void_p), ("w_host", C.c_void_p),
                ("state_host", C.c_void_p * 4), ("acc_mode", C.c_uint32), ("graph_chunk", C.c_uint32),
                ("raster_capacity", C.c_int64), ("group_host", C.c_void_p), ("n_groups", C.c_int32)]


class GenBlock(C.Structure):
    _fields_ = [("src_begin", C.c_int64), ("src_count", C.c_int64), ("tgt_begin", C.c_int64),
                ("tgt_count", C.c_int64), ("fanout", C.c_int32), ("exclude_self", C.c_int32),
                ("w_lo", C.c_float), ("w_hi", C.c_float), ("w_sign", C.c_float),
                ("d_lo", C.c_int32), ("d_hi", C.c_int32), ("stream", C.c_uint32), ("syn_offset", C.c_uint64)]


class NetStats(C.Structure):
    _fields_ = [("steps_done", C.c_int64), ("events", C.c_uint64), ("spikes", C.c_uint64),
                ("graph_launches", C.c_uint64), ("kernel_launches", C.c_uint64)]


class Peaks(C.Structure):
    _fields_ = [("l2_copy_gbs", C.c_double), ("l2_copy_bytes", C.c_int64), ("red_per_s", C.c_double),
                ("red_targets", C.c_int64)]


_lib = None

# name -> (restype, argtypes); every entry point declared in include/szsnn_cuda.h
_P, _I, _U32, _U64, _I64, _D = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_int64, C.c_double
_UPDATE_ARGS = [_P, _U64, _U32, _P, _P, _P, _U32, _P, _P, _U32, _P, _P, _P, _P, _U32, _U32]
SIGNATURES = {
    "szsnn_ctx_create": (_I, [_I, _P, C.POINTER(C.c_void_p)]),
    "szsnn_ctx_destroy": (_I, [_P]),
    "szsnn_last_error": (C.c_char_p, [_P]),
    "szsnn_set_stream": (_I, [_P, _P]),
    "szsnn_get_stream": (_P, [_P]),
    "szsnn_alloc": (_I, [_P, C.c_size_t, C.POINTER(C.c_void_p)]),
    "szsnn_free": (_I, [_P, _P]),
    "szsnn_h2d": (_I, [_P, _P, _P, C.c_size_t]),
    "szsnn_d2h": (_I, [_P, _P, _P, C.c_size_t]),
    "szsnn_memset": (_I, [_P, _P, _I, C.c_size_t]),
    "szsnn_sync": (_I, [_P]),
    "szsnn_device_error": (_I, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "szsnn_clear_device_error": (_I, [_P]),
    "szsnn_set_option": (_I, [_P, _I, _I64]),
    "szsnn_update_if_curr_exp": (_I, _UPDATE_ARGS),
    "szsnn_update_izhikevich": (_I, _UPDATE_ARGS),
    "szsnn_update_const_rate": (_I, _UPDATE_ARGS),
    "szsnn_gather": (_I, [_P, _U64, _U32, _P, _P, _U64, _P, _P, _P, _P]),
    "szsnn_scatter": (_I, [_P, _U64, _U32, _P, _P, _U32, _U32, _P, _P, _U64, _P, _P, _P, _P, _P]),
    "szsnn_layout_build": (_I, [_P, _P, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "szsnn_layout_info_get": (_I, [_P, _P]),
    "szsnn_layout_array": (_I, [_P, _I, _P, C.c_size_t]),
    "szsnn_layout_free": (_I, [_P]),
    "szsnn_net_create": (_I, [_P, _P, C.POINTER(C.c_void_p)]),
    "szsnn_net_generate": (_I, [_P, _P, _I, _U64]),
    "szsnn_net_destroy": (_I, [_P]),
    "szsnn_net_step": (_I, [_P, _P, _P, _P]),
    "szsnn_net_inject_spikes": (_I, [_P, _P]),
    "szsnn_net_set_owned": (_I, [_P, _I64, _I64, _I64, _I64]),
    "szsnn_net_run": (_I, [_P, _I64, _P, _P]),
    "szsnn_net_run_device": (_I, [_P, _I64, _P, _P, _P]),
    "szsnn_net_stats_get": (_I, [_P, _P]),
    "szsnn_net_group_spikes": (_I, [_P, _P, _I]),
    "szsnn_net_get_state": (_I, [_P, _I, _P]),
    "szsnn_net_set_state": (_I, [_P, _I, _P]),
    "szsnn_net_set_monitor": (_I, [_P, _P, C.c_int32, _U32, _I64]),
    "szsnn_net_monitor_read": (_I, [_P, _P, _I64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "szsnn_net_checkpoint_size": (_I, [_P, C.POINTER(C.c_uint64)]),
    "szsnn_net_checkpoint": (_I, [_P, _P, _U64]),
    "szsnn_net_restore": (_I, [_P, _P, _U64]),
    "szsnn_net_get_synapses": (_I, [_P, _P, _P, _P]),
    "szsnn_net_check_finite": (_I, [_P, C.POINTER(C.c_int)]),
    "szsnn_net_last_inputs": (_I, [_P, _P, _P]),
    "szsnn_net_profile": (_I, [_P, _I64, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "szsnn_net_profile_step": (_I, [_P, _I64, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "szsnn_net_timing": (_I, [_P, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "szsnn_net_set_tuning": (_I, [_P, _I, _I, _I, _I]),
    "szsnn_net_set_update_tiles": (_I, [_P, _I, _I]),
    "szsnn_net_set_resident": (_I, [_P, _I, _I, _I]),
    "szsnn_net_set_update_units": (_I, [_P, _I]),
    "szsnn_net_set_overlap": (_I, [_P, C.c_int]),
    "szsnn_step_static": (_I, [_P, C.c_char_p, C.c_size_t]),
    "szsnn_probe_peaks": (_I, [_P, _I64, _P]),
    "szsnn_bptt_workspace_bytes": (_I, [_P, C.POINTER(C.c_uint64)]),
    "szsnn_bptt_forward": (_I, [_P, C.c_char_p, C.c_size_t]),
    "szsnn_bptt_backward": (_I, [_P, C.c_char_p, C.c_size_t]),
}


def lib() -> C.CDLL:
    """Load the CUDA library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m szsnn_b200.build` "
                "(the sm_100a CUDA library is required; there is no CPU fallback)")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            if hasattr(h, name):
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
        _lib = h
    return _lib


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != SZSNN_OK:
        msg = what
        if ctx is not None:
            m = lib().szsnn_last_error(ctx)
            msg = f"{what}: {m.decode() if m else ''}"
        raise SzsnnError(rc, msg)
