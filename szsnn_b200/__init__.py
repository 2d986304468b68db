"""szsnn_b200 -- B200-native (sm_100a) clock-driven simulation step of SZSNN.

Host side of the C ABI in include/szsnn_cuda.h (libszsnn_cuda.so):
  Context        szsnn::Context seam: device, stream, buffers (Context.hpp:77-303)
  RefSimulation  szsnn::Simulation<float> on the reference buffer layout with
                 the drop-in gather / update / scatter kernels (Simulation.ipp)
  Network        native path: delay-bucketed CSR, device spike ring, Poisson
                 sources, IF_cond_exp, CUDA-graph step loop
"""
from . import _lib
from ._lib import (ACC_FIXED, ACC_FLOAT, CONST_RATE, IF_COND_EXP, IF_CURR_EXP, IZHIKEVICH, POISSON,
                   POP_IZH_HALF_STEPS, SzsnnError)
from .context import Context, DeviceBuffer
from .models import fold_dt, if_params, izh_params
from .network import GenBlock, Network, Pop, csr_from_synapses, ids_to_words, words_to_ids
from .refsim import CudaRefBackend, RefSimulation, build_layout

__all__ = [
    "ACC_FIXED", "ACC_FLOAT", "CONST_RATE", "IF_COND_EXP", "IF_CURR_EXP", "IZHIKEVICH", "POISSON",
    "POP_IZH_HALF_STEPS", "SzsnnError", "Context", "DeviceBuffer", "fold_dt", "if_params", "izh_params",
    "GenBlock", "Network", "Pop", "csr_from_synapses", "ids_to_words", "words_to_ids", "CudaRefBackend",
    "RefSimulation", "build_layout",
]
