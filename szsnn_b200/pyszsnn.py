"""pyszsnn: a differentiable recurrent IF_curr_exp layer for PyTorch.

`LIFCurrExpFunction.apply(w_in, rec_val, w_out, x_bits, v0, net)` runs the
forward simulation and, on `.backward()`, the hand-written BPTT adjoint of
libszsnn_cuda.so (szsnn_bptt_forward / szsnn_bptt_backward).  Torch tensors
only provide device memory and the stream; the work is in the sm_100a kernels.

Model (no reference counterpart for training; the neuron rule is the
reference's IF_curr_exp update, IF_curr_exp_update_kernel.cl:230-287, with
dt folded to 1 step and tau_refrac 0; a weight's sign picks the exc / inh
synaptic channel, gather_kernel.cl:172-178):
  inputs x_t (spikes of M Poisson sources) are integrated in their own step,
  recurrent spikes one step later through the sparse CSR weights `rec_val`,
  readouts y_t = alpha y_{t-1} + w_out^T s_t; outputs ymax = max_t y_t and
  vsum = sum_t v_t.  Gradients are exact except dH/du, replaced by the fast
  sigmoid 1/(1 + beta|u - v_thresh|)^2; forward spikes are kept, and u is
  recomputed from checkpoints every `checkpoint_every` steps, or read from
  the trajectory the forward kept (store_trajectory; by default whenever it
  fits the budget).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L


class BpttDesc(C.Structure):
    _fields_ = [("B", C.c_int32), ("N", C.c_int32), ("M", C.c_int32), ("K", C.c_int32), ("T", C.c_int32),
                ("checkpoint_every", C.c_int32),
                ("v_rest", C.c_float), ("cm", C.c_float), ("tau_m", C.c_float), ("tau_refrac", C.c_float),
                ("tau_syn_E", C.c_float), ("tau_syn_I", C.c_float), ("i_offset", C.c_float), ("v_reset", C.c_float),
                ("v_thresh", C.c_float), ("alpha", C.c_float), ("beta", C.c_float), ("nnz", C.c_int64),
                ("w_in", C.c_void_p), ("rec_row_ptr", C.c_void_p), ("rec_col", C.c_void_p), ("rec_val", C.c_void_p),
                ("w_out", C.c_void_p), ("x_bits", C.c_void_p), ("v0", C.c_void_p), ("spikes", C.c_void_p),
                ("ckpt", C.c_void_p), ("ymax", C.c_void_p), ("tmax", C.c_void_p), ("vsum", C.c_void_p),
                ("u_trace", C.c_void_p), ("g_ymax", C.c_void_p), ("g_vsum", C.c_void_p), ("dw_in", C.c_void_p), ("dw_rec", C.c_void_p),
                ("dw_out", C.c_void_p), ("phase_ms", C.c_void_p), ("workspace", C.c_void_p),
                ("stream", C.c_void_p)]

BACKWARD_PHASES = ("recompute", "recurrent term + dWrec", "adjoint", "dWin")


@dataclass
class LIFCurrExpRNN:
    """Structure and fixed parameters of the layer (weights are the autograd inputs)."""
    n_neurons: int
    n_inputs: int
    n_readouts: int
    rec_row_ptr: torch.Tensor          # int64 [N+1], CSR rows = presynaptic neuron
    rec_col: torch.Tensor              # int32 [nnz]
    params: dict = field(default_factory=lambda: dict(v_rest=0.0, cm=1.0, tau_m=20.0, tau_refrac=0.0,
                                                      tau_syn_E=5.0, tau_syn_I=10.0, i_offset=0.0, v_reset=0.0,
                                                      v_thresh=1.0))
    alpha: float = 0.95
    beta: float = 10.0
    checkpoint_every: int = 50
    # keep the membrane trajectory u [T,B,N] from the forward for the backward
    # (no recompute): True, False, or None = when it takes at most
    # trajectory_budget bytes and a quarter of the device's free memory
    store_trajectory: bool | None = None
    trajectory_budget: int = 16 << 30
    phase_ms: np.ndarray | None = field(default=None, repr=False)  # float64 [4]: backward adds its device ms
                                                                    # per phase (BACKWARD_PHASES) when set

    @property
    def nnz(self) -> int:
        return int(self.rec_col.numel())

    def stores_trajectory(self, T: int, B: int, device) -> bool:
        if self.store_trajectory is not None:
            return bool(self.store_trajectory)
        nbytes = 4 * T * B * self.n_neurons
        free = torch.cuda.mem_get_info(device)[0]
        return nbytes <= self.trajectory_budget and 4 * nbytes <= free


def _ptr(t):
    return None if t is None else t.data_ptr()


def _desc(net: LIFCurrExpRNN, B: int, T: int, tensors: dict) -> BpttDesc:
    d = BpttDesc()
    d.B, d.N, d.M, d.K, d.T, d.checkpoint_every = B, net.n_neurons, net.n_inputs, net.n_readouts, T, \
        net.checkpoint_every
    p = net.params
    d.v_rest, d.cm, d.tau_m, d.tau_refrac = p["v_rest"], p["cm"], p["tau_m"], p["tau_refrac"]
    d.tau_syn_E, d.tau_syn_I, d.i_offset = p["tau_syn_E"], p["tau_syn_I"], p["i_offset"]
    d.v_reset, d.v_thresh = p["v_reset"], p["v_thresh"]
    d.alpha, d.beta, d.nnz = net.alpha, net.beta, net.nnz
    d.rec_row_ptr, d.rec_col = _ptr(net.rec_row_ptr), _ptr(net.rec_col)
    for k, v in tensors.items():
        setattr(d, k, _ptr(v))
    d.stream = torch.cuda.current_stream().cuda_stream
    return d


def _check(rc: int, msg: C.Array) -> None:
    if rc:
        raise L.SzsnnError(rc, msg.value.decode())


def _forward(net: LIFCurrExpRNN, w_in, rec_val, w_out, x_bits, v0, trace_u: bool = False):
    T, B = int(x_bits.shape[0]), int(v0.shape[0])
    N, K = net.n_neurons, net.n_readouts
    dev = v0.device
    nck = (T + net.checkpoint_every - 1) // net.checkpoint_every
    out = dict(spikes=torch.empty((T, B, (N + 31) // 32), dtype=torch.int32, device=dev),
               ckpt=torch.empty((nck, 3, B, N), dtype=torch.float32, device=dev),
               ymax=torch.empty((B, K), dtype=torch.float32, device=dev),
               tmax=torch.empty((B, K), dtype=torch.int32, device=dev),
               vsum=torch.empty((B, N), dtype=torch.float32, device=dev))
    if trace_u:
        out["u_trace"] = torch.empty((T, B, N), dtype=torch.float32, device=dev)
    d = _desc(net, B, T, dict(w_in=w_in, rec_val=rec_val, w_out=w_out, x_bits=x_bits, v0=v0, **out))
    nbytes = C.c_uint64()
    L.check(L.lib().szsnn_bptt_workspace_bytes(C.byref(d), C.byref(nbytes)), None, "bptt workspace")
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=dev)
    d.workspace = ws.data_ptr()
    msg = C.create_string_buffer(256)
    _check(L.lib().szsnn_bptt_forward(C.byref(d), msg, 256), msg)
    out["workspace"] = ws
    return out


class LIFCurrExpFunction(torch.autograd.Function):
    """(w_in [M,N], rec_val [nnz], w_out [N,K], x_bits [T,B,ceil(M/32)] int32,
    v0 [B,N], net) -> (ymax [B,K], vsum [B,N])."""

    @staticmethod
    def forward(ctx, w_in, rec_val, w_out, x_bits, v0, net):
        tensors = [t.contiguous() for t in (w_in, rec_val, w_out, x_bits, v0)]
        store = net.stores_trajectory(int(x_bits.shape[0]), int(v0.shape[0]), v0.device)
        out = _forward(net, *tensors, trace_u=store)
        ctx.net = net
        ctx.ws = out["workspace"]
        ctx.u_trace = out.get("u_trace")
        ctx.save_for_backward(*tensors, out["spikes"], out["ckpt"], out["tmax"])
        return out["ymax"], out["vsum"]

    @staticmethod
    def backward(ctx, g_ymax, g_vsum):
        w_in, rec_val, w_out, x_bits, v0, spikes, ckpt, tmax = ctx.saved_tensors
        net = ctx.net
        T, B = int(x_bits.shape[0]), int(v0.shape[0])
        dw_in = torch.empty_like(w_in)
        dw_rec = torch.empty_like(rec_val)
        dw_out = torch.empty_like(w_out)
        g_ymax = None if g_ymax is None else g_ymax.contiguous().float()
        g_vsum = None if g_vsum is None else g_vsum.contiguous().float()
        d = _desc(net, B, T, dict(w_in=w_in, rec_val=rec_val, w_out=w_out, x_bits=x_bits, v0=v0, spikes=spikes,
                                  ckpt=ckpt, tmax=tmax, g_ymax=g_ymax, g_vsum=g_vsum, dw_in=dw_in, dw_rec=dw_rec,
                                  dw_out=dw_out, workspace=ctx.ws, u_trace=ctx.u_trace))
        if net.phase_ms is not None:
            if net.phase_ms.dtype != np.float64 or net.phase_ms.shape != (4,) or not net.phase_ms.flags.c_contiguous:
                raise ValueError("phase_ms must be a contiguous float64 array of 4")
            d.phase_ms = net.phase_ms.ctypes.data
        msg = C.create_string_buffer(256)
        _check(L.lib().szsnn_bptt_backward(C.byref(d), msg, 256), msg)
        return dw_in, dw_rec, dw_out, None, None, None


def simulate(net: LIFCurrExpRNN, w_in, rec_val, w_out, x_bits, v0, trace_u: bool = False) -> dict:
    """Forward only, returning spikes [T,B,ceil(N/32)] int32 words, ymax, tmax,
    vsum and, with trace_u, the pre-reset membrane u [T,B,N]."""
    with torch.no_grad():
        out = _forward(net, w_in.contiguous(), rec_val.contiguous(), w_out.contiguous(), x_bits.contiguous(),
                       v0.contiguous(), trace_u)
    return out


def poisson_bits(T: int, B: int, rates_hz: torch.Tensor, dt_ms: float = 1.0, seed: int = 0) -> torch.Tensor:
    """Input spike words [T, B, ceil(M/32)] (int32) from independent Bernoulli
    draws with p = rate * dt per step."""
    M = int(rates_hz.numel())
    g = torch.Generator(device=rates_hz.device).manual_seed(seed)
    p = (rates_hz.float() * dt_ms * 1e-3).clamp(0, 1)
    x = torch.rand((T, B, M), generator=g, device=rates_hz.device) < p
    return pack_bits(x)


def pack_bits(x: torch.Tensor) -> torch.Tensor:
    """[..., M] bool -> [..., ceil(M/32)] int32 words, bit i of word w = element 32w + i."""
    M = x.shape[-1]
    W = (M + 31) // 32
    pad = torch.zeros(*x.shape[:-1], W * 32, dtype=torch.int64, device=x.device)
    pad[..., :M] = x.to(torch.int64)
    pad = pad.view(*x.shape[:-1], W, 32)
    shifts = torch.arange(32, device=x.device, dtype=torch.int64)
    words = (pad << shifts).sum(-1)
    return (words - (words >= 2 ** 31).to(torch.int64) * 2 ** 32).to(torch.int32)


def unpack_bits(words: torch.Tensor, n: int) -> torch.Tensor:
    w = words.to(torch.int64) & 0xFFFFFFFF
    shifts = torch.arange(32, device=words.device, dtype=torch.int64)
    bits = (w.unsqueeze(-1) >> shifts) & 1
    return bits.reshape(*words.shape[:-1], -1)[..., :n].bool()


def random_recurrent(n: int, density: float, seed: int, device) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """CSR (row_ptr int64, col int32, val fp32) of a random sparse n x n matrix,
    density `density`, no self connections, values N(0, 1/sqrt(fan-in))."""
    rng = np.random.default_rng(seed)
    fan = max(int(round(density * n)), 1)
    cols = np.empty((n, fan), np.int64)
    for j in range(n):
        c = rng.choice(n - 1, fan, replace=False)
        c[c >= j] += 1
        cols[j] = np.sort(c)
    vals = rng.normal(0.0, 1.0 / np.sqrt(fan), (n, fan)).astype(np.float32)
    row_ptr = np.arange(n + 1, dtype=np.int64) * fan
    return (torch.from_numpy(row_ptr).to(device), torch.from_numpy(cols.reshape(-1).astype(np.int32)).to(device),
            torch.from_numpy(vals.reshape(-1)).to(device))
