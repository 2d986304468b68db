"""FP64 CPU reference of the differentiable IF_curr_exp RNN -- TEST INFRASTRUCTURE ONLY.

The checker for szsnn_b200.pyszsnn (forward spikes, readout, and the BPTT
gradient of the hand-written adjoint).  No reference counterpart exists for
differentiation; the forward rule is the reference's IF_curr_exp update
(szsnn1.1/src/cl/IF_curr_exp_update_kernel.cl:230-287, dt folded to 1,
tau_refrac 0 so the refractory branch never applies), the exc / inh channel of
a weight is its sign (cl/gather_kernel.cl:172-178, w == 0 contributes
nothing), input spikes are integrated in the step they occur and recurrent
spikes one step later.

Model, per trial b, neuron i, step t:
  a_t = sum_j x_t[j] Win+[j,i] + sum_j s_{t-1}[j] Wrec+[j,i]    (c_t: negative parts)
  Ie_t = de Ie_{t-1} + a_t ;  Ii_t = di Ii_{t-1} + c_t          (de = 1 - 1/tau_syn_E)
  u_t  = v_{t-1} + (Ie_t + Ii_t + i_offset)/cm + (v_rest - v_{t-1})/tau_m
  s_t  = H(u_t - v_thresh) ;  v_t = u_t (1 - s_t) + v_reset s_t
  y_t  = alpha y_{t-1} + sum_i s_t[i] Wout[i,k] ;  ymax = max_t y_t (first argmax)
  vsum = sum_t v_t
Gradient: exact, except dH/du, replaced by the fast sigmoid surrogate
1/(1 + beta|u - v_thresh|)^2 (beta <= 0: dH/du = 0, the exact derivative
wherever no spike flips).  Spikes are those of the forward pass.
"""
from __future__ import annotations

import numpy as np


def _split(W):
    return np.where(W > 0, W, 0.0), np.where(W < 0, W, 0.0)


def forward(p: dict, W_in, W_rec, W_out, x, v0, spikes=None):
    """x: [T,B,M] {0,1}; W_rec dense [N,N] (row = presynaptic).  If `spikes`
    [T,B,N] is given the spike trains are imposed (teacher forcing) and only
    the membrane is recomputed.  Returns dict of trajectories in fp64."""
    T, B, M = x.shape
    N = W_in.shape[1]
    K = W_out.shape[1]
    Wip, Win_ = _split(W_in.astype(np.float64))
    Wrp, Wrn = _split(W_rec.astype(np.float64))
    de = 1.0 - 1.0 / p["tau_syn_E"]
    di = 1.0 - 1.0 / p["tau_syn_I"]
    Ie = np.zeros((B, N))
    Ii = np.zeros((B, N))
    v = v0.astype(np.float64).copy()
    s_prev = np.zeros((B, N))
    y = np.zeros((B, K))
    U = np.zeros((T, B, N))
    S = np.zeros((T, B, N))
    Y = np.zeros((T, B, K))
    vsum = np.zeros((B, N))
    for t in range(T):
        xt = x[t].astype(np.float64)
        a = xt @ Wip + s_prev @ Wrp
        c = xt @ Win_ + s_prev @ Wrn
        Ie = de * Ie + a
        Ii = di * Ii + c
        I = Ie + Ii + p["i_offset"]
        u = v + I / p["cm"] + (p["v_rest"] - v) / p["tau_m"]
        s = (u >= p["v_thresh"]).astype(np.float64) if spikes is None else spikes[t].astype(np.float64)
        v = u * (1 - s) + p["v_reset"] * s
        y = p["alpha"] * y + s @ W_out.astype(np.float64)
        U[t], S[t], Y[t] = u, s, y
        vsum += v
        s_prev = s
    tmax = np.argmax(Y, axis=0)                      # [B,K], first maximum
    ymax = np.take_along_axis(Y, tmax[None], 0)[0]
    return dict(U=U, S=S, Y=Y, ymax=ymax, tmax=tmax, vsum=vsum)


def surrogate(x, beta):
    if beta <= 0:
        return np.zeros_like(x)
    return 1.0 / (1.0 + beta * np.abs(x)) ** 2


def backward(p: dict, W_in, W_rec, W_out, x, fw: dict, g_ymax, g_vsum, beta: float):
    """Adjoint of `forward` (given its trajectories).  Returns (dW_in, dW_rec, dW_out)
    with dW_rec nonzero only where W_rec != 0."""
    U, S, tmax = fw["U"], fw["S"], fw["tmax"]
    T, B, N = U.shape
    K = W_out.shape[1]
    Wip, Win_ = _split(W_in.astype(np.float64))
    Wrp, Wrn = _split(W_rec.astype(np.float64))
    Wo = W_out.astype(np.float64)
    de = 1.0 - 1.0 / p["tau_syn_E"]
    di = 1.0 - 1.0 / p["tau_syn_I"]
    km = 1.0 - 1.0 / p["tau_m"]
    lam_u_next = np.zeros((B, N))
    lam_e_next = np.zeros((B, N))   # dL/dIe_{t+1} (total), also dL/da_{t+1}
    lam_i_next = np.zeros((B, N))
    lam_y = np.zeros((B, K))
    dWin = np.zeros_like(Wip)
    dWrec = np.zeros_like(Wrp)
    dWout = np.zeros_like(Wo)
    g_vsum = np.zeros((B, N)) if g_vsum is None else g_vsum.astype(np.float64)
    g_ymax = np.zeros((B, K)) if g_ymax is None else g_ymax.astype(np.float64)
    pos_in, neg_in = W_in > 0, W_in < 0
    pos_rec, neg_rec = W_rec > 0, W_rec < 0
    for t in range(T - 1, -1, -1):
        lam_y = p["alpha"] * lam_y + np.where(tmax == t, g_ymax, 0.0)
        u, s = U[t], S[t]
        G_v = g_vsum + km * lam_u_next
        G_s = lam_y @ Wo.T + lam_e_next @ Wrp.T + lam_i_next @ Wrn.T + G_v * (p["v_reset"] - u)
        lam_u = G_v * (1 - s) + G_s * surrogate(u - p["v_thresh"], beta)
        lam_e = lam_u / p["cm"] + de * lam_e_next
        lam_i = lam_u / p["cm"] + di * lam_i_next
        dWout += s.T @ lam_y
        xt = x[t].astype(np.float64)
        dWin += np.where(pos_in, xt.T @ lam_e, 0.0) + np.where(neg_in, xt.T @ lam_i, 0.0)
        if t >= 1:
            sp = S[t - 1]
            dWrec += np.where(pos_rec, sp.T @ lam_e, 0.0) + np.where(neg_rec, sp.T @ lam_i, 0.0)
        lam_u_next, lam_e_next, lam_i_next = lam_u, lam_e, lam_i
    return dWin, dWrec, dWout


def loss_ce(ymax, labels):
    z = ymax - ymax.max(axis=1, keepdims=True)
    lse = np.log(np.exp(z).sum(axis=1))
    return float(np.mean(lse - z[np.arange(len(labels)), labels]))


def loss_ce_grad(ymax, labels):
    z = ymax - ymax.max(axis=1, keepdims=True)
    sm = np.exp(z) / np.exp(z).sum(axis=1, keepdims=True)
    sm[np.arange(len(labels)), labels] -= 1.0
    return sm / len(labels)
