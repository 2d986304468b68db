"""Synthetic network builders for the benchmark configurations (seeded).

  izh1000      Izhikevich pulse-coupled network: 1000 neurons (800 RS with
               a=0.02, b=0.2, c=-65+15r^2, d=8-6r^2; 200 FS with a=0.02+0.08r,
               b=0.25-0.05r, c=-65, d=2; r ~ U(0,1)), 100 distinct non-self
               targets per neuron, weights +6 / -5, excitatory delays
               U{1..20} ms, inhibitory 1 ms; thalamic input N(0,1)*5 / *2 per
               1 ms step (`thalamic`)
  if4000       IF_curr_exp balanced network: 3200 / 800 neurons, connection
               probability 0.02, tau_m 20 ms, cm 0.2 nF, v_rest -60,
               v_thresh -50, v_reset -60 mV, tau_refrac 5 ms, tau_syn_E 5,
               tau_syn_I 10 ms, w 0.25 / -2.25 nA, delays U{1..100} steps at
               dt 0.1 ms, 1000 Poisson sources at 10 Hz with fan-out
               probability 0.02; `clip_delay=64` gives the variant the
               reference layout can hold (delays <= 64)
  cond_config  IF_cond_exp network of n neurons (80/20), `fanout` random
               targets per neuron without self-loops, exc weights U(0,4) nS,
               inh U(0,51) nS, delays U{1..64} steps, n/10 Poisson sources at
               5 Hz with 100 targets each, dt 0.1 ms (1M x 1000 is the large
               configuration)

Stored delays are the user delay + 1 (NetworkGraph.ipp:431): a spike at step
t over a synapse of user delay d is integrated by the update of step t+d+1.
Parameters the configurations leave open are stated where they are set.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .models import fold_dt, if_params
from .network import GenBlock, Pop, csr_from_synapses

DT_COND_MS = 0.1


def izh_network(n=1000, fanout=100, seed=3, half_steps=False, max_delay=20):
    """The Izhikevich network as synapse lists and per-neuron parameters."""
    rng = np.random.default_rng(seed)
    ne = int(0.8 * n)
    re = rng.uniform(0, 1, ne).astype(np.float32)
    ri = rng.uniform(0, 1, n - ne).astype(np.float32)
    a = np.concatenate([np.full(ne, 0.02), 0.02 + 0.08 * ri]).astype(np.float32)
    b = np.concatenate([np.full(ne, 0.2), 0.25 - 0.05 * ri]).astype(np.float32)
    c = np.concatenate([-65 + 15 * re ** 2, np.full(n - ne, -65.0)]).astype(np.float32)
    d = np.concatenate([8 - 6 * re ** 2, np.full(n - ne, 2.0)]).astype(np.float32)
    src, tgt = [], []
    for s in range(n):
        cand = rng.choice(n - 1, fanout, replace=False)
        cand[cand >= s] += 1
        src.append(np.full(fanout, s))
        tgt.append(cand)
    src = np.concatenate(src)
    tgt = np.concatenate(tgt)
    exc = src < ne
    w = np.where(exc, 6.0, -5.0).astype(np.float32)
    d1 = np.where(exc, rng.integers(1, max_delay + 1, len(src)), 1).astype(np.uint32)
    v0 = np.full(n, -65.0, np.float32)
    u0 = (b * v0).astype(np.float32)
    return dict(n=n, src=src, tgt=tgt, w=w, d1=d1, a=a, b=b, c=c, d=d, v0=v0, u0=u0, ne=ne, D=max_delay)


def izh_native(net: dict):
    """(pops, csr, state) of izh_network's output for the native path."""
    n = net["n"]
    csr = csr_from_synapses(n, net["D"], net["src"], net["tgt"], net["w"], net["d1"])
    pn = np.zeros((12, n), np.float32)
    pn[0], pn[1], pn[2], pn[3] = net["a"], net["b"], net["c"], net["d"]
    pops = [Pop(L.IZHIKEVICH, 0, n, np.zeros(12, np.float32), per_unit=pn)]
    return pops, csr, [net["v0"], net["u0"], None, None]


def thalamic(n, ne, steps, seed=7):
    """N(0,1)*5 to excitatory, *2 to inhibitory neurons, per step: [steps, n] fp32."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((steps, n)).astype(np.float32)
    x[:, :ne] *= np.float32(5.0)
    x[:, ne:] *= np.float32(2.0)
    return x


def if4000_params():
    return fold_dt(if_params(v_rest=-60, cm=0.2, tau_m=20, tau_refrac=5, tau_syn_E=5, tau_syn_I=10,
                             v_reset=-60, v_thresh=-50), 0.1)


def if4000(seed=11, clip_delay=None):
    """The balanced IF_curr_exp network.  Returns a dict with the synapse
    lists (src, tgt, w, d1 over neurons then sources), the native form
    (pops, csr, state, D) and the Poisson rate per step (p_step).  With
    `clip_delay` the user delays are drawn from U{1..clip_delay} instead of
    U{1..100}."""
    rng = np.random.default_rng(seed)
    n, ne, p_src = 4000, 3200, 1000
    d_hi = 100 if clip_delay is None else int(clip_delay)
    src, tgt, w, d1 = [], [], [], []
    for s in range(n + p_src):
        k = rng.binomial(n, 0.02)
        t = rng.choice(n, k, replace=False)
        src.append(np.full(k, s))
        tgt.append(t)
        if s < n:
            w.append(np.full(k, 0.25 if s < ne else -2.25, np.float32))
            d1.append(rng.integers(1, d_hi + 1, k) + 1)  # stored = user delay + 1
        else:
            w.append(np.full(k, 0.25, np.float32))
            d1.append(np.full(k, 1))
    src, tgt, w, d1 = (np.concatenate(x) for x in (src, tgt, w, d1))
    D = d_hi + 1
    p_step = np.float32(10.0 * 0.1e-3)
    pops = [Pop(L.IF_CURR_EXP, 0, n, if4000_params()),
            Pop(L.POISSON, n, n + p_src, np.array([p_step], np.float32), seed=77)]
    v0 = np.concatenate([rng.uniform(-60, -50, n), np.zeros(p_src)]).astype(np.float32)
    fr = np.concatenate([np.full(n, 1e4), np.zeros(p_src)]).astype(np.float32)
    csr = csr_from_synapses(n + p_src, D, src, tgt, w, d1.astype(np.uint32))
    return dict(n=n, ne=ne, p=p_src, D=D, src=src, tgt=tgt, w=w, d1=d1.astype(np.uint32), pops=pops, csr=csr,
                state=[v0, None, None, fr], p_step=float(p_step))


def cond_config(n: int, fanout: int):
    """Generator blocks, populations and sizes of the IF_cond_exp network:
    (n, p, D, blocks, pops).  Parameters the configuration leaves open come
    from the 4000-neuron IF_curr_exp network (tau_m 20 ms, cm 0.2 nF, v_rest
    -60, v_thresh -50, v_reset -60 mV, tau_refrac 5 ms); Poisson synapses
    U(0,100) nS with delay 1 step; conductances in uS, dt folded in."""
    p = n // 10
    D = 64
    ne = int(0.8 * n)
    blocks = [GenBlock(0, ne, 0, n, fanout, 0.0, 0.004, 1.0, 1, D, True, 1),
              GenBlock(ne, n - ne, 0, n, fanout, 0.0, 0.051, -1.0, 1, D, True, 2),
              GenBlock(n, p, 0, n, 100, 0.0, 0.1, 1.0, 1, 1, False, 3)]
    pv = fold_dt(if_params(v_rest=-60, cm=0.2, tau_m=20, tau_refrac=5, tau_syn_E=5, tau_syn_I=10,
                           v_reset=-60, v_thresh=-50, e_rev_E=0.0, e_rev_I=-80.0), DT_COND_MS)
    pops = [Pop(L.IF_COND_EXP, 0, n, pv),
            Pop(L.POISSON, n, n + p, np.array([5.0 * DT_COND_MS * 1e-3], np.float32), seed=20240)]
    return n, p, D, blocks, pops


def init_state(n, p, seed):
    """v(0) ~ U(-60,-50) mV, no refractoriness; sources carry no state."""
    rng = np.random.default_rng(seed)
    v0 = np.concatenate([rng.uniform(-60, -50, n), np.zeros(p)]).astype(np.float32)
    fired = np.concatenate([np.full(n, 1e4), np.zeros(p)]).astype(np.float32)
    return [v0, None, None, fired]
