"""Shared network builders for the parity tests (seeded, small)."""
from __future__ import annotations

import numpy as np

import szsnn_b200 as sz


def if_network(n=300, n_syn=6000, max_delay=64, dyadic=True, seed=1, n_exc=None):
    """Random IF_curr_exp network; dyadic weights make every fp32 sum exact."""
    rng = np.random.default_rng(seed)
    n_exc = int(0.8 * n) if n_exc is None else n_exc
    src = rng.integers(0, n, n_syn)
    tgt = rng.integers(0, n, n_syn)
    exc = src < n_exc
    if dyadic:
        w = np.where(exc, 0.25 * rng.integers(1, 5, n_syn), -0.5 * rng.integers(1, 3, n_syn))
    else:
        w = np.where(exc, rng.uniform(0.1, 1.0, n_syn), -rng.uniform(0.2, 1.2, n_syn))
    w = w.astype(np.float32)
    d1 = rng.integers(1, max_delay + 1, n_syn).astype(np.uint32)
    pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=2, tau_syn_E=5, tau_syn_I=10, v_reset=-60,
                      v_thresh=-50)
    v0 = rng.uniform(-60, -50, n).astype(np.float32)
    return dict(n=n, src=src, tgt=tgt, w=w, d1=d1, pv=pv, v0=v0, D=max_delay)


def izh_network(n=1000, fanout=100, seed=3, dyadic=True, half_steps=False, max_delay=20):
    """Izhikevich pulse-coupled network shaped like the 1000-neuron benchmark
    (800 RS / 200 FS, 100 distinct non-self targets, exc delays U{1..20},
    inh delay 1), with parameters drawn from r ~ U(0,1)."""
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
    w = np.where(exc, 6.0, -5.0).astype(np.float32) if dyadic else np.where(exc, 6.0, -5.0).astype(np.float32)
    d1 = np.where(exc, rng.integers(1, max_delay + 1, len(src)), 1).astype(np.uint32)
    v0 = np.full(n, -65.0, np.float32)
    u0 = (b * v0).astype(np.float32)
    return dict(n=n, src=src, tgt=tgt, w=w, d1=d1, a=a, b=b, c=c, d=d, v0=v0, u0=u0, ne=ne, D=max_delay)


def thalamic(n, ne, steps, seed=7):
    """N(0,1)*5 to excitatory, *2 to inhibitory neurons, per step."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((steps, n)).astype(np.float32)
    x[:, :ne] *= np.float32(5.0)
    x[:, ne:] *= np.float32(2.0)
    return x


def forced_schedule(n, steps, every=7, first=3):
    return [list(range(0, n, every)) if t < first else None for t in range(steps)]


def forced_words(sched, n_units):
    W = (n_units + 31) // 32
    fw = np.zeros((len(sched), W), np.uint32)
    for t, ids in enumerate(sched):
        if ids is not None and len(ids):
            fw[t] = sz.ids_to_words(ids, n_units)
    return fw
