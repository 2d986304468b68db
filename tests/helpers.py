"""Shared network builders for the parity tests (seeded, small)."""
from __future__ import annotations

import numpy as np

import szsnn_b200 as sz
from szsnn_b200.workloads import izh_network, thalamic  # noqa: F401  (shared with the benchmark)


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


def forced_schedule(n, steps, every=7, first=3):
    return [list(range(0, n, every)) if t < first else None for t in range(steps)]


def forced_words(sched, n_units):
    W = (n_units + 31) // 32
    fw = np.zeros((len(sched), W), np.uint32)
    for t, ids in enumerate(sched):
        if ids is not None and len(ids):
            fw[t] = sz.ids_to_words(ids, n_units)
    return fw


def raster_bits(raster, n):
    """[steps][W] uint32 words -> [steps][n] bool."""
    return np.unpackbits(raster.view(np.uint8), bitorder="little").reshape(raster.shape[0], -1)[:, :n].astype(bool)


def rate_cv(raster, n, dt_ms):
    """(population rate in Hz, ISI-CV of the pooled inter-spike intervals, spikes) of units 0..n-1."""
    b = raster_bits(raster, n)
    steps = b.shape[0]
    rate = b.sum() / n / (steps * dt_ms * 1e-3)
    t, i = np.nonzero(b)
    order = np.lexsort((t, i))
    t, i = t[order], i[order]
    same = i[1:] == i[:-1]
    isi = (t[1:] - t[:-1])[same].astype(np.float64)
    cv = isi.std() / isi.mean() if isi.size > 10 else float("nan")
    return rate, cv, int(b.sum())
