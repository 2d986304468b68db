"""GPU: the reference's own host code on the C ABI.

oracle/_ref/refhost is the reference's unchanged Simulation<float>,
NetworkGraph and layout builders compiled against szsnn_b200/compat (its
OpenCL Context replaced by one over the szsnn C ABI).  Its stepAndFired()
runs gather -> update -> scatter on the sm_100a drop-in kernels, with the
reference's blocking waits and firing-output read-back.  Each network here
runs through it and through the reference's own kernels under the CPU
work-group emulator (Oracle B, driven by the Python mirror of the same
host); with exactly summable weights the firing output of every step and
the final neuron variables must agree bit for bit:
  * an IF_curr_exp network with forced spikes (partitions of 1024);
  * the 1000-neuron Izhikevich network (800 RS / 200 FS, 100 targets,
    weights 6 / -5, delays U{1..20}), driven by forced spikes: the
    reference's host has no current input (Simulation.ipp:463-468);
  * an IF_curr_exp network with a Const_rate input partition whose units are
    forced by Poisson trains drawn on the host (partitions of 256).
"""
import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200.workloads import izh_network
from tests import refhost
from tests.helpers import if_network

pytestmark = pytest.mark.gpu

clemu = pytest.importorskip("oracle.clemu")


def _need(small):
    if not refhost.available(small):
        pytest.skip("reference host not built (oracle/_ref/refhost)")
    variant = "small" if small else "prod"
    if not clemu.available(variant):
        pytest.skip("reference kernels not built (oracle/_ref)")


def _compare(tmp_path, small, model, params, vars_, src_ref, src_mirror, tgt, w, d1, forced, ni=0, rates=None):
    mps = 256 if small else 1024
    rates = np.zeros(0, np.float32) if rates is None else np.asarray(rates, np.float32)
    spec, out = tmp_path / "net.spec", tmp_path / "run.out"
    refhost.write_spec(spec, model, params, vars_, rates, src_ref, tgt, w, np.asarray(d1) - 1, forced)
    got = refhost.run("run", spec, out, small=small)
    consts = L.LayoutConsts(mps, mps // 4, 32, 64)
    sim = sz.RefSimulation(clemu.ClemuBackend("small" if small else "prod"), consts,
                           "IF_curr_exp" if model == 0 else "Izhikevich", params, vars_, src_mirror, tgt, w, d1,
                           input_params=None if not ni else rates[:, None],
                           input_vars=None if not ni else np.zeros((ni, 1), np.float32))
    counts, ids = got["fired_counts"], got["fired_ids"]
    assert len(counts) == len(forced)
    off, total = 0, 0
    for t, f in enumerate(forced):
        ref_ids = sim.step_and_fired(f)
        mine = np.sort(ids[off:off + counts[t]])
        off += counts[t]
        total += len(ref_ids)
        assert np.array_equal(mine, np.sort(ref_ids)), f"firing output differs at step {t}"
    n = params.shape[0]
    vc = vars_.shape[1]
    v_ref = sim.neuron_vars()
    raw = got["neuron_vars"].reshape(vc, -1)
    idx = (np.arange(n) // mps) * mps + np.arange(n) % mps
    for k in range(vc):
        assert np.array_equal(raw[k, idx], v_ref[k]), f"neuron variable {k}"
    return total


def test_reference_host_if_curr_exp_forced(tmp_path):
    _need(False)
    n, steps = 1500, 150
    net = if_network(n=n, n_syn=20 * n, dyadic=True, seed=11)
    params = np.tile(net["pv"][:9], (n, 1)).astype(np.float32)
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 1e4)], 1).astype(np.float32)
    rng = np.random.default_rng(5)
    forced = [np.sort(rng.choice(n, 60, replace=False)) if t % 3 == 0 else None for t in range(steps)]
    total = _compare(tmp_path, False, 0, params, vars_, net["src"], net["src"], net["tgt"], net["w"], net["d1"],
                     forced)
    assert total > 2000


def test_reference_host_izhikevich_1000(tmp_path):
    _need(False)
    net = izh_network(n=1000, seed=4)
    n, steps = 1000, 120
    params = np.stack([net["a"], net["b"], net["c"], net["d"]], 1).astype(np.float32)
    vars_ = np.stack([net["v0"], net["u0"]], 1).astype(np.float32)
    rng = np.random.default_rng(7)
    forced = [np.sort(rng.choice(n, 40, replace=False)) for _ in range(steps)]
    total = _compare(tmp_path, False, 1, params, vars_, net["src"], net["src"], net["tgt"], net["w"], net["d1"],
                     forced)
    assert total > 4000


def test_reference_host_input_partition_poisson(tmp_path):
    _need(True)
    rng = np.random.default_rng(9)
    n, ni, steps = 600, 200, 200
    net = if_network(n=n, n_syn=12 * n, dyadic=True, seed=2)
    in_base = -(-n // 256) * 256
    j = rng.integers(0, ni, 4000)
    src_mirror = np.concatenate([net["src"], in_base + j])
    src_ref = np.concatenate([net["src"], n + j])
    tgt = np.concatenate([net["tgt"], rng.integers(0, n, 4000)])
    w = np.concatenate([net["w"], np.full(4000, 0.75, np.float32)])
    d1 = np.concatenate([net["d1"], rng.integers(1, 10, 4000).astype(np.uint32)])
    params = np.tile(net["pv"][:9], (n, 1)).astype(np.float32)
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 1e4)], 1).astype(np.float32)
    rates = np.zeros(ni, np.float32)  # Const_rate never fires by itself (its counter starts above 0)
    forced = []
    for _ in range(steps):
        k = np.nonzero(rng.random(ni) < 0.05)[0]
        forced.append(in_base + k if len(k) else None)
    total = _compare(tmp_path, True, 0, params, vars_, src_ref, src_mirror, tgt, w, d1, forced, ni=ni, rates=rates)
    assert total > 500
