"""CPU: pin the oracle against the reference's known answers and its own kernels.

  * Philox4x32-10 against the published Random123 known-answer vectors;
  * IF_curr_exp rule against SZSNN's own fp32 debug log (szsnn1.1/bin/myfile.txt~);
  * IF_curr_exp network against the PyNN/Brian 2-neuron trace
    (szsnn1.1/bin/pyNN2neurony.vvv~), fp64 and fp32;
  * Oracle A (C restatement) against Oracle B (the reference's .cl kernels run by
    the CPU work-group emulator) through the same RefSimulation driver.
"""
import os

import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from tests.helpers import forced_schedule, forced_words, if_network, izh_network, thalamic

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_philox_known_answers(built):
    # Random123 kat_vectors, philox4x32 with 10 rounds
    assert list(oracle.philox4x32([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(oracle.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                          0x6D5451FD]
    assert list(oracle.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def _golden_log_run(net_factory):
    g = np.load(os.path.join(GOLD, "szsnn_if_curr_exp_log.npz"))
    T = len(g["v"])
    vals = [0.5, 1.0, 1.5, 3.0]
    assert set(np.unique(g["in_exc"])) <= set([0.0] + vals) and not np.any(g["in_inh"])
    fw = np.zeros((T, 1), np.uint32)
    for c in range(1, T):
        x = g["in_exc"][c]
        if x != 0:
            fw[c - 1, 0] |= np.uint32(1 << (1 + vals.index(x)))
    return g, fw, vals


def golden_log_network():
    """Neuron 0 = the logged IF_curr_exp neuron (v_rest -49, cm 1, tau_m 20,
    tau_syn 5/10, reset -70, threshold -50, no refractoriness); units 1..4 are
    sources whose forced spikes deliver the logged input sums over delay-1
    synapses (0.5, 1.0, 1.5, 3.0)."""
    vals = [0.5, 1.0, 1.5, 3.0]
    pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=0, tau_syn_E=5, tau_syn_I=10, v_reset=-70,
                      v_thresh=-50)
    P = len(vals)
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, 1, pv), sz.Pop(sz.CONST_RATE, 1, 1 + P, np.array([1e9], np.float32))]
    csr = sz.csr_from_synapses(1 + P, 1, list(range(1, 1 + P)), [0] * P, vals, [1] * P)
    st0 = np.zeros(1 + P, np.float32)
    st0[0] = -70
    st3 = np.zeros(1 + P, np.float32)
    st3[0] = 10000
    return pops, csr, [st0, None, None, st3], P


def check_golden_log(vs, ies, spk, g):
    fired_log = g["v"] >= -50
    assert np.array_equal(spk, fired_log), "spike cycles differ from the SZSNN log"
    ref = g["v"][~fired_log]
    ours = vs[~fired_log].astype(np.float64)
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    # the log prints %f; the reference GPU's fp32 divide may be off by an ulp
    # (OpenCL allows 2.5 ulp without -cl-fp32-correctly-rounded-divide-sqrt)
    assert np.max(np.abs(ours - ref) / ulp) <= 2.0
    assert np.mean(np.abs(ours - ref) <= 5.0001e-7) > 0.9
    assert np.all(vs[fired_log] == -70.0)
    assert np.max(np.abs(ies - g["ie"])) <= 5.0001e-7


def test_oracle_matches_szsnn_fp32_log(built):
    g, fw, vals = _golden_log_run(None)
    pops, csr, st, P = golden_log_network()
    on = oracle.OracleNet(1, P, 1, pops, csr, state=st)
    vs, ies, spk = [], [], []
    for c in range(len(g["v"])):
        r, _ = on.run(1, forced_words=fw[c:c + 1])
        vs.append(on.state[0][0])
        ies.append(on.state[1][0])
        spk.append(bool(r[0, 0] & 1))
    check_golden_log(np.array(vs, np.float32), np.array(ies, np.float32), np.array(spk), g)


def pynn_network():
    pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=0, tau_syn_E=5, tau_syn_I=10, v_reset=-200,
                      v_thresh=-50)
    # PyNN delay 1 ms at dt = 1 ms -> stored delay 2 (user delay + 1, NetworkGraph.ipp:431)
    csr = sz.csr_from_synapses(2, 2, [0], [1], [100.0], [2])
    st = [np.array([-70, -70], np.float32), None, None, np.array([10000, 10000], np.float32)]
    return [sz.Pop(sz.IF_CURR_EXP, 0, 2, pv)], csr, st


@pytest.mark.parametrize("dtype,rtol", [(np.float64, 1e-9), (np.float32, 1e-6)])
def test_oracle_matches_pynn_trace(built, dtype, rtol):
    tr = np.load(os.path.join(GOLD, "pynn_2neuron_v.npz"))["v"]
    pops, csr, st = pynn_network()
    on = oracle.OracleNet(2, 0, 2, pops, csr, state=st, dtype=dtype)
    v1 = []
    for _ in range(len(tr)):
        on.run(1)
        v1.append(on.state[0][1])
    v1 = np.array(v1, np.float64)
    assert np.max(np.abs(v1 - tr) / np.maximum(np.abs(tr), 1.0)) < rtol


# --------------------------------------------------------------- Oracle A vs B
clemu = pytest.importorskip("oracle.clemu")


def _need_clemu(variant):
    if not clemu.available(variant):
        pytest.skip("reference kernels not built (oracle/_ref missing)")


def _run_ab_if(net, steps, variant, consts, current):
    n = net["n"]
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    sim = sz.RefSimulation(clemu.ClemuBackend(variant), consts, "IF_curr_exp", params, vars_, net["src"],
                           net["tgt"], net["w"], net["d1"])
    sched = forced_schedule(n, steps)
    rasB = [sim.step_and_fired(sched[t], current[t]) for t in range(steps)]
    csr = sz.csr_from_synapses(n, net["D"], net["src"], net["tgt"], net["w"], net["d1"])
    on = oracle.OracleNet(n, 0, net["D"], [sz.Pop(sz.IF_CURR_EXP, 0, n, net["pv"])], csr,
                          state=[net["v0"], None, None, np.full(n, 10000.0, np.float32)])
    rasA, _ = on.run(steps, forced_words=forced_words(sched, n), current=current)
    return rasA, rasB, sim.neuron_vars(), on.state


@pytest.mark.parametrize("variant,n", [("small", 300), ("prod", 1500)])
def test_oracle_a_equals_reference_kernels_if(built, variant, n):
    _need_clemu(variant)
    mps = 256 if variant == "small" else 1024
    consts = L.LayoutConsts(mps, mps // 4, 32, 64)
    net = if_network(n=n, n_syn=20 * n, dyadic=True, seed=11)
    steps = 150
    cur = np.full((steps, n), 0.6, np.float32)
    rasA, rasB, varsB, stA = _run_ab_if(net, steps, variant, consts, cur)
    total = 0
    for t in range(steps):
        a = sz.words_to_ids(rasA[t], n)
        total += len(a)
        assert np.array_equal(a, rasB[t]), f"raster differs at step {t}"
    assert total > 100
    for k in range(4):
        assert np.array_equal(varsB[k], stA[k]), f"state var {k} differs"


def test_oracle_a_close_to_reference_kernels_continuous_weights(built):
    """Non-dyadic weights: sums depend on order, so the bar is the north-star
    tolerance -- rasters equal for the first 100 steps, state within 1e-5 rel."""
    _need_clemu("small")
    consts = L.LayoutConsts(256, 64, 32, 64)
    n = 400
    net = if_network(n=n, n_syn=8000, dyadic=False, seed=5)
    steps = 100
    cur = np.full((steps, n), 0.55, np.float32)
    rasA, rasB, varsB, stA = _run_ab_if(net, steps, "small", consts, cur)
    for t in range(steps):
        assert np.array_equal(sz.words_to_ids(rasA[t], n), rasB[t])
    for k in range(3):
        assert np.allclose(varsB[k], stA[k], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("half", [False])
def test_oracle_a_equals_reference_kernels_izhikevich(built, half):
    _need_clemu("prod")
    consts = L.LayoutConsts(1024, 256, 32, 64)
    net = izh_network(n=1000, seed=4)
    n = net["n"]
    steps = 120
    cur = thalamic(n, net["ne"], steps)
    params = np.stack([net["a"], net["b"], net["c"], net["d"]], 1)
    vars_ = np.stack([net["v0"], net["u0"]], 1)
    sim = sz.RefSimulation(clemu.ClemuBackend("prod"), consts, "Izhikevich", params, vars_, net["src"], net["tgt"],
                           net["w"], net["d1"])
    rasB = [sim.step_and_fired(None, cur[t]) for t in range(steps)]
    csr = sz.csr_from_synapses(n, net["D"], net["src"], net["tgt"], net["w"], net["d1"])
    pn = np.zeros((12, n), np.float32)
    pn[0], pn[1], pn[2], pn[3] = net["a"], net["b"], net["c"], net["d"]
    on = oracle.OracleNet(n, 0, net["D"], [sz.Pop(sz.IZHIKEVICH, 0, n, np.zeros(12, np.float32), per_unit=pn)],
                          csr, state=[net["v0"], net["u0"], None, None])
    rasA, _ = on.run(steps, current=cur)
    total = 0
    for t in range(steps):
        a = sz.words_to_ids(rasA[t], n)
        total += len(a)
        assert np.array_equal(a, rasB[t]), f"raster differs at step {t}"
    assert total > 200
    vB = sim.neuron_vars()
    assert np.array_equal(vB[0], on.state[0]) and np.array_equal(vB[1], on.state[1])


def test_oracle_a_equals_reference_kernels_with_input_partition(built):
    """Const_rate input partition (Const_rate_update_kernel.cl) feeding neurons."""
    _need_clemu("small")
    consts = L.LayoutConsts(256, 64, 32, 64)
    rng = np.random.default_rng(9)
    n, ni = 300, 40
    net = if_network(n=n, n_syn=5000, dyadic=True, seed=2)
    in_base = ((n - 1) // 256 + 1) * 256
    isrc = in_base + rng.integers(0, ni, 800)
    itgt = rng.integers(0, n, 800)
    iw = np.full(800, 0.75, np.float32)
    id1 = rng.integers(1, 10, 800).astype(np.uint32)
    rates = rng.integers(3, 12, ni).astype(np.float32)
    src = np.concatenate([net["src"], isrc])
    tgt = np.concatenate([net["tgt"], itgt])
    w = np.concatenate([net["w"], iw])
    d1 = np.concatenate([net["d1"], id1])
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    sim = sz.RefSimulation(clemu.ClemuBackend("small"), consts, "IF_curr_exp", params, vars_, src, tgt, w, d1,
                           input_params=rates[:, None], input_vars=np.zeros((ni, 1), np.float32))
    steps = 120
    rasB = [sim.step_and_fired() for _ in range(steps)]
    # Oracle A: inputs are sources N..N+ni-1; remap their global ids
    osrc = np.where(src >= in_base, src - in_base + n, src)
    csr = sz.csr_from_synapses(n + ni, 64, osrc, tgt, w, d1)
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net["pv"]),
            sz.Pop(sz.CONST_RATE, n, n + ni, np.zeros(12, np.float32), per_unit=rates[None, :])]
    on = oracle.OracleNet(n, ni, 64, pops, csr, state=[np.concatenate([net["v0"], np.zeros(ni, np.float32)]), None,
                                                        None, np.concatenate([np.full(n, 1e4, np.float32),
                                                                              np.zeros(ni, np.float32)])])
    rasA, _ = on.run(steps)
    total = 0
    for t in range(steps):
        a = sz.words_to_ids(rasA[t], n + ni)
        a = a[a < n]
        total += len(a)
        assert np.array_equal(a, rasB[t]), f"raster differs at step {t}"
    assert total > 50


def test_oracle_generator_and_fixed_point(built):
    """Generator is deterministic, delay-bucketed and stable; fixed-point sums
    are order independent (1 thread vs 8 threads give identical rasters)."""
    from szsnn_b200.network import GenBlock

    n, p = 2000, 200
    blocks = [GenBlock(0, 1600, 0, n, 50, 0.0, 0.4, 1.0, 1, 16, True, 1),
              GenBlock(1600, 400, 0, n, 50, 0.0, 2.0, -1.0, 1, 16, True, 2),
              GenBlock(n, p, 0, n, 20, 0.5, 0.5, 1.0, 1, 1, False, 3)]
    rp, tg, w = oracle.generate(blocks, 1234, n + p, 16)
    rp2, tg2, w2 = oracle.generate(blocks, 1234, n + p, 16)
    assert np.array_equal(rp, rp2) and np.array_equal(tg, tg2) and np.array_equal(w, w2)
    assert rp[-1] == len(tg) == 1600 * 50 + 400 * 50 + 200 * 20
    assert np.all(np.diff(rp.astype(np.int64)) >= 0)
    rows = np.repeat(np.arange(n + p), 16)
    for s in (0, 5, 1700, n + 3):
        seg = tg[rp[s * 16]: rp[s * 16 + 16]]
        assert s >= n or s not in seg  # no self-loops
    pv = sz.if_params(v_rest=-65, cm=0.25, tau_m=2.0, tau_refrac=2.0, tau_syn_E=5.0, tau_syn_I=10.0, v_reset=-65,
                      v_thresh=-55)
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, pv), sz.Pop(sz.POISSON, n, n + p, np.array([0.05], np.float32), seed=77)]
    rasters = []
    for threads in (1, 8):
        on = oracle.OracleNet(n, p, 16, pops, (rp, tg, w), state=[np.full(n + p, -60, np.float32), None, None, None])
        r, ev = on.run(200, acc_mode=oracle.ACC_FIXED, nthreads=threads)
        rasters.append(r)
    assert np.array_equal(rasters[0], rasters[1])
    assert rasters[0][:, : n // 32].any()


def test_bptt_reference_matches_finite_differences():
    """FP64 BPTT reference: adjoint == central finite differences where no spike
    flips (subthreshold, surrogate off: beta = 0 gives the exact derivative)."""
    from oracle import bptt_ref as R

    rng = np.random.default_rng(0)
    T, B, M, N, K = 40, 3, 20, 30, 5
    p = dict(v_rest=0.0, cm=1.0, tau_m=20.0, tau_syn_E=5.0, tau_syn_I=10.0, i_offset=0.0, v_reset=0.0,
             v_thresh=1.0, alpha=0.95)
    x = (rng.random((T, B, M)) < 0.1).astype(np.float64)
    W_in = rng.normal(0, 0.004, (M, N))
    W_rec = rng.normal(0, 0.004, (N, N)) * (rng.random((N, N)) < 0.3)
    W_out = rng.normal(0, 1, (N, K))
    v0 = rng.uniform(-0.5, 0.5, (B, N))
    c = rng.normal(size=(B, N))

    def loss(Wi):
        fw = R.forward(p, Wi, W_rec, W_out, x, v0)
        assert fw["S"].sum() == 0
        return float((c * fw["vsum"]).sum()), fw

    _, fw = loss(W_in)
    dWin, _, _ = R.backward(p, W_in, W_rec, W_out, x, fw, None, c, beta=0.0)
    eps = 1e-6
    for _ in range(20):
        j, i = rng.integers(M), rng.integers(N)
        Wp, Wm = W_in.copy(), W_in.copy()
        Wp[j, i] += eps
        Wm[j, i] -= eps
        fd = (loss(Wp)[0] - loss(Wm)[0]) / (2 * eps)
        assert abs(fd - dWin[j, i]) <= 1e-7 * max(abs(fd), 1e-3)
