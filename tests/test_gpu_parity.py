"""GPU parity: the sm_100a kernels, through the C ABI, against the oracle.

Bar (from the acceptance criteria): spike rasters bit-exact and state
bit-exact wherever fp32 sums are order independent (dyadic weights, or the
fixed-point accumulation mode); with order-dependent fp32 sums, rasters equal
for the first 100 steps and state within 1e-5 relative.
"""
import os

import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from tests.helpers import forced_schedule, forced_words, if_network, izh_network, thalamic
from tests.test_oracle import (GOLD, _golden_log_run, check_golden_log, golden_log_network, pynn_network)

pytestmark = pytest.mark.gpu

clemu = pytest.importorskip("oracle.clemu")


@pytest.fixture(scope="module")
def ctx_small(built):
    c = sz.Context(0, max_partition_size=256, threads_per_group=64, warp_size=32, max_synaptic_delay=64)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_prod(built):
    c = sz.Context(0)
    yield c
    c.close()


# ------------------------------------------------------------ golden vectors
def test_gpu_matches_szsnn_fp32_log(ctx_prod):
    g, fw, vals = _golden_log_run(None)
    pops, csr, st, P = golden_log_network()
    net = sz.Network(ctx_prod, 1, P, 1, pops, csr=csr, state=st)
    vs, ies, spk = [], [], []
    for c in range(len(g["v"])):
        out = net.step(forced_words=fw[c])
        vs.append(net.get_state(0)[0])
        ies.append(net.get_state(1)[0])
        spk.append(bool(out[0] & 1))
    check_golden_log(np.array(vs, np.float32), np.array(ies, np.float32), np.array(spk), g)


def test_gpu_matches_pynn_trace_and_oracle(ctx_prod):
    tr = np.load(os.path.join(GOLD, "pynn_2neuron_v.npz"))["v"]
    pops, csr, st = pynn_network()
    net = sz.Network(ctx_prod, 2, 0, 2, pops, csr=csr, state=st)
    on = oracle.OracleNet(2, 0, 2, pops, csr, state=st)
    v_gpu, v_orc = [], []
    for _ in range(len(tr)):
        net.step()
        on.run(1)
        v_gpu.append(net.get_state(0)[1])
        v_orc.append(on.state[0][1])
    v_gpu = np.array(v_gpu, np.float32)
    assert np.array_equal(v_gpu, np.array(v_orc, np.float32))
    assert np.max(np.abs(v_gpu - tr) / np.maximum(np.abs(tr), 1.0)) < 1e-6


# ------------------------------------------- drop-in kernels vs reference kernels
def _ref_pair(ctx, variant, model, params, vars_, src, tgt, w, d1, **kw):
    mps = 256 if variant == "small" else 1024
    consts = L.LayoutConsts(mps, mps // 4, 32, 64)
    gpu = sz.RefSimulation(sz.CudaRefBackend(ctx), consts, model, params, vars_, src, tgt, w, d1, **kw)
    ref = sz.RefSimulation(clemu.ClemuBackend(variant), consts, model, params, vars_, src, tgt, w, d1, **kw)
    return gpu, ref


@pytest.mark.parametrize("variant,n", [("small", 700), ("prod", 3000)])
def test_dropin_if_curr_exp_equals_reference_kernels(ctx_small, ctx_prod, variant, n):
    if not clemu.available(variant):
        pytest.skip("reference kernels not built")
    ctx = ctx_small if variant == "small" else ctx_prod
    net = if_network(n=n, n_syn=20 * n, dyadic=True, seed=21)
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    gpu, ref = _ref_pair(ctx, variant, "IF_curr_exp", params, vars_, net["src"], net["tgt"], net["w"], net["d1"])
    steps = 160
    sched = forced_schedule(n, steps)
    cur = np.full((steps, n), 0.6, np.float32)
    total = 0
    for t in range(steps):
        a = gpu.step_and_fired(sched[t], cur[t])
        b = ref.step_and_fired(sched[t], cur[t])
        total += len(b)
        assert np.array_equal(a, b), f"raster differs at step {t}"
    assert total > 200
    assert np.array_equal(gpu.neuron_vars(), ref.neuron_vars())
    assert np.array_equal(gpu.currents(), ref.currents())
    ctx.sync()


def test_dropin_izhikevich_equals_reference_kernels(ctx_prod):
    if not clemu.available("prod"):
        pytest.skip("reference kernels not built")
    net = izh_network(n=1000, seed=8)
    n = net["n"]
    params = np.stack([net["a"], net["b"], net["c"], net["d"]], 1)
    vars_ = np.stack([net["v0"], net["u0"]], 1)
    gpu, ref = _ref_pair(ctx_prod, "prod", "Izhikevich", params, vars_, net["src"], net["tgt"], net["w"], net["d1"])
    steps = 150
    cur = thalamic(n, net["ne"], steps, seed=3)
    for t in range(steps):
        assert np.array_equal(gpu.step_and_fired(None, cur[t]), ref.step_and_fired(None, cur[t])), t
    assert np.array_equal(gpu.neuron_vars(), ref.neuron_vars())
    ctx_prod.sync()


def test_dropin_input_partition_equals_reference_kernels(ctx_small):
    if not clemu.available("small"):
        pytest.skip("reference kernels not built")
    rng = np.random.default_rng(19)
    n, ni = 500, 60
    net = if_network(n=n, n_syn=8000, dyadic=True, seed=6)
    in_base = ((n - 1) // 256 + 1) * 256
    src = np.concatenate([net["src"], in_base + rng.integers(0, ni, 900)])
    tgt = np.concatenate([net["tgt"], rng.integers(0, n, 900)])
    w = np.concatenate([net["w"], np.full(900, 0.75, np.float32)])
    d1 = np.concatenate([net["d1"], rng.integers(1, 10, 900).astype(np.uint32)])
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    rates = rng.integers(3, 12, ni).astype(np.float32)[:, None]
    gpu, ref = _ref_pair(ctx_small, "small", "IF_curr_exp", params, vars_, src, tgt, w, d1, input_params=rates,
                         input_vars=np.zeros((ni, 1), np.float32))
    for t in range(120):
        assert np.array_equal(gpu.step_and_fired(), ref.step_and_fired()), t
    assert np.array_equal(gpu.neuron_vars(), ref.neuron_vars())


def test_dropin_continuous_weights_within_tolerance(ctx_small):
    if not clemu.available("small"):
        pytest.skip("reference kernels not built")
    n = 700
    net = if_network(n=n, n_syn=14000, dyadic=False, seed=12)
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    gpu, ref = _ref_pair(ctx_small, "small", "IF_curr_exp", params, vars_, net["src"], net["tgt"], net["w"], net["d1"])
    sched = forced_schedule(n, 100)
    for t in range(100):
        assert np.array_equal(gpu.step_and_fired(sched[t], None), ref.step_and_fired(sched[t], None)), t
    g, r = gpu.neuron_vars(), ref.neuron_vars()
    assert np.allclose(g[:3], r[:3], rtol=1e-5, atol=1e-4)


def test_dropin_overflow_reported_not_dropped(ctx_small):
    """A gather whose counter exceeds the queue pitch sets the sticky device
    error instead of reading past the queue (gather_kernel.cl has no check)."""
    n = 100
    net = if_network(n=n, n_syn=400, dyadic=True, seed=1)
    params = np.tile(net["pv"][:9], (n, 1))
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    consts = L.LayoutConsts(256, 64, 32, 64)
    sim = sz.RefSimulation(sz.CudaRefBackend(ctx_small), consts, "IF_curr_exp", params, vars_, net["src"], net["tgt"],
                           net["w"], net["d1"])
    gqc = np.zeros(len(sim.arrays_host[L.L_GQ_COUNTER]), np.uint32)
    gqc[1] = sim.info.gq_pitch + 5  # read slot of cycle 0
    sim.buf[L.L_GQ_COUNTER].write(gqc)
    sim.step()
    with pytest.raises(L.SzsnnError):
        ctx_small.sync()
    assert ctx_small.device_error()[0] == 2
    ctx_small.clear_device_error()
    ctx_small.sync()


# ------------------------------------------------------ native network path
def _native_pair(ctx, n, p, D, pops, csr, state, acc=L.ACC_FLOAT):
    net = sz.Network(ctx, n, p, D, pops, csr=csr, state=state, acc_mode=acc, graph_chunk=50)
    on = oracle.OracleNet(n, p, D, pops, csr, state=state)
    return net, on


@pytest.mark.parametrize("D", [64, 100])
def test_native_if_curr_exp_equals_oracle(ctx_prod, D):
    n = 4000
    net_ = if_network(n=n, n_syn=80 * n, max_delay=D, dyadic=True, seed=31)
    csr = sz.csr_from_synapses(n, D, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net, on = _native_pair(ctx_prod, n, 0, D, pops, csr, st)
    steps = 300
    sched = forced_schedule(n, steps)
    fw = forced_words(sched, n)
    r_gpu = net.run(steps, forced_words=fw)
    r_orc, ev = on.run(steps, forced_words=fw)
    assert np.array_equal(r_gpu, r_orc)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    s = net.stats()
    assert s["events"] == ev and s["steps_done"] == steps
    assert s["spikes"] == int(np.unpackbits(r_orc.view(np.uint8)).sum())


def test_native_fixed_point_bit_exact_continuous_weights(ctx_prod):
    n = 3000
    net_ = if_network(n=n, n_syn=60 * n, dyadic=False, seed=41)
    csr = sz.csr_from_synapses(n, 64, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx_prod, n, 0, 64, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED)
    on = oracle.OracleNet(n, 0, 64, pops, csr, state=st)
    fw = forced_words(forced_schedule(n, 400), n)
    cur = np.full((400, n), 0.5, np.float32)
    r_gpu = np.stack([net.step(forced_words=fw[t], current=cur[t]) for t in range(400)])
    r_orc, _ = on.run(400, forced_words=fw, current=cur, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(r_gpu, r_orc)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])


def test_native_float_continuous_weights_tolerance(ctx_prod):
    n = 3000
    net_ = if_network(n=n, n_syn=60 * n, dyadic=False, seed=43)
    csr = sz.csr_from_synapses(n, 64, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net, on = _native_pair(ctx_prod, n, 0, 64, pops, csr, st)
    fw = forced_words(forced_schedule(n, 100), n)
    r_gpu = net.run(100, forced_words=fw)
    r_orc, _ = on.run(100, forced_words=fw)
    assert np.array_equal(r_gpu, r_orc)
    assert np.allclose(net.get_state(0), on.state[0], rtol=1e-5, atol=1e-4)


def test_native_izhikevich_half_steps_equals_oracle(ctx_prod):
    net_ = izh_network(n=1000, seed=5)
    n = net_["n"]
    csr = sz.csr_from_synapses(n, 20, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pn = np.zeros((12, n), np.float32)
    pn[0], pn[1], pn[2], pn[3] = net_["a"], net_["b"], net_["c"], net_["d"]
    pops = [sz.Pop(sz.IZHIKEVICH, 0, n, np.zeros(12, np.float32), per_unit=pn, flags=sz.POP_IZH_HALF_STEPS)]
    st = [net_["v0"], net_["u0"], None, None]
    net, on = _native_pair(ctx_prod, n, 0, 20, pops, csr, st)
    cur = thalamic(n, net_["ne"], 300, seed=9)
    r_gpu = np.stack([net.step(current=cur[t]) for t in range(300)])
    r_orc, _ = on.run(300, current=cur)
    assert np.array_equal(r_gpu, r_orc)
    assert np.array_equal(net.get_state(0), on.state[0])


def cond_network(n=20000, p=2000, fanout=100, D=64, seed=99):
    """IF_cond_exp + Poisson network shaped like the 1M-neuron benchmark, scaled."""
    from szsnn_b200.network import GenBlock
    ne = int(0.8 * n)
    blocks = [GenBlock(0, ne, 0, n, fanout, 0.0, 0.004, 1.0, 1, D, True, 1),
              GenBlock(ne, n - ne, 0, n, fanout, 0.0, 0.051, -1.0, 1, D, True, 2),
              GenBlock(n, p, 0, n, 100, 0.0, 0.1, 1.0, 1, 1, False, 3)]
    pv = sz.fold_dt(sz.if_params(v_rest=-60, cm=0.2, tau_m=20, tau_refrac=5, tau_syn_E=5, tau_syn_I=10,
                                 v_reset=-60, v_thresh=-50, e_rev_E=0.0, e_rev_I=-80.0), 0.1)
    pops = [sz.Pop(sz.IF_COND_EXP, 0, n, pv), sz.Pop(sz.POISSON, n, n + p, np.array([5.0 * 0.1e-3 * 20], np.float32),
                                                     seed=2024)]
    rng = np.random.default_rng(seed)
    v0 = np.concatenate([rng.uniform(-60, -50, n), np.zeros(p)]).astype(np.float32)
    st = [v0, None, None, np.concatenate([np.full(n, 1e4), np.zeros(p)]).astype(np.float32)]
    return blocks, pops, st


def test_device_generator_matches_oracle(ctx_prod):
    n, p, D = 20000, 2000, 64
    blocks, pops, st = cond_network(n, p, D=D)
    net = sz.Network(ctx_prod, n, p, D, pops, state=st)
    net.generate(blocks, seed=555)
    rp, tg, w = net.synapses()
    rp2, tg2, w2 = oracle.generate(blocks, 555, n + p, D)
    assert np.array_equal(rp, rp2)
    assert np.array_equal(tg, tg2)
    assert np.array_equal(w, w2)


@pytest.mark.parametrize("acc", [L.ACC_FIXED, L.ACC_FLOAT])
def test_native_if_cond_exp_poisson_equals_oracle(ctx_prod, acc):
    n, p, D = 20000, 2000, 64
    blocks, pops, st = cond_network(n, p, D=D)
    net = sz.Network(ctx_prod, n, p, D, pops, state=st, acc_mode=acc)
    net.generate(blocks, seed=777)
    csr = oracle.generate(blocks, 777, n + p, D)
    on = oracle.OracleNet(n, p, D, pops, csr, state=st)
    steps = 300 if acc == L.ACC_FIXED else 100
    r_gpu = net.run(steps)
    r_orc, ev = on.run(steps, acc_mode=oracle.ACC_FIXED if acc == L.ACC_FIXED else oracle.ACC_FLOAT)
    assert np.array_equal(r_gpu, r_orc)
    assert int(np.unpackbits(r_orc.view(np.uint8)).sum()) > 100
    if acc == L.ACC_FIXED:
        for k in range(4):
            assert np.array_equal(net.get_state(k), on.state[k])
        assert net.stats()["events"] == ev
    else:
        assert np.allclose(net.get_state(0), on.state[0], rtol=1e-5, atol=1e-4)


def test_poisson_rate(ctx_prod):
    n, p = 32, 20000
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, sz.if_params(v_thresh=1e9)),
            sz.Pop(sz.POISSON, n, n + p, np.array([0.01], np.float32), seed=5)]
    net = sz.Network(ctx_prod, n, p, 1, pops, csr=sz.csr_from_synapses(n + p, 1, [], [], [], []))
    r = net.run(500)
    spikes = np.unpackbits(r.view(np.uint8), bitorder="little").reshape(500, -1)[:, n: n + p].sum()
    expected = 0.01 * p * 500
    assert abs(spikes - expected) < 5 * np.sqrt(expected)


def test_graph_chunks_checkpoint_and_restore(ctx_prod):
    n, p, D = 20000, 2000, 64
    blocks, pops, st = cond_network(n, p, D=D, seed=3)
    net = sz.Network(ctx_prod, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=40)
    net.generate(blocks, seed=1)
    net.run(130, raster=False)
    blob = net.checkpoint()
    r1 = net.run(170)
    net.restore(blob)
    r2 = np.stack([net.step() for _ in range(170)])
    assert np.array_equal(r1, r2)
    assert net.check_finite()


def test_native_bad_target_sets_device_error(ctx_prod):
    n = 64
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, sz.if_params(v_thresh=-50, v_rest=-49))]
    csr = sz.csr_from_synapses(n, 1, [0, 1], [5, n + 100], [1.0, 1.0], [1, 1])
    net = sz.Network(ctx_prod, n, 0, 1, pops, csr=csr)
    fw = np.zeros(2, np.uint32)
    fw[0] = 0b11
    net.step(forced_words=fw)
    net.step()
    with pytest.raises(L.SzsnnError):
        ctx_prod.sync()
    assert ctx_prod.device_error() == (1, n + 100)
    ctx_prod.clear_device_error()
    ctx_prod.sync()


@pytest.mark.parametrize("mode,group,blocks,ub", [(0, 4, 148, 128), (0, 32, 592, 256), (1, 8, 296, 64),
                                                   (1, 16, 1184, 256), (1, 32, 2368, 96)])
def test_launch_shapes_are_bit_identical(ctx_prod, mode, group, blocks, ub):
    """Every propagate variant / launch shape gives the oracle's fixed-point result."""
    n, p, D = 20000, 2000, 64
    blocks_, pops, st = cond_network(n, p, D=D, seed=8)
    net = sz.Network(ctx_prod, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED)
    net.generate(blocks_, seed=4242)
    net.set_tuning(mode, group, blocks, ub)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks_, 4242, n + p, D), state=st)
    r_gpu = net.run(150)
    r_orc, ev = on.run(150, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(r_gpu, r_orc)
    assert np.array_equal(net.get_state(0), on.state[0])
    assert net.stats()["events"] == ev
