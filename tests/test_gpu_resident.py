"""GPU: resident stepping (szsnn_net_set_resident) against the oracle, bit for
bit in fixed-point accumulation.

Each run chunk is one cooperative launch whose blocks keep their neurons'
state in shared memory across the chunk's steps; update warps and delivery
warps share every block, and a bounded grid barrier ends each step.  Covered:
  * IF_cond_exp + Poisson with several update-warp splits and block counts
    (block counts that do not divide the words, 11 blocks of ~9,100 neurons);
  * chunks of several lengths in one run (graph_chunk 25 over 60 steps);
  * forced spikes through the host run (IF_curr_exp) and an external
    current with Izhikevich half-steps through the device run;
  * a network smaller than one word per block, and neuron counts that are
    not multiples of 32 (a raster word of neurons and sources);
  * several populations, one boundary inside a block's range;
  * switching between resident chunks and the per-step graphs mid-run, and
    single steps (szsnn_net_step) between resident runs;
  * fp32 accumulation with dyadic weights (exact sums in any order);
  * per-unit parameter tables (the 1000-neuron Izhikevich network);
  * the networks resident stepping refuses, with the reason.
"""
import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200.workloads import thalamic
from tests.helpers import forced_schedule, forced_words, if_network
from tests.test_gpu_parity import cond_network

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


def _spikes(r):
    return int(np.unpackbits(r.view(np.uint8)).sum())


def _check(net, on, r, ro, ev, slots=4):
    assert _spikes(ro) > 500
    assert np.array_equal(r, ro)
    for k in range(slots):
        assert np.array_equal(net.get_state(k), on.state[k]), f"state slot {k}"
    assert net.stats()["events"] == ev
    assert net.ctx.device_error() == (0, 0)


@pytest.mark.parametrize("uw,blocks", [(16, 0), (8, 0), (24, 0), (16, 37), (16, 11)])
def test_resident_cond_equals_oracle(ctx, uw, blocks):
    n, p, D = 100_000, 10_000, 16
    bl, pops, st = cond_network(n, p, fanout=40, D=D, seed=8)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.generate(bl, seed=77)
    net.set_resident(True, uw, blocks)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(bl, 77, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev)
    net.close()


def test_resident_forced_if_curr_exp_host_run(ctx):
    n = 110_000
    net_ = if_network(n=n, n_syn=40 * n, max_delay=8, dyadic=False, seed=12)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx, n, 0, 8, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=16)
    net.set_resident(True)
    on = oracle.OracleNet(n, 0, 8, pops, csr, state=st)
    fw = forced_words(forced_schedule(n, 40), n)
    r = net.run(40, forced_words=fw)
    ro, ev = on.run(40, forced_words=fw, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev)
    net.close()


def test_resident_izhikevich_current_odd_size(ctx):
    """Izhikevich in 2 x 0.5 ms half-steps with a thalamic current, 50,003
    neurons (the last word holds 19), through the device run."""
    n = 50_003
    net_ = if_network(n=n, n_syn=30 * n, max_delay=8, dyadic=False, seed=21)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"] * 4, net_["d1"])
    pv = sz.izh_params(0.02, 0.2, -65.0, 8.0)
    v0 = (np.full(n, -70.0) + 5 * np.random.default_rng(3).random(n)).astype(np.float32)
    st = [v0, (0.2 * v0).astype(np.float32), None, None]
    pops = [sz.Pop(sz.IZHIKEVICH, 0, n, pv, flags=sz.POP_IZH_HALF_STEPS)]
    steps = 50
    cur = thalamic(n, int(0.8 * n), steps, seed=4)
    net = sz.Network(ctx, n, 0, 8, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=20)
    net.set_resident(True, 12)
    dcur = ctx.upload(cur)
    raster = ctx.buffer(steps * net.words * 4)
    net.run_device(steps, current_ptr=dcur.ptr, raster_ptr=raster.ptr)
    r = raster.read(np.uint32, steps * net.words).reshape(steps, net.words)
    on = oracle.OracleNet(n, 0, 8, pops, csr, state=st)
    ro, ev = on.run(steps, current=cur, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev, slots=2)
    dcur.free()
    raster.free()
    net.close()


def test_resident_small_network_and_mixed_word(ctx):
    """1,000 neurons and 100 sources (35 words, fewer than the blocks of a
    one-per-SM grid): the word holding neurons 992..999 also holds sources
    1000..1023."""
    n, p, D = 1000, 100, 8
    bl, pops, st = cond_network(n, p, fanout=60, D=D, seed=5)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=50)
    net.generate(bl, seed=9)
    net.set_resident(True)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(bl, 9, n + p, D), state=st)
    r = net.run(200)
    ro, ev = on.run(200, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev)
    net.close()


def test_resident_population_boundary_inside_a_block(ctx):
    n, p, D = 60_000, 6_000, 16
    bl, pops, st = cond_network(n, p, fanout=40, D=D, seed=9)
    pv2 = np.array(pops[0].params, np.float32).copy()
    pv2[8] = pv2[8] + np.float32(0.5)  # a different threshold
    cut = 30_050
    pops = [sz.Pop(pops[0].model, 0, cut, pops[0].params), sz.Pop(pops[0].model, cut, n, pv2), pops[1]]
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=30)
    net.generate(bl, seed=78)
    net.set_resident(True)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(bl, 78, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev)
    net.close()


def test_resident_switch_mid_run_single_steps_float_dyadic(ctx):
    """Graphs, resident chunks, single steps, resident again, graphs: fp32
    accumulation with dyadic weights, every step equal to the oracle."""
    n = 90_000
    net_ = if_network(n=n, n_syn=40 * n, max_delay=16, dyadic=True, seed=33)
    csr = sz.csr_from_synapses(n, 16, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx, n, 0, 16, pops, csr=csr, state=st, graph_chunk=20)
    on = oracle.OracleNet(n, 0, 16, pops, csr, state=st)
    parts = [net.run(30)]
    net.set_resident(True)
    parts.append(net.run(30))
    parts.append(np.stack([net.step() for _ in range(3)]))
    parts.append(net.run(27))
    net.set_resident(False)
    parts.append(net.run(30))
    r = np.concatenate(parts)
    ro, ev = on.run(120)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()


def test_resident_per_unit_izhikevich_equals_oracle(ctx):
    """The 1000-neuron Izhikevich network with per-neuron a, b, c, d (per-unit
    parameter tables, updated unit by unit), thalamic current, half-steps."""
    from szsnn_b200 import workloads as WL
    izh = WL.izh_network(n=1000, seed=5)
    pops, csr, st = WL.izh_native(izh)
    pops[0].flags = sz.POP_IZH_HALF_STEPS
    steps = 300
    cur = WL.thalamic(1000, izh["ne"], steps, seed=9)
    net = sz.Network(ctx, 1000, 0, izh["D"], pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=100)
    net.set_resident(True)
    dcur = ctx.upload(cur)
    raster = ctx.buffer(steps * net.words * 4)
    net.run_device(steps, current_ptr=dcur.ptr, raster_ptr=raster.ptr)
    r = raster.read(np.uint32, steps * net.words).reshape(steps, net.words)
    on = oracle.OracleNet(1000, 0, izh["D"], pops, csr, state=st)
    ro, ev = on.run(steps, current=cur, acc_mode=oracle.ACC_FIXED)
    _check(net, on, r, ro, ev, slots=2)
    dcur.free()
    raster.free()
    net.close()


def test_resident_refusals(ctx):
    n = 2000
    net_ = if_network(n=n, n_syn=20 * n, max_delay=8, dyadic=True, seed=2)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    const = sz.Network(ctx, n, 32, 8, [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"]),
                                       sz.Pop(sz.CONST_RATE, n, n + 32, np.array([7.0], np.float32))],
                       csr=sz.csr_from_synapses(n + 32, 8, net_["src"], net_["tgt"], net_["w"], net_["d1"]),
                       state=[np.concatenate([net_["v0"], np.zeros(32, np.float32)]), None, None,
                              np.concatenate([np.full(n, 1e4, np.float32), np.zeros(32, np.float32)])])
    with pytest.raises(sz.SzsnnError, match="sources other than Poisson"):
        const.set_resident(True)
    const.close()
    net = sz.Network(ctx, n, 0, 8, [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])], csr=csr, state=st)
    net.set_overlap(False)
    with pytest.raises(sz.SzsnnError, match="overlapped"):
        net.set_resident(True)
    net.set_overlap(True)
    net.set_resident(True)
    net.set_monitor([1, 2, 3])
    with pytest.raises(sz.SzsnnError, match="monitor"):
        net.run(5)
    net.close()
