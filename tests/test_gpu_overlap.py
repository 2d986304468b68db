"""GPU: the overlapped step order and the pipelined host I/O.

  * overlapped order (delays >= 2 delivered while the update runs, delay 1
    delivered by the update itself) equals the classic order and the oracle bit
    for bit in fixed-point accumulation, including D = 1 and D = 2 (no far
    delivery / a one-bucket far delivery);
  * switching the order mid-run and restoring a checkpoint taken in the other
    order rebuild the next step's inputs from the spike ring: same rasters,
    state and event counts;
  * host arrays in page-locked memory (DMA) and pageable memory (bounce
    buffers), and device arrays, give the same raster, for chunk counts that
    exercise both stage buffers;
  * the update's tiles of four units per thread (bulk-copied inline tiles for
    IF_cond_exp, IF_curr_exp, Izhikevich and Poisson, and a generic tile across
    a population boundary) equal the oracle in both step orders.
"""
import numpy as np
import pytest
import torch

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from tests.helpers import forced_schedule, forced_words, if_network
from tests.test_gpu_parity import cond_network

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


def _cond(ctx, overlap, seed=4242, chunk=40, n=20000, p=2000, D=64):
    blocks, pops, st = cond_network(n, p, D=D, seed=8)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=chunk)
    net.generate(blocks, seed=seed)
    net.set_overlap(overlap)
    return net, blocks, pops, st


def test_overlapped_equals_classic_and_oracle(ctx):
    n, p, D = 20000, 2000, 64
    a, blocks, pops, st = _cond(ctx, True)
    b, *_ = _cond(ctx, False)
    ra, rb = a.run(150), b.run(150)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 4242, n + p, D), state=st)
    ro, ev = on.run(150, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(ra, ro) and np.array_equal(rb, ro)
    for k in range(4):
        assert np.array_equal(a.get_state(k), on.state[k])
        assert np.array_equal(b.get_state(k), on.state[k])
    sa, sb = a.stats(), b.stats()
    assert sa["events"] == sb["events"] == ev
    assert sa["spikes"] == sb["spikes"] == int(np.unpackbits(ro.view(np.uint8)).sum())
    # single steps continue the same trajectory in both orders
    for _ in range(7):
        assert np.array_equal(a.step(), b.step())
    a.close()
    b.close()


@pytest.mark.parametrize("D", [1, 2, 3])
def test_short_delays_equal_oracle(ctx, D):
    n = 3000
    net_ = if_network(n=n, n_syn=60 * n, max_delay=D, dyadic=False, seed=60 + D)
    csr = sz.csr_from_synapses(n, D, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx, n, 0, D, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    on = oracle.OracleNet(n, 0, D, pops, csr, state=st)
    fw = forced_words(forced_schedule(n, 200), n)
    r = net.run(200, forced_words=fw)
    ro, ev = on.run(200, forced_words=fw, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(r, ro)
    assert np.array_equal(net.get_state(0), on.state[0])
    assert net.stats()["events"] == ev
    net.close()


def test_switching_order_mid_run(ctx):
    n, p, D = 20000, 2000, 64
    net, blocks, pops, st = _cond(ctx, True, seed=99, chunk=30)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 99, n + p, D), state=st)
    parts = []
    for overlap, steps in ((True, 45), (False, 50), (True, 37), (True, 20), (False, 8)):
        net.set_overlap(overlap)
        parts.append(net.run(steps))
    ro, ev = on.run(160, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(np.concatenate(parts), ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()


@pytest.mark.parametrize("save_overlap,load_overlap", [(True, False), (False, True), (True, True)])
def test_checkpoint_across_orders(ctx, save_overlap, load_overlap):
    a, *_ = _cond(ctx, save_overlap, seed=7)
    a.run(90, raster=False)
    blob = a.checkpoint()
    ev0 = a.stats()["events"]
    r1 = a.run(70)
    ev1 = a.stats()["events"]
    b, *_ = _cond(ctx, load_overlap, seed=7)
    b.restore(blob)
    assert b.stats()["events"] == ev0
    r2 = b.run(70)
    assert np.array_equal(r1, r2)
    assert b.stats()["events"] == ev1
    for k in range(4):
        assert np.array_equal(a.get_state(k), b.get_state(k))
    a.close()
    b.close()


def test_host_io_pinned_pageable_and_device(ctx):
    steps = 230  # chunks of 40: both stage buffers, a partial last chunk
    n = 20000
    nets = [_cond(ctx, True, seed=5)[0] for _ in range(3)]
    words = nets[0].words
    rng = np.random.default_rng(0)
    fw = np.zeros((steps, words), np.uint32)
    ids = rng.integers(0, n, 400)
    ts = rng.integers(0, steps, 400)
    for t, i in zip(ts, ids):
        fw[t, i >> 5] |= np.uint32(1) << np.uint32(i & 31)
    # pageable in / out
    r_page = nets[0].run(steps, forced_words=fw)
    # page-locked in / out
    fw_pin = torch.empty((steps, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    fw_pin[:] = fw
    out_pin = torch.empty((steps, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    r_pin = nets[1].run(steps, forced_words=fw_pin, out=out_pin)
    # device in / out
    fw_dev = torch.from_numpy(fw.view(np.int32)).cuda()
    out_dev = torch.empty((steps, words), dtype=torch.int32, device="cuda")
    nets[2].run_device(steps, forced_ptr=fw_dev.data_ptr(), raster_ptr=out_dev.data_ptr())
    ctx.sync()
    r_dev = out_dev.cpu().numpy().view(np.uint32)
    assert np.array_equal(r_page, r_pin) and np.array_equal(r_page, r_dev)
    assert int(np.unpackbits(r_page.view(np.uint8)).sum()) > 1000
    for net in nets:
        net.close()


# Tiles of four units per thread.  The update picks them when its grid still
# holds at least four blocks per SM; with 32-thread update blocks that is from
# 75,776 units on (110,000 units: ceil(110000 / (148 * 32)) = 24 blocks per SM
# at one unit per thread, 24 / 4 >= 4).  Each tile of 128 units inside one
# population is brought into shared memory by bulk copies; the tile that
# straddles the neuron / source boundary runs the generic update.
TILE_N, TILE_P = 100_000, 10_000


@pytest.mark.parametrize("overlap", [True, False])
def test_four_unit_tiles_cond_equal_oracle(ctx, overlap):
    n, p, D = TILE_N, TILE_P, 16
    blocks, pops, st = cond_network(n, p, fanout=40, D=D, seed=8)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.generate(blocks, seed=77)
    net.set_overlap(overlap)
    net.set_tuning(1, 32, 0, 32)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 77, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    assert int(np.unpackbits(ro.view(np.uint8)).sum()) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()


def _forced_tile_net(ctx, model, overlap):
    n = TILE_N + TILE_P
    net_ = if_network(n=n, n_syn=40 * n, max_delay=8, dyadic=False, seed=12)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    if model == sz.IZHIKEVICH:
        pv = np.zeros(12, np.float32)
        pv[:4] = (0.02, 0.2, -65.0, 8.0)
        v0 = np.full(n, -65.0, np.float32) + net_["v0"] + 60.0
        st = [v0, (0.2 * v0).astype(np.float32), None, None]
    else:
        pv = net_["pv"]
        st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    pops = [sz.Pop(model, 0, n, pv)]
    net = sz.Network(ctx, n, 0, 8, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.set_overlap(overlap)
    net.set_tuning(1, 32, 0, 32)
    return net, oracle.OracleNet(n, 0, 8, pops, csr, state=st), n


@pytest.mark.parametrize("model,overlap", [(sz.IF_CURR_EXP, True), (sz.IZHIKEVICH, False)])
def test_four_unit_tiles_forced_equal_oracle(ctx, model, overlap):
    net, on, n = _forced_tile_net(ctx, model, overlap)
    fw = forced_words(forced_schedule(n, 40), n)
    r = net.run(40, forced_words=fw)
    ro, ev = on.run(40, forced_words=fw, acc_mode=oracle.ACC_FIXED)
    assert int(np.unpackbits(ro.view(np.uint8)).sum()) > 1000
    assert np.array_equal(r, ro)
    for k in range(2 if model == sz.IZHIKEVICH else 4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()
