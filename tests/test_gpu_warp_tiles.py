"""GPU: the persistent update tile schemes (szsnn_net_set_update_tiles mode 1,
warp tiles, and mode 2, persistent block tiles) against the oracle, bit for
bit in fixed-point accumulation.

Each warp of the update grid streams 128-unit tiles through a two-stage
shared-memory ring (bulk copies in, bulk stores out); tiles that straddle a
population boundary run the generic per-unit update.  Covered:
  * IF_cond_exp + Poisson in both step orders, one and three update blocks
    per SM (so warps take several tiles each);
  * forced spikes (IF_curr_exp) and an external current (Izhikevich in two
    half-steps) through the tiles;
  * a network whose unit count is not a multiple of 128 (the last tile is
    short and its bulk transfers are rounded to 16 bytes);
  * populations whose boundaries fall inside warp tiles (generic tiles);
  * switching between the three schemes mid-run;
  * fp32 accumulation with dyadic weights (exact sums in any order);
  * block tiles of 1, 2, 5 and 8 units per thread (szsnn_net_set_update_units).
Persistent block tiles take the block tiles of mode 0 in turn, one mbarrier
phase per loaded tile, in blocks that stay resident for the whole launch.
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


@pytest.mark.parametrize("mode,overlap,per_sm", [(1, True, 1), (1, True, 3), (1, False, 2), (2, True, 0),
                                                 (2, False, 0), (2, True, 1)])
def test_warp_tiles_cond_equal_oracle(ctx, mode, overlap, per_sm):
    n, p, D = 100_000, 10_000, 16
    blocks, pops, st = cond_network(n, p, fanout=40, D=D, seed=8)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.generate(blocks, seed=77)
    net.set_overlap(overlap)
    net.set_update_tiles(mode, per_sm)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 77, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    assert net.ctx.device_error() == (0, 0)
    net.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_warp_tiles_forced_if_curr_exp(ctx, mode):
    n = 110_000
    net_ = if_network(n=n, n_syn=40 * n, max_delay=8, dyadic=False, seed=12)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx, n, 0, 8, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.set_update_tiles(mode, 2 if mode == 1 else 0)
    on = oracle.OracleNet(n, 0, 8, pops, csr, state=st)
    fw = forced_words(forced_schedule(n, 40), n)
    r = net.run(40, forced_words=fw)
    ro, ev = on.run(40, forced_words=fw, acc_mode=oracle.ACC_FIXED)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_warp_tiles_izhikevich_current_short_last_tile(ctx, mode):
    """Izhikevich in 2 x 0.5 ms half-steps with a thalamic current; 50,003
    units, so the last warp tile holds 83 units."""
    n = 50_003
    net_ = if_network(n=n, n_syn=30 * n, max_delay=8, dyadic=False, seed=21)
    csr = sz.csr_from_synapses(n, 8, net_["src"], net_["tgt"], net_["w"] * 4, net_["d1"])
    pv = sz.izh_params(0.02, 0.2, -65.0, 8.0)
    v0 = (np.full(n, -70.0) + 5 * np.random.default_rng(3).random(n)).astype(np.float32)
    st = [v0, (0.2 * v0).astype(np.float32), None, None]
    pops = [sz.Pop(sz.IZHIKEVICH, 0, n, pv, flags=sz.POP_IZH_HALF_STEPS)]
    steps = 50
    cur = thalamic(n, int(0.8 * n), steps, seed=4)
    net = sz.Network(ctx, n, 0, 8, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.set_update_tiles(mode, 2 if mode == 1 else 0)
    dcur = ctx.upload(cur)
    raster = ctx.buffer(steps * net.words * 4)
    net.run_device(steps, current_ptr=dcur.ptr, raster_ptr=raster.ptr)
    r = raster.read(np.uint32, steps * net.words).reshape(steps, net.words)
    on = oracle.OracleNet(n, 0, 8, pops, csr, state=st)
    ro, ev = on.run(steps, current=cur, acc_mode=oracle.ACC_FIXED)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(2):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    dcur.free()
    raster.free()
    net.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_warp_tiles_population_boundaries_inside_tiles(ctx, mode):
    """Three populations whose boundaries fall inside warp tiles: those tiles
    take the generic per-unit update, the others the shared-memory ring."""
    n, p, D = 60_000, 6_000, 16
    blocks, pops, st = cond_network(n, p, fanout=40, D=D, seed=9)
    pv2 = np.array(pops[0].params, np.float32).copy()
    pv2[8] = pv2[8] + np.float32(0.5)  # a different threshold
    cut = 30_050
    pops = [sz.Pop(pops[0].model, 0, cut, pops[0].params), sz.Pop(pops[0].model, cut, n, pv2), pops[1]]
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.generate(blocks, seed=78)
    net.set_update_tiles(mode, 2 if mode == 1 else 0)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 78, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    net.close()


def test_warp_tiles_switch_mid_run_and_float_dyadic(ctx):
    """Block tiles, then warp tiles, then block tiles again, fp32 accumulation
    with dyadic weights: every step equals the oracle."""
    n = 90_000
    net_ = if_network(n=n, n_syn=40 * n, max_delay=16, dyadic=True, seed=33)
    csr = sz.csr_from_synapses(n, 16, net_["src"], net_["tgt"], net_["w"], net_["d1"])
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, net_["pv"])]
    st = [net_["v0"], None, None, np.full(n, 1e4, np.float32)]
    net = sz.Network(ctx, n, 0, 16, pops, csr=csr, state=st, graph_chunk=20)
    on = oracle.OracleNet(n, 0, 16, pops, csr, state=st)
    parts = [net.run(30)]
    net.set_update_tiles(1, 2)
    parts.append(net.run(30))
    net.set_update_tiles(2, 0)
    parts.append(net.run(30))
    net.set_update_tiles(0, 0)
    parts.append(net.run(30))
    r = np.concatenate(parts)
    ro, ev = on.run(120)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    net.close()


@pytest.mark.parametrize("units", [1, 2, 5, 8])
def test_update_units_per_thread_equal_oracle(ctx, units):
    """szsnn_net_set_update_units: longer or shorter block tiles (block size
    x units), including tiles that do not divide the populations, give the
    oracle's rasters and state bit for bit."""
    n, p, D = 60_000, 6_000, 16
    blocks, pops, st = cond_network(n, p, fanout=40, D=D, seed=10)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=25)
    net.generate(blocks, seed=79)
    net.set_tuning(1, 16, 296, 128)
    net.set_update_units(units)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 79, n + p, D), state=st)
    r = net.run(60)
    ro, ev = on.run(60, acc_mode=oracle.ACC_FIXED)
    assert _spikes(ro) > 1000
    assert np.array_equal(r, ro)
    for k in range(4):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    with pytest.raises(sz.SzsnnError):
        net.set_update_units(17)
    net.close()
