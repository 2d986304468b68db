"""GPU: the benchmark network at its full size (1M IF_cond_exp neurons x 1000
synapses + 100k Poisson sources x 100, delays U{1..64}), where the oracle
cannot follow, through properties that do not depend on size:

  * in fixed-point accumulation the overlapped step order (one fused launch:
    four-unit bulk-copied update tiles, delay-1 delivery by the spiking warps,
    delays 2..64 by the delivery blocks) and the classic order (delivery, then
    update) give the same rasters, state, spike and event counts, bit for bit;
  * a checkpoint taken in one order and restored into the other network
    continues the same trajectory.
"""
import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L

pytestmark = pytest.mark.gpu

STEPS = 60


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


def _bench_net(ctx, overlap):
    import bench
    n, p, D, blocks, pops = bench.cond_config(1_000_000, 1000)
    net = sz.Network(ctx, n, p, D, pops, state=bench.init_state(n, p, 1), acc_mode=L.ACC_FIXED, graph_chunk=20)
    net.generate(blocks, seed=1)
    net.set_overlap(overlap)
    return net


def test_full_size_orders_agree_and_checkpoint_continues(ctx):
    a = _bench_net(ctx, True)
    b = _bench_net(ctx, False)
    ra, rb = a.run(STEPS), b.run(STEPS)
    assert int(np.unpackbits(ra.view(np.uint8)).sum()) > 10_000
    assert np.array_equal(ra, rb)
    for k in range(4):
        assert np.array_equal(a.get_state(k), b.get_state(k))
    sa, sb = a.stats(), b.stats()
    assert sa["events"] == sb["events"] and sa["spikes"] == sb["spikes"]
    assert sa["events"] > 1_000_000

    blob = a.checkpoint()
    ra2 = a.run(STEPS // 2)
    b.run(7)  # b moves on, then takes a's checkpoint (in the other order)
    b.restore(blob)
    rb2 = b.run(STEPS // 2)
    assert np.array_equal(ra2, rb2)
    for k in range(4):
        assert np.array_equal(a.get_state(k), b.get_state(k))
    assert a.stats()["events"] == b.stats()["events"]
    a.close()
    b.close()
