"""GPU: a network sharded in two (szsnn_net_set_owned + szsnn_net_inject_spikes)
equals the unsharded network and the oracle, bit for bit in fixed point.

Both shards run on one device, one after the other in one process, with the
exchange done on the host between steps (no kernel waits on another); a run
over two devices does the same exchange with an all-gather
(szsnn_b200.sharded.dist_exchange, tested on CPU over gloo).  Each shard
updates its own neuron and source ranges, keeps the synapses into its own
targets, and receives the other shard's spike words after every step.
Both step orders; the union raster, the owned neurons' state and the event
counts must match."""
import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200 import sharded as S
from tests.test_gpu_parity import cond_network

pytestmark = pytest.mark.gpu

STEPS = 120


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("overlap", [True, False])
def test_two_shards_equal_unsharded(ctx, overlap):
    n, p, D = 20_000, 2_000, 32
    blocks, pops, st = cond_network(n, p, fanout=60, D=D, seed=8)
    csr = oracle.generate(blocks, 91, n + p, D)
    U = n + p
    ranges = S.plan(n, p, 2)
    shards = []
    for r in ranges:
        net = sz.Network(ctx, n, p, D, pops, csr=S.shard_csr(csr, U, D, r), state=st, acc_mode=L.ACC_FIXED)
        net.set_overlap(overlap)
        net.set_owned(r.n_lo, r.n_hi, r.s_lo, r.s_hi)
        shards.append(net)
    full = sz.Network(ctx, n, p, D, pops, csr=csr, state=st, acc_mode=L.ACC_FIXED)
    full.set_overlap(overlap)
    union, ref = [], []
    for _ in range(STEPS):
        own = [S.own_words(net.step(), r, U) for net, r in zip(shards, ranges)]
        shards[0].inject_spikes(own[1])
        shards[1].inject_spikes(own[0])
        union.append(own[0] | own[1])
        ref.append(full.step())
    union, ref = np.stack(union), np.stack(ref)
    on = oracle.OracleNet(n, p, D, pops, csr, state=st)
    ro, ev = on.run(STEPS, acc_mode=oracle.ACC_FIXED)
    assert int(np.unpackbits(ro.view(np.uint8)).sum()) > 2000
    assert np.array_equal(ref, ro)
    assert np.array_equal(union, ro)
    for net, r in zip(shards, ranges):
        for k in range(4):
            assert np.array_equal(net.get_state(k)[r.n_lo:r.n_hi], on.state[k][r.n_lo:r.n_hi])
        assert ctx.device_error() == (0, 0)
    assert sum(net.stats()["events"] for net in shards) == ev == full.stats()["events"]
    for net in shards + [full]:
        net.close()


def test_inject_before_any_step_is_refused(ctx):
    n, p, D = 1000, 100, 4
    blocks, pops, st = cond_network(n, p, fanout=10, D=D, seed=3)
    net = sz.Network(ctx, n, p, D, pops, csr=oracle.generate(blocks, 5, n + p, D), state=st)
    with pytest.raises(sz.SzsnnError):
        net.inject_spikes(np.zeros(net.words, np.uint32))
    with pytest.raises(sz.SzsnnError):
        net.set_owned(0, n + 1, n, n + p)
    net.close()
