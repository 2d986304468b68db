"""GPU: the state monitor.

Traces of chosen units' state slots, recorded on the device after every step,
equal the oracle's state after each step (fixed-point accumulation), in both
step orders, through CUDA-graph runs from the host, single steps and device
runs.  Steps past the capacity are counted, not recorded, and each read
restarts the recording.
"""
import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from tests.test_gpu_parity import cond_network

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


def _oracle_steps(on, steps, ids, slots):
    out = []
    for _ in range(steps):
        on.run(1, acc_mode=oracle.ACC_FIXED)
        out.append(np.stack([on.state[k][ids] for k in slots]))
    return np.stack(out)


@pytest.mark.parametrize("overlap", [True, False])
def test_monitor_traces_equal_oracle(ctx, overlap):
    n, p, D = 3000, 300, 8
    blocks, pops, st = cond_network(n, p, fanout=50, D=D, seed=3)
    net = sz.Network(ctx, n, p, D, pops, state=st, acc_mode=L.ACC_FIXED, graph_chunk=10)
    net.generate(blocks, seed=21)
    net.set_overlap(overlap)
    on = oracle.OracleNet(n, p, D, pops, oracle.generate(blocks, 21, n + p, D), state=st)
    ids = np.sort(np.random.default_rng(0).choice(n + p, 40, replace=False)).astype(np.int32)

    net.set_monitor(ids, slots=(0, 1, 3), capacity=64)
    net.run(25)                 # host run: graphs of 1, 10, 10, 3 and 1 steps
    for _ in range(3):
        net.step()
    net.run_device(7)
    ctx.sync()
    tr, dropped = net.monitor_read()
    assert dropped == 0 and tr.shape == (35, 3, 40)
    assert np.array_equal(tr, _oracle_steps(on, 35, ids, (0, 1, 3)))

    # past the capacity: counted, not recorded
    net.set_monitor(ids, slots=(0,), capacity=5)
    net.run(8)
    tr2, dropped2 = net.monitor_read()
    ref2 = _oracle_steps(on, 8, ids, (0,))
    assert tr2.shape == (5, 1, 40) and dropped2 == 3
    assert np.array_equal(tr2, ref2[:5])

    # the read restarted the recording at the current step
    net.run(2)
    tr3, dropped3 = net.monitor_read()
    assert dropped3 == 0 and np.array_equal(tr3, _oracle_steps(on, 2, ids, (0,)))

    net.set_monitor([], slots=(0,))  # off
    with pytest.raises(ValueError):
        net.monitor_read()
    net.close()


def test_monitor_rejects_bad_arguments(ctx):
    n, p, D = 500, 50, 4
    blocks, pops, st = cond_network(n, p, fanout=10, D=D, seed=5)
    net = sz.Network(ctx, n, p, D, pops, state=st)
    with pytest.raises(L.SzsnnError):
        net.set_monitor([0, n + p], slots=(0,))   # unit id outside the network
    with pytest.raises(L.SzsnnError):
        net.set_monitor([0], slots=(0,), capacity=0)
    with pytest.raises(ValueError):
        net.set_monitor([0], slots=(4,))
    net.close()
