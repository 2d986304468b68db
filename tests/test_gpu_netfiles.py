"""GPU: a network assembled from the reference's own files runs on the native
path exactly like the oracle.

The reference's 100-neuron Izhikevich example (src/main.cpp:131-208):
excitatory and inhibitory connection files izi1.conn / izi2.conn, both
populations a 0.02, b 0.2, c -65, d 2 (here as template population files),
v -65, u -13, every neuron forced to fire at cycles 1, 41 and 100, 341 cycles.
"""
import os

import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200 import netfiles as NF

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ctx(built):
    c = sz.Context(0)
    yield c
    c.close()


def test_izhikevich_example_from_reference_files(ctx, tmp_path):
    for name, size, first in (("exc", 80, 0), ("inh", 20, 80)):
        (tmp_path / f"{name}.pop").write_text(f"# Izhikevich template\n{size}\n{first}\n{name}\n0.02 0.2 -65 2\n-65 -13\n")
    nf = NF.NetworkFiles()
    nf.populations.append(NF.read_population(str(tmp_path / "exc.pop"), L.IZHIKEVICH, template=True))
    nf.populations.append(NF.read_population(str(tmp_path / "inh.pop"), L.IZHIKEVICH, template=True))
    nf.connections.append(NF.read_conn(os.path.join(GOLD, "izi1.conn")))
    nf.connections.append(NF.read_conn(os.path.join(GOLD, "izi2.conn")))
    net = nf.build(ctx, acc_mode=L.ACC_FIXED, graph_chunk=20)
    src, tgt, w, d1 = nf.synapses()
    csr = sz.csr_from_synapses(100, int(d1.max()), src, tgt, w, d1.astype(np.uint32))
    pops = [sz.Pop(sz.IZHIKEVICH, 0, 80, sz.izh_params(0.02, 0.2, -65, 2)),
            sz.Pop(sz.IZHIKEVICH, 80, 100, sz.izh_params(0.02, 0.2, -65, 2))]
    st = [np.full(100, -65, np.float32), np.full(100, -13, np.float32), None, None]
    on = oracle.OracleNet(100, 0, int(d1.max()), pops, csr, state=st)
    steps = 341
    fw = np.zeros((steps, net.words), np.uint32)
    for c in (1, 41, 100):
        fw[c] = sz.ids_to_words(np.arange(100), 100)
    r_gpu = net.run(steps, forced_words=fw)
    r_orc, ev = on.run(steps, forced_words=fw, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(r_gpu, r_orc)
    for k in range(2):
        assert np.array_equal(net.get_state(k), on.state[k])
    assert net.stats()["events"] == ev
    assert int(np.unpackbits(r_gpu.view(np.uint8)).sum()) >= 300
    net.close()
