"""CPU: the reference's network-file formats (szsnn_b200.netfiles), against the
reference's own example connection files (tests/golden/izi*.conn, copied from
szsnn1.1/bin by tests/golden/make_golden.py) and crafted cases of the rules
Connection::loadFromFile and Population::loadFrom(Template)File follow."""
import os

import numpy as np
import pytest

from szsnn_b200 import _lib as L
from szsnn_b200 import netfiles as NF

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _data_lines(path):
    with open(path) as f:
        lines = f.read().split("\n")[2:]
    return [ln.split() for ln in lines if ln.strip()]


def test_reference_izi_files():
    c1 = NF.read_conn(os.path.join(GOLD, "izi1.conn"))
    c2 = NF.read_conn(os.path.join(GOLD, "izi2.conn"))
    raw1, raw2 = _data_lines(os.path.join(GOLD, "izi1.conn")), _data_lines(os.path.join(GOLD, "izi2.conn"))
    assert len(c1.src) == len({(r[0], r[1]) for r in raw1}) == len(raw1)
    assert len(c2.src) == len(raw2)
    assert c1.src.max() < 80 and c1.tgt.max() < 100 and np.all(c1.w == np.float32(2e-10))
    assert c2.src.min() >= 80 and c2.src.max() < 100 and np.all(c2.w == np.float32(-0.03))
    assert np.all(c1.delay == 0) and np.all(c2.delay == 0)
    key = c1.src * 1000 + c1.tgt  # ascending (from, to), the map's order
    assert np.all(np.diff(key) > 0)
    first = raw1[0]
    assert (c1.src[0], c1.tgt[0]) == (int(first[0]), int(first[1]))


def test_conn_rules(tmp_path):
    p = tmp_path / "a.conn"
    p.write_text("# h1\n# h2\n3 4 0.5 2\n1 2 0.25 1\n3 4 0.75 5\n2.0 7.0 1e-3 3.0\n\n")
    c = NF.read_conn(str(p), from_start=10, to_start=20)
    assert list(zip(c.src, c.tgt)) == [(1, 2), (2, 7), (3, 4)]
    assert c.w[2] == np.float32(0.75) and c.delay[2] == 5       # a later line for the pair replaces it
    assert (c.from_start, c.to_start) == (10, 20)
    bad = tmp_path / "b.conn"
    bad.write_text("# h1\n# h2\n0 1 0.5 1\n0 2 0.5\n1 1 0.5 1\n")
    with pytest.raises(NF.NetFileError, match="line #4"):
        NF.read_conn(str(bad))
    bad2 = tmp_path / "c.conn"
    bad2.write_text("# h1\n# h2\n0 1 x 1\n")
    with pytest.raises(NF.NetFileError):
        NF.read_conn(str(bad2))


def test_population_files(tmp_path):
    full = tmp_path / "full.pop"
    full.write_text("#\n# two IF_curr_exp neurons\n#\n2\n5\nexc\n"
                    "-65 1 20 0 5 5 0 -70 -50\n-66 0 0 1e4\n"
                    "-64 1 20 0 5 5 0.5 -70 -50\n-60 0 0 1e4\n")
    pf = NF.read_population(str(full), L.IF_CURR_EXP)
    assert (pf.size, pf.first_id, pf.label) == (2, 5, "exc")
    assert pf.params.shape == (9, 2) and pf.vars.shape == (4, 2)
    assert pf.params[6, 1] == np.float32(0.5) and pf.vars[0, 0] == np.float32(-66)
    tmpl = tmp_path / "t.pop"
    tmpl.write_text("# template\n3\n0\nizh\n0.02 0.2 -65 2\n-65 -13\n")
    pt = NF.read_population(str(tmpl), L.IZHIKEVICH, template=True)
    assert pt.params.shape == (4, 3) and np.all(pt.params[2] == -65) and np.all(pt.vars[1] == -13)
    short = tmp_path / "s.pop"
    short.write_text("2\n0\nx\n0.02 0.2 -65 2\n-65 -13\n")
    with pytest.raises(NF.NetFileError, match="not enough data"):
        NF.read_population(str(short), L.IZHIKEVICH)


def test_assembly_offsets_and_delays():
    nf = NF.NetworkFiles()
    nf.populations.append(NF.PopulationFile(L.IZHIKEVICH, 3, 0, "a", np.zeros((4, 3), np.float32),
                                            np.zeros((2, 3), np.float32)))
    nf.populations.append(NF.PopulationFile(L.IZHIKEVICH, 2, 3, "b", np.zeros((4, 2), np.float32),
                                            np.zeros((2, 2), np.float32)))
    nf.inputs.append(NF.PopulationFile(L.CONST_RATE, 2, 0, "in", np.ones((1, 2), np.float32),
                                       np.zeros((1, 2), np.float32)))
    nf.connections.append(NF.Connections(np.array([0, 1]), np.array([1, 0]), np.array([1.0, 2.0], np.float32),
                                         np.array([0, 4]), from_start=3, to_start=0))
    nf.input_connections.append(NF.Connections(np.array([1]), np.array([2]), np.array([3.0], np.float32),
                                               np.array([2]), from_start=0, to_start=2))
    src, tgt, w, d1 = nf.synapses()
    # neuron ids = start + local index; inputs follow the 5 neurons; stored delay = delay + 1
    assert list(src) == [3, 4, 5 + 1] and list(tgt) == [1, 0, 4] and list(d1) == [1, 5, 3]
    assert (nf.n_neurons, nf.n_inputs) == (5, 2)
