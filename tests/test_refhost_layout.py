"""CPU: the layout restatement (szsnn_layout_build) against the reference's
own builders.

The reference's NetworkGraph, NeuronData, SynapseData, SynapseIndex and
GroupData (compiled unchanged, oracle/_ref/refhost, built from the
reference sources by oracle/refhost/build_refhost.py) build the layout of the
same network on the host; szsnn_layout_build (the library's restatement that
feeds the drop-in kernels) builds it too.  Required equal:
  * partition sizes, neuron and input parameters and variables (SoA per
    partition), bundle targets and weights, the per-neuron delay bitmaps;
  * the scatter tables: for every (partition, neuron, delay) slot the same
    (target partition, bundle) entries -- the reference visits its source
    keys in Boost hash-map order, which permutes groupMatrix rows only;
  * groupPitch, groupStep and the most incoming bundles of a partition.
Skipped when the reference host was not built (no reference checkout)."""
import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200.workloads import izh_network
from tests import refhost
from tests.helpers import if_network


def _compare(tmp_path, small, model, params, vars_, src_ref, src_lib, tgt, w, d1, ni=0, rates=None):
    if not refhost.available(small):
        pytest.skip("reference host not built (oracle/_ref/refhost)")
    mps = 256 if small else 1024
    spec, out = tmp_path / "net.spec", tmp_path / "layout.out"
    rates = np.zeros(0, np.float32) if rates is None else np.asarray(rates, np.float32)
    refhost.write_spec(spec, model, params, vars_, rates, src_ref, tgt, w, np.asarray(d1) - 1, [])
    ref = refhost.run("layout", spec, out, small=small)
    consts = L.LayoutConsts(mps, mps // 4, 32, 64)
    info, arr = sz.build_layout(consts, params.shape[0], params, vars_, src_lib, tgt, w, d1, ni,
                                None if not ni else rates[:, None], None if not ni else np.zeros((ni, 1), np.float32))
    assert np.array_equal(ref["partition_sizes"], arr[L.L_PARTITION_SIZES][: len(ref["partition_sizes"])])
    for name, key in (("neuron_params", L.L_NEURON_PARAMS), ("neuron_vars", L.L_NEURON_VARS),
                      ("targets", L.L_TARGETS), ("weights", L.L_WEIGHTS), ("delay_bits", L.L_DELAY_BITS)):
        assert np.array_equal(ref[name], arr[key]), name
    if ni:
        assert np.array_equal(ref["input_params"], arr[L.L_INPUT_PARAMS])
        assert np.array_equal(ref["input_vars"], arr[L.L_INPUT_VARS])
    assert refhost.group_entries(ref["group_ptrs"], ref["group_matrix"]) == \
        refhost.group_entries(arr[L.L_GROUP_PTRS], arr[L.L_GROUP_MATRIX])
    assert len(ref["group_matrix"]) == len(arr[L.L_GROUP_MATRIX])
    pitch, step, maxb = (int(x) for x in ref["pitch_step_maxbundles"])
    assert (pitch, step, maxb) == (info.group_pitch, info.group_step, info.gq_pitch)
    return ref


@pytest.mark.parametrize("small,n", [(False, 1500), (True, 700)])
def test_layout_if_curr_exp_equals_reference_builders(tmp_path, small, n):
    net = if_network(n=n, n_syn=20 * n, dyadic=False, seed=13)
    params = np.tile(net["pv"][:9], (n, 1)).astype(np.float32)
    params[:, 8] += np.linspace(0, 1, n, dtype=np.float32)  # per-neuron thresholds
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 1e4)], 1).astype(np.float32)
    ref = _compare(tmp_path, small, 0, params, vars_, net["src"], net["src"], net["tgt"], net["w"], net["d1"])
    assert len(ref["targets"]) >= 20 * n


def test_layout_izhikevich_1000_equals_reference_builders(tmp_path):
    net = izh_network(n=1000, seed=4)
    params = np.stack([net["a"], net["b"], net["c"], net["d"]], 1).astype(np.float32)
    vars_ = np.stack([net["v0"], net["u0"]], 1).astype(np.float32)
    _compare(tmp_path, False, 1, params, vars_, net["src"], net["src"], net["tgt"], net["w"], net["d1"])


def test_layout_with_input_partition_equals_reference_builders(tmp_path):
    rng = np.random.default_rng(9)
    n, ni = 300, 40
    net = if_network(n=n, n_syn=5000, dyadic=True, seed=2)
    in_base = -(-n // 256) * 256
    j = rng.integers(0, ni, 800)
    src_lib = np.concatenate([net["src"], in_base + j])
    src_ref = np.concatenate([net["src"], n + j])
    tgt = np.concatenate([net["tgt"], rng.integers(0, n, 800)])
    w = np.concatenate([net["w"], np.full(800, 0.75, np.float32)])
    d1 = np.concatenate([net["d1"], rng.integers(1, 10, 800).astype(np.uint32)])
    params = np.tile(net["pv"][:9], (n, 1)).astype(np.float32)
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 1e4)], 1).astype(np.float32)
    rates = rng.integers(3, 12, ni).astype(np.float32)
    _compare(tmp_path, True, 0, params, vars_, src_ref, src_lib, tgt, w, d1, ni=ni, rates=rates)
