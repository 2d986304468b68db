"""GPU: batched sweeps -- one block-diagonal launch of many uneven networks.

  * every net of a batch produces exactly the spikes it produces alone through
    the plain path (fixed-point accumulation: bit-reproducible sums);
  * the batch equals the oracle run over the same layout;
  * the autotuner's launch shape leaves results bit-identical.
"""
import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200 import batch as B
from szsnn_b200.autotune import tune

pytestmark = pytest.mark.gpu


def _ids_in(ids, lo, hi, base):
    sel = ids[(ids >= lo) & (ids < hi)]
    return sel - lo + base


def test_batched_equals_looped(ctx):
    specs = B.sweep_specs(12, seed=3, n_min=200, n_max=3000)
    steps = 200
    bt = B.Batch(ctx, specs, acc_mode=L.ACC_FIXED, graph_chunk=50)
    lay = bt.layout
    ras_b = bt.net.run(steps)
    spikes_b = bt.spikes_per_net()
    U = bt.net.U
    total = 0
    for i, spec in enumerate(specs):
        net = B.single_network(ctx, spec, acc_mode=L.ACC_FIXED, graph_chunk=50)
        ras_s = net.run(steps)
        assert net.group_spikes()[0] == spikes_b[i]
        a, b = int(lay["n_off"][i]), int(lay["n_off"][i + 1])
        pa, pb = int(lay["p_off"][i]), int(lay["p_off"][i + 1])
        for t in range(0, steps, 7):
            g = sz.words_to_ids(ras_b[t], U)
            mine = np.concatenate([_ids_in(g, a, b, 0), _ids_in(g, pa, pb, spec.n)])
            assert np.array_equal(mine, sz.words_to_ids(ras_s[t], net.U)), (i, t)
        total += int(spikes_b[i])
        net.close()
    assert total > 1000
    bt.close()


def test_batch_equals_oracle(ctx):
    specs = B.sweep_specs(6, seed=5, n_min=200, n_max=1500)
    bt = B.Batch(ctx, specs, acc_mode=L.ACC_FIXED, graph_chunk=40)
    lay = bt.layout
    U = lay["N"] + lay["P"]
    csr = oracle.generate(lay["blocks"], 12345, U, lay["D"])
    on = oracle.OracleNet(lay["N"], lay["P"], lay["D"], lay["pops"], csr, state=lay["state"])
    r_gpu = bt.net.run(150)
    r_orc, ev = on.run(150, acc_mode=oracle.ACC_FIXED)
    assert np.array_equal(r_gpu, r_orc)
    for k in range(2):
        assert np.array_equal(bt.net.get_state(k), on.state[k])
    assert bt.net.stats()["events"] == ev
    bt.close()


def test_autotune_keeps_results(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("SZSNN_TUNE_CACHE", str(tmp_path / "tune.json"))
    specs = B.sweep_specs(10, seed=7, n_min=500, n_max=4000)
    ref = B.Batch(ctx, specs, acc_mode=L.ACC_FIXED)
    r_ref = ref.net.run(120)
    ref.close()
    bt = B.Batch(ctx, specs, acc_mode=L.ACC_FIXED)
    choice = tune(bt.net, replays=5)
    assert choice["update_block"] in (64, 128, 256) and not choice["cached"]
    assert tune(bt.net, replays=5)["cached"]  # same device, same workload shape
    # the tuning replays ran on scratch state: the simulation still starts at step 0
    assert bt.net.stats()["steps_done"] == 0
    r = bt.net.run(120)
    assert np.array_equal(r, r_ref)
    bt.close()
