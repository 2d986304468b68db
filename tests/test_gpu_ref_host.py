"""GPU: the C++ host on the drop-in kernel seam (szsnn_b200/szsnn_ref_host, built
from csrc/ref_host.cpp against the C ABI alone) makes the reference
Simulation's call sequence: same spikes every cycle and the same final neuron
state as the Python driver of the same kernels (szsnn_b200.refsim, itself
checked against the reference's own kernels in test_gpu_parity.py)."""
import os
import struct
import subprocess

import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from szsnn_b200.build import REF_HOST
from tests.helpers import forced_schedule, if_network

pytestmark = pytest.mark.gpu


def _write_net(path, model, mps, tpg, D, params, vars_, src, tgt, w, d1, steps, sched):
    n, pc = params.shape
    vc = vars_.shape[1]
    forced = [(t, ids) for t, ids in enumerate(sched) if ids is not None and len(ids)]
    with open(path, "wb") as f:
        f.write(b"SZRH0001")
        f.write(struct.pack("<9I", model, mps, tpg, D, n, pc, vc, steps, len(forced)))
        f.write(struct.pack("<Q", len(src)))
        for a, dt in ((params, np.float32), (vars_, np.float32), (src, np.uint32), (tgt, np.uint32),
                      (w, np.float32), (d1, np.uint32)):
            f.write(np.ascontiguousarray(a, dtype=dt).tobytes())
        for t, ids in forced:
            f.write(struct.pack("<2I", t, len(ids)))
            f.write(np.asarray(ids, np.uint32).tobytes())


def _read_out(path, steps, vc, n):
    data = open(path, "rb").read()
    off, spikes = 0, []
    for _ in range(steps):
        (cnt,) = struct.unpack_from("<I", data, off)
        off += 4
        spikes.append(np.frombuffer(data, np.uint32, cnt, off).astype(np.int64))
        off += 4 * cnt
    vars_ = np.frombuffer(data, np.float32, vc * n, off).reshape(vc, n)
    return spikes, vars_


@pytest.mark.parametrize("mps,n", [(256, 700), (1024, 3000)])
def test_cpp_host_equals_python_driver(built, tmp_path, mps, n):
    assert os.path.exists(REF_HOST), "szsnn_ref_host is built with the library"
    net = if_network(n=n, n_syn=20 * n, dyadic=True, seed=23)
    params = np.tile(net["pv"][:9], (n, 1)).astype(np.float32)
    vars_ = np.stack([net["v0"], np.zeros(n), np.zeros(n), np.full(n, 10000.0)], 1).astype(np.float32)
    steps = 200
    sched = forced_schedule(n, steps)
    tpg = mps // 4
    fin, fout = str(tmp_path / "net.bin"), str(tmp_path / "out.bin")
    _write_net(fin, L.IF_CURR_EXP, mps, tpg, 64, params, vars_, net["src"], net["tgt"], net["w"], net["d1"],
               steps, sched)
    r = subprocess.run([REF_HOST, fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    spikes_cpp, vars_cpp = _read_out(fout, steps, 4, n)
    ctx = sz.Context(0, max_partition_size=mps, threads_per_group=tpg, warp_size=32, max_synaptic_delay=64)
    sim = sz.RefSimulation(sz.CudaRefBackend(ctx), L.LayoutConsts(mps, tpg, 32, 64), "IF_curr_exp", params, vars_,
                           net["src"], net["tgt"], net["w"], net["d1"])
    total = 0
    for t in range(steps):
        ids = sim.step_and_fired(sched[t])
        total += len(ids)
        assert np.array_equal(ids, spikes_cpp[t]), f"cycle {t}"
    assert total > 500
    assert np.array_equal(sim.neuron_vars(), vars_cpp)
    ctx.sync()
    ctx.close()
