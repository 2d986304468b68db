"""CPU: the C-ABI library loads, exports every declared symbol, and its host-only
parts (the reference-layout builder) behave like the reference's builders."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L
from tests.helpers import if_network

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(szsnn_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(L.LIB_PATH)
    decl = declared_symbols()
    assert len(decl) > 40
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (szsnn_\w+)", out))
    assert decl <= exported


def test_signatures_cover_declarations(built):
    # every declared entry point has a ctypes signature in the binding
    missing = sorted(declared_symbols() - set(L.SIGNATURES))
    assert not missing, f"no ctypes signature for {missing}"


def test_no_cuda_device_needed_for_layout(built):
    net = if_network(n=1500, n_syn=20000, seed=3)
    params = np.tile(net["pv"][:9], (1500, 1))
    vars_ = np.zeros((1500, 4), np.float32)
    info, arr = sz.build_layout(L.LayoutConsts(1024, 256, 32, 64), 1500, params, vars_, net["src"], net["tgt"],
                                net["w"], net["d1"])
    assert info.neuron_partitions == 2 and info.total_partitions == 2
    assert list(arr[L.L_PARTITION_SIZES]) == [1024, 476]
    # every synapse is in exactly one bundle slot, bundle 0 unused
    tg = arr[L.L_TARGETS].reshape(-1, 32)
    ww = arr[L.L_WEIGHTS].reshape(-1, 32)
    assert not ww[0].any()
    assert np.count_nonzero(ww) == np.count_nonzero(net["w"])
    assert np.isclose(ww.sum(), net["w"].sum(), rtol=1e-5)
    # delay bitmap: bit (delay1 - 1) set for each source (SynapseData.ipp:80-81)
    bits = arr[L.L_DELAY_BITS]
    s0 = net["src"][0]
    assert bits[s0] >> np.uint64(net["d1"][0] - 1) & np.uint64(1)
    # groupPtrs (off, len) entries point into groupMatrix (tp, bundle) pairs
    gp = arr[L.L_GROUP_PTRS].reshape(-1, 2)
    gm = arr[L.L_GROUP_MATRIX].reshape(-1, 2)
    used = gp[gp[:, 1] > 0]
    assert used[:, 1].sum() == info.bundles - 1
    assert np.all(gm[used[:, 0], 1] >= 1)
    assert info.group_pitch >= 1 and info.group_pitch * info.group_step == 256


@pytest.mark.parametrize("bad", ["delay", "target", "inputs"])
def test_layout_limits_raise(built, bad):
    n = 100
    params = np.zeros((n, 9), np.float32)
    vars_ = np.zeros((n, 4), np.float32)
    src, tgt, w, d1 = [0], [1], [1.0], [1]
    kw = {}
    if bad == "delay":
        d1 = [65]  # MAX_SYNAPTIC_DELAY = 64 (uint64 delay bitmap)
    elif bad == "target":
        tgt = [n]
    else:
        kw = dict(input_params=np.zeros((2000, 1), np.float32), input_vars=np.zeros((2000, 1), np.float32))
    with pytest.raises(L.SzsnnError):
        ni = 2000 if bad == "inputs" else 0
        sz.build_layout(L.LayoutConsts(1024, 256, 32, 64), n, params, vars_, src, tgt, w, d1, ni,
                        kw.get("input_params"), kw.get("input_vars"))


def test_csr_bucketing_and_words():
    rp, tg, w = sz.csr_from_synapses(3, 4, [2, 0, 2, 1, 0], [0, 1, 1, 2, 2], [1, 2, 3, 4, 5], [3, 1, 1, 4, 1])
    assert list(rp) == [0, 2, 2, 2, 2, 2, 2, 2, 3, 4, 4, 5, 5]
    assert list(tg) == [1, 2, 2, 1, 0]
    ids = np.array([0, 5, 31, 32, 70])
    assert np.array_equal(sz.words_to_ids(sz.ids_to_words(ids, 80), 80), ids)


def test_cpp_host_builds_and_checks_its_input(built, tmp_path):
    """The C++ host on the kernel seam links against the library alone; input
    errors are reported before any device work."""
    from szsnn_b200.build import REF_HOST
    r = subprocess.run([REF_HOST], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTANETWORKFILE")
    r = subprocess.run([REF_HOST, str(bad), str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "not a network file" in r.stderr
    out = subprocess.run(["ldd", REF_HOST], capture_output=True, text=True).stdout
    assert "libszsnn_cuda.so" in out


def test_reference_driver_rejects_mismatched_layout_constants(built):
    """The drop-in kernels index with the context's layout constants, so a
    layout built with other constants is refused before anything runs."""
    class FakeCtx:
        consts = L.LayoutConsts(1024, 256, 32, 64)

    class FakeBackend:
        ctx = FakeCtx()

    n = 8
    params = np.tile(sz.if_params()[:9], (n, 1))
    vars_ = np.zeros((n, 4), np.float32)
    with pytest.raises(ValueError, match="layout constants"):
        sz.RefSimulation(FakeBackend(), L.LayoutConsts(256, 64, 32, 64), "IF_curr_exp", params, vars_,
                         [0], [1], [0.5], [1])
