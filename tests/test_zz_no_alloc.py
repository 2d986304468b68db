"""GPU: the allocation-free step against the regular network step.

Some callers cannot let a library allocate device memory: hosts that own and
partition all of it (a fixed-budget pool or arena, a framework's caching
allocator), or real-time loops that cannot take cudaMalloc's implicit device
synchronisation.  szsnn_step_static serves them: the caller passes every
buffer and the step's scratch lives in a static device array inside the
library.  This test builds one network, runs two steps in a row through the
regular entry point (szsnn_net_step, scratch allocated by the library) and
through szsnn_step_static (buffers allocated by the test, as such a caller
would), and requires identical spikes and state; the weights are exactly
summable in fp32, so the comparison is bit-exact like the other parity tests.
"""
import ctypes as C

import numpy as np
import pytest

import szsnn_b200 as sz
from szsnn_b200 import _lib as L

pytestmark = pytest.mark.gpu

STATIC_MAX_NEURONS = 262144


class StaticStep(C.Structure):
    _fields_ = [("n_neurons", C.c_int64), ("n_sources", C.c_int64), ("max_delay", C.c_int32),
                ("step", C.c_int64), ("model", C.c_int32), ("flags", C.c_uint32), ("params", C.c_float * 12),
                ("source_p", C.c_float), ("seed", C.c_uint64), ("row_ptr", C.c_void_p), ("syn", C.c_void_p),
                ("state", C.c_void_p * 4), ("ring_cnt", C.c_void_p), ("ring_ids", C.c_void_p),
                ("fired_words", C.c_void_p), ("error_word", C.c_void_p), ("stream", C.c_void_p)]


def _network(n=3000, p=400, D=16, seed=5):
    rng = np.random.default_rng(seed)
    ns = 40 * n
    src = rng.integers(0, n, ns)
    tgt = rng.integers(0, n, ns)
    w = np.where(src < int(0.8 * n), 0.25 * rng.integers(1, 5, ns), -0.5 * rng.integers(1, 3, ns)).astype(np.float32)
    d = rng.integers(1, D + 1, ns)
    psrc = n + np.repeat(np.arange(p), 20)
    ptgt = rng.integers(0, n, 20 * p)
    src = np.concatenate([src, psrc])
    tgt = np.concatenate([tgt, ptgt])
    w = np.concatenate([w, np.full(20 * p, 0.5, np.float32)])
    d = np.concatenate([d, np.ones(20 * p, np.int64)])
    csr = sz.csr_from_synapses(n + p, D, src, tgt, w, d)
    pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=2, tau_syn_E=5, tau_syn_I=10, v_reset=-60,
                      v_thresh=-50)
    v0 = np.concatenate([np.where(rng.random(n) < 0.3, -50.01, rng.uniform(-60, -51, n)), np.zeros(p)])
    st = [v0.astype(np.float32), np.zeros(n + p, np.float32), np.zeros(n + p, np.float32),
          np.concatenate([np.full(n, 1e4), np.zeros(p)]).astype(np.float32)]
    return n, p, D, csr, pv, st


def test_static_step_matches_net_step(ctx):
    n, p, D, csr, pv, st = _network()
    source_p, seed = 0.2, 99
    # regular entry point: the library allocates the step's scratch
    pops = [sz.Pop(sz.IF_CURR_EXP, 0, n, pv), sz.Pop(sz.POISSON, n, n + p, np.array([source_p], np.float32),
                                                  seed=seed)]
    net = sz.Network(ctx, n, p, D, pops, csr=csr, state=st)
    ref_words, ref_state = [], []
    for _ in range(2):
        ref_words.append(net.step())
        ref_state.append([net.get_state(k) for k in range(4)])
    net.close()

    # allocation-free entry point: the caller owns every buffer
    U = n + p
    words = (U + 31) // 32
    syn = np.empty((len(csr[1]), 2), np.int32)
    syn[:, 0] = csr[1]
    syn[:, 1] = csr[2].view(np.int32)
    bufs = dict(row_ptr=ctx.upload(csr[0]), syn=ctx.upload(syn),
                state=[ctx.upload(np.asarray(s, np.float32)) for s in st],
                ring_cnt=ctx.upload(np.zeros(D + 1, np.uint32)), ring_ids=ctx.upload(np.zeros((D + 1) * U, np.int32)),
                fired=ctx.upload(np.zeros(words, np.uint32)), err=ctx.upload(np.zeros(2, np.uint32)))
    lib = L.lib()
    msg = C.create_string_buffer(256)
    for t in range(2):  # two calls in a row share the static scratch
        s = StaticStep()
        s.n_neurons, s.n_sources, s.max_delay, s.step = n, p, D, t
        s.model, s.flags = sz.IF_CURR_EXP, 0
        for i in range(12):
            s.params[i] = float(pv[i])
        s.source_p, s.seed = source_p, seed
        s.row_ptr, s.syn = bufs["row_ptr"].ptr, bufs["syn"].ptr
        for k in range(4):
            s.state[k] = bufs["state"][k].ptr
        s.ring_cnt, s.ring_ids = bufs["ring_cnt"].ptr, bufs["ring_ids"].ptr
        s.fired_words, s.error_word, s.stream = bufs["fired"].ptr, bufs["err"].ptr, ctx.stream
        rc = lib.szsnn_step_static(C.byref(s), msg, 256)
        assert rc == 0, msg.value.decode()
        ctx.sync()
        fired = bufs["fired"].read(np.uint32, words)
        assert np.array_equal(fired, ref_words[t]), f"spikes differ at call {t}"
        for k in range(4):
            assert np.array_equal(bufs["state"][k].read(np.float32, U), ref_state[t][k]), f"state {k} at call {t}"
        assert not bufs["err"].read(np.uint32, 2).any()
    # both calls did real work: spikes at call 0 were delivered at call 1
    assert np.unpackbits(ref_words[0].view(np.uint8)).sum() > 100
    assert np.abs(ref_state[1][1][:n]).sum() > 0
    for b in [bufs["row_ptr"], bufs["syn"], bufs["ring_cnt"], bufs["ring_ids"], bufs["fired"], bufs["err"],
              *bufs["state"]]:
        b.free()


def test_static_step_rejects_oversized_network(built):
    s = StaticStep()
    s.n_neurons, s.n_sources, s.max_delay, s.model = STATIC_MAX_NEURONS + 1, 0, 4, sz.IF_CURR_EXP
    msg = C.create_string_buffer(256)
    rc = L.lib().szsnn_step_static(C.byref(s), msg, 256)
    assert rc == 4  # SZSNN_ERR_LIMIT
    assert b"maximum" in msg.value
