"""GPU: the allocation-free step against the regular network step and the oracle.

Some callers cannot let a library allocate device memory: hosts that own and
partition all of it (a fixed-budget pool or arena, a framework's caching
allocator), or real-time loops that cannot take cudaMalloc's implicit device
synchronisation.  szsnn_step_static serves them: the caller passes every
buffer and the step's scratch lives in a static device array inside the
library.

For each neuron model (IF_curr_exp, IF_cond_exp, Izhikevich in two 0.5 ms
half-steps), with and without Poisson sources, one network runs STEPS steps
through the regular entry point (szsnn_net_step, scratch allocated by the
library), through szsnn_step_static (buffers allocated by the test, as such a
caller would; every call shares the static scratch, so consecutive calls
exercise its reuse) and through the CPU oracle.  The delays (1..16) wrap the
ring of the allocation-free step several times.  Weights are exactly summable
in fp32, so spikes and all four state slots must agree bit for bit, like the
other parity tests.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import szsnn_b200 as sz
from szsnn_b200 import _lib as L

pytestmark = pytest.mark.gpu

STATIC_MAX_NEURONS = 262144
STEPS = 40


class StaticStep(C.Structure):
    _fields_ = [("n_neurons", C.c_int64), ("n_sources", C.c_int64), ("max_delay", C.c_int32),
                ("step", C.c_int64), ("model", C.c_int32), ("flags", C.c_uint32), ("params", C.c_float * 12),
                ("source_p", C.c_float), ("seed", C.c_uint64), ("row_ptr", C.c_void_p), ("syn", C.c_void_p),
                ("state", C.c_void_p * 4), ("ring_cnt", C.c_void_p), ("ring_ids", C.c_void_p),
                ("fired_words", C.c_void_p), ("error_word", C.c_void_p), ("stream", C.c_void_p)]


def _network(model, n=3000, p=400, D=16, seed=5):
    """Random network with dyadic weights (every fp32 sum exact in any order)."""
    rng = np.random.default_rng(seed)
    ns = 40 * n
    src = rng.integers(0, n, ns)
    tgt = rng.integers(0, n, ns)
    exc = src < int(0.8 * n)
    flags = 0
    if model == sz.IZHIKEVICH:
        w = np.where(exc, 2.0 * rng.integers(1, 3, ns), -1.0 * rng.integers(1, 3, ns))
        w_src = 8.0
        pv = sz.izh_params(a=0.02, b=0.2, c=-65.0, d=8.0)
        flags = sz.POP_IZH_HALF_STEPS
        v0 = np.where(rng.random(n) < 0.3, 31.0, rng.uniform(-70, -60, n))
        st = [v0, 0.2 * v0, np.zeros(n), np.zeros(n)]
    elif model == sz.IF_COND_EXP:
        w = np.where(exc, 0.0078125 * rng.integers(1, 5, ns), -0.015625 * rng.integers(1, 3, ns))
        w_src = 0.015625
        pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=2, tau_syn_E=5, tau_syn_I=10, v_reset=-60,
                          v_thresh=-50, e_rev_E=0.0, e_rev_I=-80.0)
        v0 = np.where(rng.random(n) < 0.3, -50.01, rng.uniform(-60, -51, n))
        st = [v0, np.zeros(n), np.zeros(n), np.full(n, 1e4)]
    else:
        w = np.where(exc, 0.25 * rng.integers(1, 5, ns), -0.5 * rng.integers(1, 3, ns))
        w_src = 0.5
        pv = sz.if_params(v_rest=-49, cm=1, tau_m=20, tau_refrac=2, tau_syn_E=5, tau_syn_I=10, v_reset=-60,
                          v_thresh=-50)
        v0 = np.where(rng.random(n) < 0.3, -50.01, rng.uniform(-60, -51, n))
        st = [v0, np.zeros(n), np.zeros(n), np.full(n, 1e4)]
    w = w.astype(np.float32)
    d = rng.integers(1, D + 1, ns)
    if p:
        psrc = n + np.repeat(np.arange(p), 20)
        src = np.concatenate([src, psrc])
        tgt = np.concatenate([tgt, rng.integers(0, n, 20 * p)])
        w = np.concatenate([w, np.full(20 * p, w_src, np.float32)])
        d = np.concatenate([d, np.ones(20 * p, np.int64)])
    csr = sz.csr_from_synapses(n + p, D, src, tgt, w, d)
    st = [np.concatenate([np.asarray(s, np.float64), np.zeros(p)]).astype(np.float32) for s in st]
    return n, p, D, csr, pv, flags, st


def _static_run(ctx, model, n, p, D, csr, pv, flags, st, source_p, seed, steps):
    """Run `steps` calls of szsnn_step_static on buffers the test allocates."""
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
    out_words, out_state = [], []
    try:
        for t in range(steps):
            s = StaticStep()
            s.n_neurons, s.n_sources, s.max_delay, s.step = n, p, D, t
            s.model, s.flags = model, flags
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
            out_words.append(bufs["fired"].read(np.uint32, words))
            out_state.append([bufs["state"][k].read(np.float32, U) for k in range(4)])
        err = bufs["err"].read(np.uint32, 2)
    finally:
        for b in [bufs["row_ptr"], bufs["syn"], bufs["ring_cnt"], bufs["ring_ids"], bufs["fired"], bufs["err"],
                  *bufs["state"]]:
            b.free()
    return np.stack(out_words), out_state, err


@pytest.mark.parametrize("p", [400, 0])
@pytest.mark.parametrize("model", [sz.IF_CURR_EXP, sz.IF_COND_EXP, sz.IZHIKEVICH],
                         ids=["if_curr_exp", "if_cond_exp", "izhikevich_half_steps"])
def test_static_step_matches_net_step_and_oracle(ctx, model, p):
    n, p, D, csr, pv, flags, st = _network(model, p=p)
    source_p, seed = 0.2, 99
    pops = [sz.Pop(model, 0, n, pv, flags=flags)]
    if p:
        pops.append(sz.Pop(sz.POISSON, n, n + p, np.array([source_p], np.float32), seed=seed))
    # regular entry point: the library allocates the step's scratch
    net = sz.Network(ctx, n, p, D, pops, csr=csr, state=st)
    ref_words, ref_state = [], []
    for _ in range(STEPS):
        ref_words.append(net.step())
        ref_state.append([net.get_state(k) for k in range(4)])
    net.close()
    ref_words = np.stack(ref_words)

    # allocation-free entry point: the caller owns every buffer
    words, state, err = _static_run(ctx, model, n, p, D, csr, pv, flags, st, source_p, seed, STEPS)
    assert not err.any(), err
    for t in (0, 1):  # two calls in a row against the regular entry point, every state slot
        assert np.array_equal(words[t], ref_words[t]), f"spikes differ at call {t}"
        for k in range(4):
            assert np.array_equal(state[t][k], ref_state[t][k]), f"state {k} at call {t}"
    assert np.array_equal(words, ref_words)
    for k in range(4):
        assert np.array_equal(state[-1][k], ref_state[-1][k]), f"state {k} after {STEPS} calls"

    # the CPU oracle on the same network and inputs
    onet = oracle.OracleNet(n, p, D, pops, csr, state=st)
    r_orc, _ = onet.run(STEPS)
    assert np.array_equal(words, r_orc)
    for k in range(4):
        assert np.array_equal(state[-1][k], onet.state[k]), f"state {k} against the oracle"
    # the run did real work: spikes every few steps, delivered over delays that wrap the ring
    spikes = np.unpackbits(words.view(np.uint8)).sum()
    assert spikes > 200, spikes
    assert np.unpackbits(words[D + 2:].view(np.uint8)).sum() > 0


def test_static_step_requires_error_word(ctx):
    n, p, D, csr, pv, flags, st = _network(sz.IF_CURR_EXP, n=64, p=0)
    s = StaticStep()
    s.n_neurons, s.n_sources, s.max_delay, s.model = n, 0, D, sz.IF_CURR_EXP
    s.row_ptr = s.syn = s.ring_cnt = s.ring_ids = 1  # never dereferenced: the call stops at the argument check
    for k in range(4):
        s.state[k] = 1
    msg = C.create_string_buffer(256)
    rc = L.lib().szsnn_step_static(C.byref(s), msg, 256)
    assert rc == 1  # SZSNN_ERR_ARG
    assert b"error_word" in msg.value


def test_static_step_rejects_oversized_network(built):
    s = StaticStep()
    s.n_neurons, s.n_sources, s.max_delay, s.model = STATIC_MAX_NEURONS + 1, 0, 4, sz.IF_CURR_EXP
    msg = C.create_string_buffer(256)
    rc = L.lib().szsnn_step_static(C.byref(s), msg, 256)
    assert rc == 4  # SZSNN_ERR_LIMIT
    assert b"maximum" in msg.value
