"""Batched sweeps: many independent networks of uneven size in one launch per phase.

No reference counterpart (the reference simulates one network per Simulation,
szsnn1.1/src/Simulation.hpp:38-132).  A batch is laid out as one
block-diagonal network on the device:

  neurons of net 0 | neurons of net 1 | ... | sources of net 0 | sources of net 1 | ...

Every net keeps its own populations (parameter sets), its own synapse rows
(targets only inside the net), its own Poisson streams (keyed by the index
inside the population, so a net draws the same spikes alone or in a batch) and
its own per-delay spike queue entries in the shared device ring.  One step of
the whole batch is one propagate and one update launch; steps run in CUDA
graphs of `graph_chunk` steps; a per-unit group map gives spikes per net.
The looped baseline runs each net alone through the same plain path.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .models import fold_dt, if_params, izh_params
from .network import GenBlock, Network, Pop


@dataclass
class NetSpec:
    model: int           # IF_CURR_EXP or IZHIKEVICH
    n: int               # neurons (80 % excitatory)
    fanout: int          # recurrent synapses per neuron
    d_max: int           # delays U{1..d_max} steps
    w_scale: float       # multiplies the base weights
    rate_hz: float       # Poisson drive rate
    seed: int
    n_sources: int = 0   # 0 -> n // 10 Poisson sources, 100 targets each


def sweep_specs(n_nets: int = 512, seed: int = 0, n_min: int = 200, n_max: int = 20000, fanout: int = 100,
                d_max: int = 20) -> list[NetSpec]:
    """The batched-sweep workload: N_i log-uniform in [n_min, n_max], weight
    scale linear 0.5..2.0, Poisson rate linear 5..20 Hz, IF_curr_exp for even
    i and Izhikevich for odd i, seed i."""
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_nets))).astype(int)
    specs = []
    for i in range(n_nets):
        f = i / max(n_nets - 1, 1)
        specs.append(NetSpec(L.IF_CURR_EXP if i % 2 == 0 else L.IZHIKEVICH, int(ns[i]), fanout, d_max,
                             0.5 + 1.5 * f, 5.0 + 15.0 * f, i))
    return specs


DT_MS = 1.0
# IF_curr_exp at dt = 1 ms with the 4000-neuron configuration's parameters;
# Izhikevich regular-spiking / fast-spiking parameter rules of the pulse-coupled network.
IF_PARAMS = fold_dt(if_params(v_rest=-60, cm=0.2, tau_m=20, tau_refrac=5, tau_syn_E=5, tau_syn_I=10, v_reset=-60,
                              v_thresh=-50), DT_MS)
BASE_W = {L.IF_CURR_EXP: (0.25, -2.25), L.IZHIKEVICH: (6.0, -5.0)}


def _izh_per_unit(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(10_000 + seed)
    ne = int(0.8 * n)
    re = rng.uniform(0, 1, ne).astype(np.float32)
    ri = rng.uniform(0, 1, n - ne).astype(np.float32)
    pn = np.zeros((12, n), np.float32)
    pn[0] = np.concatenate([np.full(ne, 0.02), 0.02 + 0.08 * ri])
    pn[1] = np.concatenate([np.full(ne, 0.2), 0.25 - 0.05 * ri])
    pn[2] = np.concatenate([-65 + 15 * re ** 2, np.full(n - ne, -65.0)])
    pn[3] = np.concatenate([8 - 6 * re ** 2, np.full(n - ne, 2.0)])
    return pn


def _initial(spec: NetSpec, p_count: int):
    rng = np.random.default_rng(20_000 + spec.seed)
    n = spec.n
    st = [np.zeros(n + p_count, np.float32) for _ in range(4)]
    if spec.model == L.IF_CURR_EXP:
        st[0][:n] = rng.uniform(-60, -50, n)
        st[3][:n] = 1e4
    else:
        pn = _izh_per_unit(n, spec.seed)
        st[0][:n] = -65.0
        st[1][:n] = pn[1] * -65.0
    return st


def layout(specs: list[NetSpec]):
    """Populations, generator blocks, initial state and group map of the batch."""
    nn = np.array([s.n for s in specs], np.int64)
    pp = np.array([s.n_sources or max(s.n // 10, 1) for s in specs], np.int64)
    n_off = np.concatenate([[0], np.cumsum(nn)])
    N = int(n_off[-1])
    p_off = N + np.concatenate([[0], np.cumsum(pp)])
    U = int(p_off[-1])
    D = max(s.d_max for s in specs)
    pops, blocks_n, blocks_p = [], [], []
    state = [np.zeros(U, np.float32) for _ in range(4)]
    group = np.zeros(U, np.int32)
    for i, s in enumerate(specs):
        a, b = int(n_off[i]), int(n_off[i + 1])
        pa, pb = int(p_off[i]), int(p_off[i + 1])
        ne = int(0.8 * s.n)
        if s.model == L.IF_CURR_EXP:
            pops.append(Pop(L.IF_CURR_EXP, a, b, IF_PARAMS))
        else:
            pops.append(Pop(L.IZHIKEVICH, a, b, np.zeros(12, np.float32), per_unit=_izh_per_unit(s.n, s.seed)))
        we, wi = BASE_W[s.model]
        we, wi = np.float32(we * s.w_scale), np.float32(wi * s.w_scale)
        blocks_n.append(GenBlock(a, ne, a, s.n, s.fanout, float(we), float(we), 1.0, 1, s.d_max, True, 4 * s.seed))
        blocks_n.append(GenBlock(a + ne, s.n - ne, a, s.n, s.fanout, float(-wi), float(-wi), -1.0, 1, s.d_max, True,
                                 4 * s.seed + 1))
        blocks_p.append(GenBlock(pa, pb - pa, a, s.n, 100, float(we), float(we), 1.0, 1, 1, False, 4 * s.seed + 2))
        st = _initial(s, pb - pa)
        for k in range(4):
            state[k][a:b] = st[k][: s.n]
        group[a:b] = i
        group[pa:pb] = i
    for i, s in enumerate(specs):
        pa, pb = int(p_off[i]), int(p_off[i + 1])
        pops.append(Pop(L.POISSON, pa, pb, np.array([s.rate_hz * DT_MS * 1e-3], np.float32), seed=1000 + s.seed))
    pops.sort(key=lambda p: p.begin)
    return dict(N=N, P=U - N, D=D, pops=pops, blocks=blocks_n + blocks_p, state=state, group=group,
                n_off=n_off, p_off=p_off)


class Batch:
    """All nets of `specs` as one device network.  tune=True tunes at
    construction (step 0); tuning after a warm-up (autotune.tune on .net) sees
    the network's working event rate."""

    def __init__(self, ctx, specs: list[NetSpec], acc_mode: int = L.ACC_FLOAT, graph_chunk: int = 100,
                 gen_seed: int = 12345, tune: bool = False):
        self.specs = specs
        lay = layout(specs)
        self.layout = lay
        self.net = Network(ctx, lay["N"], lay["P"], lay["D"], lay["pops"], state=lay["state"], acc_mode=acc_mode,
                           graph_chunk=graph_chunk, groups=lay["group"], n_groups=len(specs))
        self.net.generate(lay["blocks"], gen_seed)
        if tune:
            from .autotune import tune as _tune
            _tune(self.net)

    def run(self, steps: int) -> None:
        self.net.run_device(steps)

    def spikes_per_net(self, reset: bool = False) -> np.ndarray:
        return self.net.group_spikes(reset)

    def close(self):
        self.net.close()


def single_network(ctx, spec: NetSpec, acc_mode: int = L.ACC_FLOAT, graph_chunk: int = 100,
                   gen_seed: int = 12345) -> Network:
    """One net of the sweep on its own (the looped plain path); same streams as in a batch."""
    lay = layout([spec])
    net = Network(ctx, lay["N"], lay["P"], lay["D"], lay["pops"], state=lay["state"], acc_mode=acc_mode,
                  graph_chunk=graph_chunk, groups=lay["group"], n_groups=1)
    net.generate(lay["blocks"], gen_seed)
    return net


def compare_batched_looped(ctx, specs: list[NetSpec], steps: int = 1000, acc_mode: int = L.ACC_FLOAT,
                           graph_chunk: int = 100, tune: bool = True, gen_seed: int = 12345,
                           warmup: int | None = None, tune_loop: bool = True) -> dict:
    """nets/s of one batched run against the plain path looped per net.

    Both sides are timed on the device (CUDA events on the launching stream)
    from the first step to the last, networks already built on the device;
    the looped side is the sum over nets.  Wall-clock times (with a device
    synchronisation at each end) are reported beside them.  The loop runs
    twice: each net in the default launch shape, and (tune_loop) each net in
    the shape the same autotuner picks for it after the same warm-up, tuned
    once per workload bucket (size, delays, event rate) and shared by the
    nets of that bucket."""
    batch = Batch(ctx, specs, acc_mode, graph_chunk, gen_seed)
    warm = warmup if warmup is not None else 3 * graph_chunk
    batch.run(warm)  # graph instantiation and initial transient outside the timed region
    ctx.sync()
    if tune:  # on the warmed-up network: replays of a representative step
        from .autotune import tune as _tune
        _tune(batch.net, replays=20)
        batch.run(graph_chunk)  # graphs of the chosen shape
        ctx.sync()
    batch.spikes_per_net(reset=True)
    t0 = time.perf_counter()
    batch.run(steps)
    ctx.sync()
    w_batch = time.perf_counter() - t0
    t_batch = batch.net.device_ms() / 1e3
    s_batch = batch.spikes_per_net()
    st = batch.net.stats()
    batch.close()
    t_loop = 0.0
    w_loop = 0.0
    s_loop = np.zeros(len(specs), np.uint64)
    for i, spec in enumerate(specs):
        net = single_network(ctx, spec, acc_mode, graph_chunk, gen_seed)
        net.run_device(warm + (graph_chunk if tune else 0))  # same warm-up as the batch
        ctx.sync()
        net.group_spikes(reset=True)
        t0 = time.perf_counter()
        net.run_device(steps)
        ctx.sync()
        w_loop += time.perf_counter() - t0
        t_loop += net.device_ms() / 1e3
        s_loop[i] = net.group_spikes()[0]
        net.close()
    out = dict(nets=len(specs), steps=steps, batched_s=t_batch, looped_s=t_loop,
               batched_nets_per_s=len(specs) / t_batch, looped_nets_per_s=len(specs) / t_loop,
               speedup=t_loop / t_batch, wall_batched_s=w_batch, wall_looped_s=w_loop,
               neurons=int(sum(s.n for s in specs)),
               synapses=int(batch.net.n_synapses), spikes_batched=s_batch, spikes_looped=s_loop,
               events_batched=int(st["events"]))
    if tune_loop:
        from .autotune import tune as _tune
        shared: dict = {}
        t_tuned = 0.0
        s_tuned = np.zeros(len(specs), np.uint64)
        for i, spec in enumerate(specs):
            net = single_network(ctx, spec, acc_mode, graph_chunk, gen_seed)
            net.run_device(warm)
            ctx.sync()
            _tune(net, replays=20, cache=shared)
            net.run_device(graph_chunk)  # graphs of the chosen shape; the batch's warm-up length
            ctx.sync()
            net.group_spikes(reset=True)
            net.run_device(steps)
            ctx.sync()
            t_tuned += net.device_ms() / 1e3
            s_tuned[i] = net.group_spikes()[0]
            net.close()
        out.update(looped_tuned_s=t_tuned, looped_tuned_nets_per_s=len(specs) / t_tuned,
                   speedup_vs_tuned_loop=t_tuned / t_batch, spikes_looped_tuned=s_tuned,
                   loop_tuning={"buckets": len(shared), "shapes": sorted({(c["overlap"], c["mode"], c["group"],
                                                                            c["blocks"], c["update_block"])
                                                                           for c in shared.values()})})
    return out


def _main(argv=None) -> None:
    """Run a batched sweep from the command line:
    python -m szsnn_b200.batch [--nets N] [--every K] [--steps S] [--warmup W]
                               [--shape order,mode,group,blocks,update_block | --tune]
    --every K keeps every K-th net of the 512-net sweep (a smaller batch of the same mix)."""
    import argparse
    import json

    from .context import Context

    ap = argparse.ArgumentParser(prog="python -m szsnn_b200.batch")
    ap.add_argument("--nets", type=int, default=512)
    ap.add_argument("--every", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=300)
    ap.add_argument("--shape", default=None)
    ap.add_argument("--tune", action="store_true")
    a = ap.parse_args(argv)
    ctx = Context(0)
    specs = sweep_specs(a.nets, seed=0)[:: a.every]
    bt = Batch(ctx, specs)
    if a.shape:
        order, mode, group, blocks, ub = a.shape.split(",")
        bt.net.set_overlap(order == "overlapped")
        bt.net.set_tuning(int(mode), int(group), int(blocks), int(ub))
    bt.run(a.warmup)
    ctx.sync()
    choice = None
    if a.tune:
        from .autotune import tune as _tune
        choice = {k: v for k, v in _tune(bt.net).items() if k != "trials"}
    s0 = bt.net.stats()
    bt.run(a.steps)
    ctx.sync()
    s1 = bt.net.stats()
    ms = bt.net.device_ms()
    print(json.dumps({"nets": len(specs), "units": bt.net.U, "synapses": bt.net.n_synapses, "steps": a.steps,
                      "device_ms": ms, "events_per_step": (s1["events"] - s0["events"]) / max(a.steps, 1),
                      "nets_per_s": len(specs) / (ms / 1e3), "tuning": choice}))
    bt.close()
    ctx.close()


if __name__ == "__main__":
    _main()
