#!/usr/bin/env python
"""Benchmark: synaptic events/s of the 1M-neuron IF_cond_exp network on B200.

Workload (the large IF_cond_exp configuration, szsnn_b200.workloads.cond_config):
1,000,000 IF_cond_exp neurons (800k excitatory / 200k inhibitory), 1000 random
synapses per neuron (1e9 synapses; targets uniform without self-loops; weights
exc ~U(0,4) nS, inh ~U(0,51) nS stored negative; delays U{1..64} steps),
e_rev_E 0, e_rev_I -80 mV, tau_syn_E 5, tau_syn_I 10 ms, dt 0.1 ms, 100,000
Poisson inputs at 5 Hz with 100 targets each, fp32 state.  Parameters the
configuration leaves open are taken from the 4000-neuron IF_curr_exp
configuration (tau_m 20 ms, cm 0.2 nF, v_rest -60, v_thresh -50, v_reset
-60 mV, tau_refrac 5 ms); Poisson synapses ~U(0,100) nS with delay 1 step;
v(0) ~ U(-60,-50) mV.  Conductances in uS.

Timing.  `--steps K` timed steps, `--warmup W` warm-up steps; one step is S
simulation time steps (propagate + update), S = ceil(20,000 / K) on the GPU
(ceil(2000 / K) in the CPU reference arm), so every timed region covers at
least 20,000 (2000) simulation steps.  `ms_per_step` is per SIMULATION step;
the timed region is steps x sim_steps_per_step of them.  The network is built
on the device by the fixed fan-out generator; inputs are larger than L2 (8 GB
synapse table), and the per-neuron state (16 MB) stays L2-resident across
steps as it does in any run of this network.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun (N > 1) each rank runs an independent replica (the path does not
shard: replicas only), value = all ranks' events / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "syn-events/s @1M IF_cond_exp"
UNIT = "syn-events/s"
DT_MS = 0.1
GPU_SIM_STEPS = 20_000   # least simulation steps in the GPU arm's timed region
REF_SIM_STEPS = 2_000    # least simulation steps in the CPU reference arm's timed region
CPU_WARM_STEPS = 500     # oracle warm-up simulation steps (past the v(0) volley and its echo)
CPU_TIMED_STEPS = 200    # simulation steps timed by the cpu_baseline leg
BYTES_PER_EVENT = 8      # int32 target + fp32 weight, delay implied by the bucket
BYTES_PER_NEURON = 48    # 16 B state read + 16 B write + 8 B input read + 8 B clear
# k_step of the benchmark network itself (1M x 1000, fp32, the tuned shape), L2 left warm as in the
# timed run (ncu --cache-control none, one-pass DRAM counters, mean of three launches in the timed
# region): 3.88 MB per launch, about the ~500k synapses the step delivers; the neuron state, ring and
# bucket index stay in L2
NCU_STEP_TRAFFIC_WARM = 3_882_752


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--neurons", type=int, default=1_000_000)
    ap.add_argument("--fanout", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--acc", default="float", choices=["float", "fixed"])
    ap.add_argument("--sim-steps", type=int, default=None,
                    help="least simulation steps in the timed region (default 20000 on the GPU, 2000 in the "
                         "reference arm); one timed step is ceil(this / --steps) simulation steps")
    ap.add_argument("--classic", dest="overlap", action="store_false",
                    help="propagate-then-update order (two launches per step) instead of the overlapped one")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep the default launch shape instead of autotuning after the warm-up")
    ap.add_argument("--tune-after", type=int, default=3000, help="steps simulated before the tuner's replays")
    ap.add_argument("--live-shapes", type=int, default=4,
                    help="the tuner's best overlapped shapes (by replay time) timed live; the fastest is kept")
    ap.add_argument("--shape", default=None,
                    help="fixed launch shape 'order,mode,group,blocks,update_block[,tiles,per_sm]' (order: "
                         "overlapped|classic; tiles 0 block tiles, 1 persistent warp tiles with per_sm update "
                         "blocks per SM) instead of the tuner")
    ap.add_argument("--resident", default="auto", choices=["auto", "on", "off"],
                    help="resident stepping (one cooperative launch per 100-step chunk, neuron state in shared "
                         "memory): auto keeps it when its live step time beats the tuned graphs'")
    ap.add_argument("--resident-warps", default="12,16,20,24",
                    help="update warps per block the resident choice tries")
    ap.add_argument("--e2e-steps", type=int, default=5000,
                    help="simulation steps of the end-to-end run (host input words in, raster out, every step)")
    ap.add_argument("--profile-steps", type=int, default=200)
    ap.add_argument("--cpu-neurons", type=int, default=None,
                    help="neurons of the network the CPU port runs (default: the benchmark's own --neurons)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the 1000-neuron and 4000-neuron configurations")
    ap.add_argument("--no-secondary", action="store_true", help="skip the batched-sweep and BPTT measurements")
    ap.add_argument("--batch-nets", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=1000)
    ap.add_argument("--bptt-scale", type=float, default=1.0)
    ap.add_argument("--bptt-steps", type=int, default=500)
    ap.add_argument("--bptt-trajectory", default="auto", choices=["auto", "keep", "recompute"],
                    help="keep the forward's membrane trajectory for the backward, or recompute it from checkpoints")
    return ap.parse_args(argv)


def sim_steps_per_step(k: int, least: int) -> int:
    """S: simulation steps in one timed step so that k of them cover `least`."""
    return max(1, -(-least // max(1, k)))


def cond_config(n: int, fanout: int):
    from szsnn_b200.workloads import cond_config as cc
    return cc(n, fanout)


def init_state(n, p, seed):
    from szsnn_b200.workloads import init_state as ist
    return ist(n, p, seed)


def headline_config(n, p, D, n_syn, acc):
    """The workload description both arms report (identical keys and values
    when both run the same network)."""
    return {"workload": "IF_cond_exp 1M neurons x 1000 synapses (1e9), 100k Poisson x 100, "
                        "delays U{1..64} steps, dt 0.1 ms",
            "neurons": n, "sources": p, "synapses": int(n_syn), "max_delay": D, "accumulation": acc,
            "l2": "inputs larger than L2 (8 GB synapse table); neuron state L2-resident across steps"}


class ClockSampler:
    """SM clocks, power and throttle reasons sampled during the timed region
    (NVML, read-only, every 20 ms; nvidia-smi every 100 ms when NVML is not
    importable).  The device is found by the CUDA device's UUID."""

    HW, HW_THERMAL, SW_THERMAL, SW_POWER = 0x8, 0x40, 0x20, 0x4

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self._stop = threading.Event()
        self._t = None
        self._nv = None
        self._h = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            for cand in (uuid, "GPU-" + uuid):
                try:
                    self._h = nv.nvmlDeviceGetHandleByUUID(cand)
                    break
                except Exception:
                    continue
            if self._h is None:
                self._h = nv.nvmlDeviceGetHandleByIndex(index)
            self._nv = nv
        except Exception:
            self._nv = None

    def _sample_nvml(self):
        nv, h = self._nv, self._h
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        return float(sm), float(mx), int(rs)

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=5)
        f = [x.strip() for x in out.stdout.strip().splitlines()[0].split(",")]
        bits = 0
        for flag, v in zip((self.HW, self.HW_THERMAL, self.SW_THERMAL, self.SW_POWER), f[2:6]):
            if v.lower() in ("active", "1"):
                bits |= flag
        return float(f[0]), float(f[1]), bits

    def _run(self):
        period = 0.02 if self._nv else 0.1
        while not self._stop.is_set():
            try:
                self.samples.append(self._sample_nvml() if self._nv else self._sample_smi())
            except Exception:
                pass
            self._stop.wait(period)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [s[0] for s in self.samples]
        names = {self.HW: "hw_slowdown", self.HW_THERMAL: "hw_thermal_slowdown",
                 self.SW_THERMAL: "sw_thermal_slowdown", self.SW_POWER: "sw_power_cap"}
        reasons = sorted({nm for s in self.samples for bit, nm in names.items() if s[2] & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "samples": len(self.samples), "source": "nvml" if self._nv else "nvidia-smi"}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def pinned_words(steps, words):
    """uint32 [steps, words] in page-locked host memory (torch's pinned allocator)."""
    import torch
    return torch.empty((steps, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)


def cpu_port_measure(n, fanout, seed, warm, timed, threads=None):
    """The oracle port of the reference's step on the benchmark network of n
    neurons (all host threads): generated with the GPU generator's algorithm
    and seed, `warm` untimed simulation steps, then `timed` timed ones.
    Returns (events/s, events, seconds, description)."""
    import oracle

    threads = threads or os.cpu_count() or 1
    n, p, D, blocks, pops = cond_config(n, fanout)
    t0 = time.perf_counter()
    csr = oracle.generate(blocks, seed, n + p, D)
    gen_s = time.perf_counter() - t0
    on = oracle.OracleNet(n, p, D, pops, csr, state=init_state(n, p, seed))
    on.run(warm, nthreads=threads)
    t0 = time.perf_counter()
    _, ev = on.run(timed, nthreads=threads)
    dt = time.perf_counter() - t0
    desc = (f"{n} IF_cond_exp neurons x {fanout} synapses + {p} Poisson x 100 (the benchmark network, same "
            f"generator and seed); {timed} simulation steps timed after {warm} warm-up steps; {ev} events in "
            f"{dt:.2f} s on {threads} threads (generation {gen_s:.1f} s, untimed)")
    del on, csr
    return ev / dt, ev, dt, desc, threads


def cpu_baseline(args):
    """The oracle port on the benchmark network itself: 500 warm-up and 200
    timed simulation steps (the reference arm's procedure, shorter)."""
    n = args.cpu_neurons or args.neurons
    v, ev, dt, desc, threads = cpu_port_measure(n, args.fanout, args.seed, CPU_WARM_STEPS, CPU_TIMED_STEPS)
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
            "same_network": n == args.neurons}


def bench_configs(ctx, args):
    """The 1000-neuron Izhikevich and 4000-neuron IF_curr_exp configurations:
    syn-events/s, neuron-updates/s and device time per 1000 simulation steps
    (the reference's published unit) on the GPU, with CPU baselines in the
    same run: the reference's own kernels under the work-group emulator
    (Oracle B, one host thread: the emulator runs work-groups in turn) on a
    bounded sample, and the oracle port on all host threads."""
    import oracle
    import szsnn_b200 as sz
    from szsnn_b200 import workloads as WL

    hbm, _ = peaks()
    out = {}

    def gpu_run(net, steps, n_units, bytes_per_unit, current_ptr=None):
        net.run_device(steps, current_ptr=current_ptr)  # warm-up: graphs, transient
        ctx.sync()
        s0 = net.stats()
        net.run_device(steps, current_ptr=current_ptr)
        ctx.sync()
        ms = net.device_ms()
        s1 = net.stats()
        ev = s1["events"] - s0["events"]
        us = ms / steps * 1e3
        return {"syn_events_per_s": ev / (ms * 1e-3), "neuron_updates_per_s": n_units * steps / (ms * 1e-3),
                "ms_per_1000_steps": ms / steps * 1000.0, "us_per_step": us, "steps": steps,
                "events_per_step": ev / steps,
                "roofline_hbm_frac": (n_units * bytes_per_unit + ev / steps * BYTES_PER_EVENT) / (us * 1e-6) / 1e9
                / hbm,
                "bound": "launch and latency: one fused kernel per step over a few thousand units"}

    def best_run(net, steps, n_units, bytes_per_unit, current_ptr=None):
        """The per-step graphs at the default and at the tuned launch shape,
        then resident stepping (one cooperative launch per 100 steps) at a few
        grid sizes; the fastest is reported as `gpu`, every timing beside it."""
        runs = {"graphs_default_shape": gpu_run(net, steps, n_units, bytes_per_unit, current_ptr)}
        from szsnn_b200.autotune import tune
        ch = tune(net, replays=50, use_cache=False)  # order and launch shape on replays of the warmed-up step
        live = refine_live(net, ctx, ch, 4, current_ptr=current_ptr) if ch["overlap"] else None
        runs["graphs_tuned"] = gpu_run(net, steps, n_units, bytes_per_unit, current_ptr)
        runs["graphs_tuned"]["shape"] = live["chosen"] if live else {
            k: ch[k] for k in ("overlap", "mode", "group", "blocks", "update_block")}
        for blocks in (0, 32, 8):
            if not net.overlap:  # the tuner chose the classic order, which resident stepping does not run
                break
            try:
                net.set_resident(True, 16, blocks)
            except Exception as e:
                runs["resident"] = f"refused: {e}"
                break
            r = gpu_run(net, steps, n_units, bytes_per_unit, current_ptr)
            r["bound"] = f"resident stepping, {blocks or 'one per SM'} blocks: grid barrier and latency per step"
            runs[f"resident_{blocks or 'sms'}"] = r
        net.set_resident(False)
        timed = {k: v for k, v in runs.items() if isinstance(v, dict)}
        best = min(timed, key=lambda k: timed[k]["us_per_step"])
        return dict(timed[best], scheme=best), {k: (round(v["us_per_step"], 3) if isinstance(v, dict) else v)
                                               for k, v in runs.items()}

    # configuration 1: Izhikevich 1000, 2 x 0.5 ms half-steps, thalamic input
    izh = WL.izh_network(n=1000, seed=5)
    n = izh["n"]
    pops, csr, st = WL.izh_native(izh)
    pops[0].flags = sz.POP_IZH_HALF_STEPS
    steps1 = 1000
    cur = WL.thalamic(n, izh["ne"], steps1, seed=9)
    net = sz.Network(ctx, n, 0, izh["D"], pops, csr=csr, state=st, graph_chunk=100)
    dcur = ctx.upload(cur)
    g1, s1 = best_run(net, steps1, n, 16, current_ptr=dcur.ptr)  # v, u read + write
    net.close()
    dcur.free()
    c1 = {"gpu": g1, "us_per_step_by_scheme": s1}
    # oracle port, all threads, full 1000 steps
    on = oracle.OracleNet(n, 0, izh["D"], pops, csr, state=st)
    t0 = time.perf_counter()
    _, ev = on.run(steps1, current=cur, nthreads=os.cpu_count())
    dt = time.perf_counter() - t0
    c1["cpu_port"] = {"ms_per_1000_steps": dt / steps1 * 1e6, "syn_events_per_s": ev / dt,
                      "neuron_updates_per_s": n * steps1 / dt, "cores": os.cpu_count(), "kind": "port",
                      "sample": f"all {steps1} steps, 2 x 0.5 ms half-steps"}
    # the reference's own kernels (single 1 ms step, the reference's rule), bounded sample
    try:
        import oracle.clemu as clemu
        from szsnn_b200 import _lib as L
        consts = L.LayoutConsts(1024, 256, 32, 64)
        params = np.stack([izh["a"], izh["b"], izh["c"], izh["d"]], 1)
        vars_ = np.stack([izh["v0"], izh["u0"]], 1)
        sim = sz.RefSimulation(clemu.ClemuBackend("prod"), consts, "Izhikevich", params, vars_, izh["src"],
                               izh["tgt"], izh["w"], izh["d1"])
        kb = 60
        spikes = 0
        t0 = time.perf_counter()
        for k in range(kb):
            spikes += len(sim.step_and_fired(None, cur[k]))
        dt = time.perf_counter() - t0
        evb = spikes * 100  # every spike of this network reaches its 100 targets
        c1["cpu_reference_kernels"] = {
            "ms_per_1000_steps": dt / kb * 1e6, "syn_events_per_s": evb / dt,
            "neuron_updates_per_s": n * kb / dt, "cores": 1, "kind": "reference",
            "sample": f"first {kb} of {steps1} steps (single 1 ms steps, the reference's Izhikevich rule), "
                      "reference kernels under the work-group emulator, driven by the Simulation mirror"}
    except Exception as e:  # the emulator library is built only where the reference tree was present
        c1["cpu_reference_kernels"] = {"unavailable": f"{type(e).__name__}: {e}"}
    out["izh1000"] = c1

    # configuration 2: IF_curr_exp 4000, delays U{1..100}, 1000 Poisson at 10 Hz, 10,000 steps
    w = WL.if4000(seed=11)
    steps2 = 10_000
    net = sz.Network(ctx, w["n"], w["p"], w["D"], w["pops"], csr=w["csr"], state=w["state"], graph_chunk=100)
    g2, s2 = best_run(net, steps2, w["n"] + w["p"], 48)
    net.close()
    c2 = {"gpu": g2, "us_per_step_by_scheme": s2}
    on = oracle.OracleNet(w["n"], w["p"], w["D"], w["pops"], w["csr"], state=w["state"])
    t0 = time.perf_counter()
    _, ev = on.run(steps2, nthreads=os.cpu_count())
    dt = time.perf_counter() - t0
    c2["cpu_port"] = {"ms_per_1000_steps": dt / steps2 * 1e6, "syn_events_per_s": ev / dt,
                      "neuron_updates_per_s": (w["n"] + w["p"]) * steps2 / dt, "cores": os.cpu_count(),
                      "kind": "port", "sample": f"all {steps2} steps"}
    # the reference's kernels on the variant its layout holds (delays <= 64): the
    # Poisson trains drawn on the host, forced onto an input partition
    try:
        import oracle.clemu as clemu
        from szsnn_b200 import _lib as L
        wb = WL.if4000(seed=11, clip_delay=63)  # stored delays 2..64
        nn, pp = wb["n"], wb["p"]
        consts = L.LayoutConsts(1024, 256, 32, 64)
        params = np.tile(WL.if4000_params()[:9], (nn, 1))
        vars_ = np.stack([wb["state"][0][:nn], np.zeros(nn), np.zeros(nn), np.full(nn, 1e4)], 1).astype(np.float32)
        in_base = -(-nn // 1024) * 1024
        src = np.where(wb["src"] >= nn, wb["src"] - nn + in_base, wb["src"])
        sim = sz.RefSimulation(clemu.ClemuBackend("prod"), consts, "IF_curr_exp", params, vars_, src, wb["tgt"],
                               wb["w"], wb["d1"], input_params=np.zeros((pp, 1), np.float32),
                               input_vars=np.zeros((pp, 1), np.float32))
        rng = np.random.default_rng(3)
        kb = 300
        spikes = 0
        t0 = time.perf_counter()
        for k in range(kb):
            ids = in_base + np.nonzero(rng.random(pp) < wb["p_step"])[0]
            spikes += len(sim.step_and_fired(ids if len(ids) else None))
        dt = time.perf_counter() - t0
        c2["cpu_reference_kernels"] = {
            "ms_per_1000_steps": dt / kb * 1e6, "neuron_updates_per_s": (nn + pp) * kb / dt,
            "cores": 1, "kind": "reference",
            "sample": f"first {kb} of {steps2} steps of the delays <= 64 variant (the reference layout's "
                      "limit), Poisson trains forced onto an input partition, reference kernels under the "
                      "work-group emulator"}
    except Exception as e:
        c2["cpu_reference_kernels"] = {"unavailable": f"{type(e).__name__}: {e}"}
    out["if4000"] = c2
    return out


def bench_batched(ctx, args):
    """Batched sweep: the nets/s of one block-diagonal run of `batch_nets`
    uneven networks (N log-uniform 200..20,000, fan-out 100, delays U{1..20},
    weight scale 0.5..2.0, Poisson 5..20 Hz, IF_curr_exp / Izhikevich
    alternating, 100-step graphs, autotuned launch shape) against the plain
    path looped over the same nets; device time on both sides."""
    from szsnn_b200 import batch as B

    specs = B.sweep_specs(args.batch_nets, seed=0)
    r = B.compare_batched_looped(ctx, specs, steps=args.batch_steps, graph_chunk=100, tune=True)
    same = bool(np.array_equal(r["spikes_batched"], r["spikes_looped"]))
    keys = ("nets", "steps", "batched_nets_per_s", "looped_nets_per_s", "speedup", "batched_s", "looped_s",
            "wall_batched_s", "wall_looped_s", "neurons", "synapses")
    res = {"metric": "nets/s (batched sweep)", **{k: r[k] for k in keys},
           "syn_events_per_s_batched": r["events_batched"] / r["batched_s"],
           "spike_counts_equal_looped": same, "accumulation": "float",
           "workload": f"{r['nets']} nets, N log-uniform 200..20000, fan-out 100, delays U{{1..20}} steps, "
                       f"w scale 0.5..2.0, Poisson 5..20 Hz, dt 1 ms, {r['steps']} steps"}
    for k in ("looped_tuned_s", "looped_tuned_nets_per_s", "speedup_vs_tuned_loop", "loop_tuning"):
        if k in r:
            res[k] = r[k]
    if "spikes_looped_tuned" in r:
        res["spike_counts_equal_tuned_loop"] = bool(np.array_equal(r["spikes_batched"], r["spikes_looped_tuned"]))
    return res


def bench_bptt(args):
    """Differentiable IF_curr_exp RNN: one forward (simulate) against one
    forward + cross-entropy + backward through the autograd function, batch 64
    trials, 700 Poisson inputs (U(0,50) Hz), dense 700 x 10,000 input weights
    |N(0,1)| * scale / sqrt(700), 10,000 neurons with 10 % random recurrent
    weights N(0, 1/sqrt(fan-in)), 20 readouts, dt 1 ms, 500 steps, surrogate
    slope 10, checkpoints every 50 steps.  CUDA events on torch's stream (the
    stream the library launches on)."""
    import torch
    from szsnn_b200 import pyszsnn as P

    dev = torch.device("cuda")
    N, M, K, Bt, T = 10000, 700, 20, 64, args.bptt_steps
    rp, col, val = P.random_recurrent(N, 0.1, 0, dev)
    g = torch.Generator().manual_seed(0)
    w_in = (torch.randn((M, N), generator=g).abs() * args.bptt_scale / np.sqrt(M)).to(dev)
    w_out = (torch.randn((N, K), generator=g) / np.sqrt(N)).to(dev)
    rates = (torch.rand(M, generator=g) * 50).to(dev)
    x = P.poisson_bits(T, Bt, rates, 1.0, 0)
    v0 = torch.zeros((Bt, N), device=dev)
    labels = torch.randint(0, K, (Bt,), generator=g).to(dev)
    net = P.LIFCurrExpRNN(N, M, K, rp, col, beta=10.0, checkpoint_every=50,
                          store_trajectory={"auto": None, "keep": True, "recompute": False}[args.bptt_trajectory])
    for t in (w_in, val, w_out):
        t.requires_grad_(True)

    def fwd():
        return P.simulate(net, w_in.detach(), val.detach(), w_out.detach(), x, v0)

    def fwdbwd():
        for t in (w_in, val, w_out):
            t.grad = None
        ymax, _ = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
        loss = torch.nn.functional.cross_entropy(ymax, labels)
        loss.backward()
        return loss

    for _ in range(2):
        fwd()
        fwdbwd()
    torch.cuda.synchronize()
    reps = 3
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(reps):
        out = fwd()
    e[1].record()
    for _ in range(reps):
        loss = fwdbwd()
    e[2].record()
    torch.cuda.synchronize()
    f_ms = e[0].elapsed_time(e[1]) / reps
    fb_ms = e[1].elapsed_time(e[2]) / reps
    rate = float(P.unpack_bits(out["spikes"], N).float().mean()) * 1e3
    stored = net.stores_trajectory(T, Bt, dev)
    net.phase_ms = np.zeros(4)  # one more backward, timed per phase (untimed above)
    fwdbwd()
    torch.cuda.synchronize()
    phases = {k: round(float(v), 3) for k, v in zip(P.BACKWARD_PHASES, net.phase_ms)}
    net.phase_ms = None
    return {"metric": "BPTT forward+backward cost / forward cost", "fwd_ms": f_ms, "fwd_bwd_ms": fb_ms,
            "ratio": fb_ms / f_ms, "rate_hz": rate, "loss": float(loss.detach()), "trials": Bt, "steps": T,
            "neurons": N, "inputs": M, "readouts": K, "synapses": int(col.numel()), "w_in_scale": args.bptt_scale,
            "stored_trajectory": stored, "backward_phase_ms": phases,
            "workload": "IF_curr_exp RNN 10,000 neurons (10 % recurrent), 700 Poisson inputs, 20 readouts, "
                        "batch 64, 500 steps, fast-sigmoid slope 10, "
                        + ("membrane trajectory kept by the forward for the backward" if stored
                           else "checkpoints every 50 steps, recomputed in the backward")}


def run_reference(args, rank):
    """The reference arm: the oracle port of the reference's step (all host
    threads) on the benchmark network itself (--cpu-neurons overrides its
    size).  One step is S simulation steps, S = ceil(2000 / K), so the K
    timed steps cover at least 2000 simulation steps; the warm-up is
    max(500, W * S) simulation steps, past the start-up volley."""
    if rank != 0:
        return
    K, W = max(1, args.steps), max(1, args.warmup)
    S = sim_steps_per_step(K, args.sim_steps or REF_SIM_STEPS)
    n = args.cpu_neurons or args.neurons
    warm = max(CPU_WARM_STEPS, W * S)
    value, ev, dt, desc, threads = cpu_port_measure(n, args.fanout, args.seed, warm, K * S)
    nn, p, D, _, _ = cond_config(n, args.fanout)
    cb = {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": dt / (K * S) * 1e3, "sim_steps_per_step": S,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(nn, p, D, nn * args.fanout + p * 100, "float"),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def refine_live(net, ctx, ch, k, steps=1000, warm=200, current_ptr=None):
    """The tuner ranks shapes on replays of one step; the live step (a
    different spike pattern each step, the graphs' back-to-back launches)
    can order them differently.  The k best overlapped shapes by replay time
    are timed live (CUDA events around szsnn_net_run_device) and the fastest
    is applied.  The network advances meanwhile: this is warm-up."""
    sms = 148
    cand, seen = [], set()
    for tr in sorted((t for t in ch.get("trials", []) if t[0] == "overlapped"), key=lambda t: t[-1]):
        _, ub, mode, group, tps, _us = tr
        shape = (mode, group, max(1, tps * sms // ub), ub)
        if shape not in seen:
            seen.add(shape)
            cand.append(shape)
        if len(cand) == k:
            break
    live = []
    for mode, group, blocks, ub in cand:
        net.set_tuning(mode, group, blocks, ub)
        net.run_device(warm, current_ptr=current_ptr)
        ctx.sync()
        net.run_device(steps, current_ptr=current_ptr)
        ctx.sync()
        live.append((net.device_ms() / steps * 1e3, (mode, group, blocks, ub)))
    best = min(live)
    net.set_tuning(*best[1])
    return {"chosen": dict(zip(("mode", "group", "blocks", "update_block"), best[1])),
            "candidates_us": [[round(us, 3), list(sh)] for us, sh in live]}


def choose_resident(net, ctx, mode, warps, steps=1000, warm=200):
    """Live device time per step (CUDA events around szsnn_net_run_device)
    of the tuned graphs and of resident stepping with each update-warp split;
    resident stepping stays on when it is faster (mode "auto") or always
    (mode "on", with its fastest split).  The network advances meanwhile:
    this is warm-up."""
    def live():
        net.run_device(warm)
        ctx.sync()
        net.run_device(steps)
        ctx.sync()
        return net.device_ms() / steps * 1e3

    net.set_resident(False)
    trials = {"graphs": round(live(), 3)}
    best = None
    for uw in warps:
        try:
            net.set_resident(True, uw)
        except Exception as e:  # the network does not qualify: graphs only
            trials[f"resident_{uw}"] = f"refused: {e}"
            break
        us = live()
        trials[f"resident_{uw}"] = round(us, 3)
        if best is None or us < best[0]:
            best = (us, uw)
    on = best is not None and (mode == "on" or best[0] < trials["graphs"])
    net.set_resident(on, best[1] if on else 0)
    return {"resident": on, "update_warps": best[1] if on else None, "live_us": trials}


def reduce_replicas(dist, t, units):
    """Replicas only: (max over ranks of the timed duration, sum over ranks of
    the units processed).  Every rank calls it in the same order; `dist` is
    torch.distributed (NCCL on GPUs, gloo in the CPU tests) or None."""
    if dist is None:
        return float(t), float(units)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    x = torch.tensor([float(t), float(units)], dtype=torch.float64, device=dev)
    m = x[:1].clone()
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    u = x[1:].clone()
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(m.item()), float(u.item())


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import szsnn_b200 as sz
    from szsnn_b200 import _lib as L

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist

    def barrier():
        if dist is not None:
            dist.barrier()

    K, W = max(1, args.steps), max(1, args.warmup)
    S = sim_steps_per_step(K, args.sim_steps or GPU_SIM_STEPS)
    ctx = sz.Context(local_rank)
    n, p, D, blocks, pops = cond_config(args.neurons, args.fanout)
    acc = L.ACC_FIXED if args.acc == "fixed" else L.ACC_FLOAT
    net = sz.Network(ctx, n, p, D, pops, state=init_state(n, p, args.seed + rank), acc_mode=acc, graph_chunk=100)
    t0 = time.perf_counter()
    net.generate(blocks, seed=args.seed + 1000 * rank)
    net.set_overlap(args.overlap)
    gen_s = time.perf_counter() - t0

    # warm-up: W x S simulation steps (graph capture, the start-up transient),
    # then the launch shape chosen by the autotuner on replays of a warmed-up
    # step (scratch state), then W x S more steps in the chosen shape
    net.run_device(W * S)
    ctx.sync()
    tuning = None
    if args.shape:
        f = args.shape.split(",")
        order, mode, group, blocks_, ub = f[:5]
        tiles, per_sm = (int(f[5]), int(f[6])) if len(f) >= 7 else (0, 0)
        net.set_overlap(order == "overlapped")
        net.set_tuning(int(mode), int(group), int(blocks_), int(ub))
        net.set_update_tiles(tiles, per_sm)
        tuning = {"overlap": order == "overlapped", "mode": int(mode), "group": int(group), "blocks": int(blocks_),
                  "update_block": int(ub), "update_tiles": tiles, "update_per_sm": per_sm, "source": "--shape"}
    elif args.tune:  # past the start-up transient (v(0) ~ U(-60,-50) fires a first volley)
        from szsnn_b200.autotune import tune
        net.run_device(max(0, args.tune_after - W * S))
        ctx.sync()
        ch = tune(net, replays=50, use_cache=False)
        tuning = {k: ch[k] for k in ("overlap", "mode", "group", "blocks", "update_block", "step_us",
                                     "classic_step_us")}
        if ch["overlap"] and args.live_shapes > 1:
            tuning["live"] = refine_live(net, ctx, ch, args.live_shapes)
    resident = None
    if args.resident != "off" and net.overlap:
        resident = choose_resident(net, ctx, args.resident, [int(x) for x in args.resident_warps.split(",") if x])
    net.run_device(W * S)
    ctx.sync()
    overlap = bool(net.overlap)
    res_on = bool(resident and resident["resident"])
    s0 = net.stats()
    barrier()
    ctx.sync()
    # timed: K x S simulation steps in CUDA graphs (every graph already
    # instantiated: szsnn_net_run_device builds them before its first event)
    # or in resident chunks (one cooperative launch per 100 steps); CUDA
    # events on the net's stream around the launches
    with ClockSampler(local_rank) as clk:
        t_wall = time.perf_counter()
        net.run_device(K * S)
        ctx.sync()
        t_wall = time.perf_counter() - t_wall
    ms_timed = net.device_ms()
    barrier()
    s1 = net.stats()
    sim_steps = K * S
    events = s1["events"] - s0["events"]
    spikes = s1["spikes"] - s0["spikes"]
    ms_max, ev_tot = reduce_replicas(dist, ms_timed, events)
    value = ev_tot / (ms_max / 1e3)
    us_live = ms_max / sim_steps * 1e3

    # end to end through the public API: host input words in, host raster out,
    # every step, both in page-locked host memory (DMA overlapped with compute)
    e2e_steps = min(args.e2e_steps, sim_steps)
    forced, raster = pinned_words(e2e_steps, net.words), pinned_words(e2e_steps, net.words)
    forced[:] = 0
    # untimed warm-up through the same call (its graphs and bounce paths)
    warm = min(e2e_steps, 2 * net.graph_chunk)
    net.run(warm, forced_words=forced[:warm], out=raster[:warm])
    ctx.sync()
    s2 = net.stats()
    barrier()
    t_e2e = time.perf_counter()
    net.run(e2e_steps, forced_words=forced, out=raster)
    ctx.sync()
    t_e2e = time.perf_counter() - t_e2e
    s3 = net.stats()
    e2e_events = s3["events"] - s2["events"]
    e2e_max, e2e_tot = reduce_replicas(dist, t_e2e, e2e_events)
    del raster, forced

    # per-kernel device time: replays of the current step on scratch state,
    # CUDA events on the launching stream around each group of launches
    prof = net.profile_step(args.profile_steps)
    steps_p = args.profile_steps
    ev_launch = prof["events_per_launch"]
    hbm, peak_kind = peaks()
    prop_us = prof["propagate_ms"] / steps_p * 1e3
    upd_us = prof["update_ms"] / steps_p * 1e3
    step_us = prof["step_ms"] / steps_p * 1e3
    ev_step = events / sim_steps
    upd_bytes = n * BYTES_PER_NEURON
    step_bytes = upd_bytes + ev_step * BYTES_PER_EVENT
    chip = ctx.probe_peaks(n)  # measured L2 copy bandwidth and random-reduction rate
    # the dominant kernel: k_step (one fused launch per step: the update of
    # every unit, the delay-1 buckets of its spikes and the delay >= 2
    # delivery of the next step) in the overlapped order; its live time per
    # launch is the timed region's time per simulation step
    traffic = (NCU_STEP_TRAFFIC_WARM
               if (n + p == 1_100_000 and args.fanout == 1000 and overlap and not res_on) else None)
    achieved = step_bytes / (us_live * 1e-6) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": traffic,
                "kernel": "k_resident" if res_on else ("k_step" if overlap else "k_propagate + k_update"),
                "peak_source": peak_kind,
                "us_per_launch": round(us_live, 3), "algorithmic_bytes_per_launch": int(step_bytes),
                "timing": "live: the timed region's device time per simulation step",
                "l2_gbs_peak": round(chip["l2_copy_gbs"], 1),
                "l2_frac": round(achieved / chip["l2_copy_gbs"], 4),
                "atomic_per_s_peak": chip["red_per_s"],
                "atomic_frac": round(ev_step / (us_live * 1e-6) / chip["red_per_s"], 4),
                "ceilings": "l2_gbs_peak: L2-resident copy of 2 x 16 MB; atomic_per_s_peak: random fp32 red into "
                            "2 x N floats (szsnn_probe_peaks, this device, this run)",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_step on this workload, L2 "
                                  "warm as in the timed run (--cache-control none), mean of three launches",
                "replays": {"step_us": round(step_us, 3), "order": "overlapped" if overlap else "classic",
                            "of": "the per-step launches (k_step) on scratch state" if res_on else "the timed kernels",
                            "delivery_alone_us": round(prop_us, 3), "delivery_events": ev_launch,
                            "delivery_gbs": round(ev_launch * BYTES_PER_EVENT / (prop_us * 1e-6) / 1e9, 1),
                            "delays": "2..64" if overlap else "1..64",
                            "update_alone_us": round(upd_us, 3),
                            "update_gbs": round(upd_bytes / (upd_us * 1e-6) / 1e9, 1)}}
    n_syn, words = net.n_synapses, net.words
    net.close()  # frees the 8 GB synapse table before the other workloads

    configs = batched = bptt = None
    if rank == 0 and world == 1 and not args.no_configs:
        try:
            configs = bench_configs(ctx, args)
        except Exception as e:  # reported beside the headline, not required for it
            configs = {"error": f"{type(e).__name__}: {e}"}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cb = cpu_baseline(args)
        except Exception as e:  # the baseline is reported, not required
            cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}
    if rank == 0 and world == 1 and not args.no_secondary:
        try:
            batched = bench_batched(ctx, args)
        except Exception as e:
            batched = {"error": f"{type(e).__name__}: {e}"}
        try:
            bptt = bench_bptt(args)
        except Exception as e:
            bptt = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / sim_steps, "sim_steps_per_step": S, "sim_steps_timed": sim_steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(n, p, D, n_syn, args.acc),
            "parallelism": f"replicas x{world}", "step_order": "overlapped" if overlap else "classic",
            "graph_chunk": 100, "tuning": tuning, "resident": resident,
            "neuron_updates_per_s": (n + p) * sim_steps * world / (ms_max / 1e3),
            "mean_rate_hz": spikes / max(n + p, 1) / (sim_steps * DT_MS * 1e-3),
            "events_per_step": events / sim_steps,
            "wall_s_timed": t_wall,
            "generate_s": gen_s,
            "roofline": roofline,
            "cpu_baseline": cb,
            "e2e": {"value": e2e_tot / e2e_max, "unit": UNIT, "steps": e2e_steps,
                    "h2d_bytes_per_step": int(words * 4), "d2h_bytes_per_step": int(words * 4),
                    "api": "szsnn_net_run (forced-spike words in, raster out, page-locked host arrays)"},
            "gpu_launches": int((sim_steps + 99) // 100 if res_on
                                else (1 if overlap else 2) * sim_steps + (sim_steps + 99) // 100),
            "clocks": clk.summary(),
            "configs": configs,
            "batched": batched,
            "bptt": bptt,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
