#!/usr/bin/env python
"""Benchmark: synaptic events/s of the 1M-neuron IF_cond_exp network on B200.

Workload (the large IF_cond_exp configuration): 1,000,000 IF_cond_exp neurons
(800k excitatory / 200k inhibitory), 1000 random synapses per neuron (1e9
synapses; targets uniform without self-loops; weights exc ~U(0,4) nS, inh
~U(0,51) nS stored negative; delays U{1..64} steps), e_rev_E 0, e_rev_I -80 mV,
tau_syn_E 5, tau_syn_I 10 ms, dt 0.1 ms, 100,000 Poisson inputs at 5 Hz with
100 targets each, fp32 state.  Parameters the configuration leaves open are
taken from the 4000-neuron IF_curr_exp configuration (tau_m 20 ms, cm 0.2 nF,
v_rest -60, v_thresh -50, v_reset -60 mV, tau_refrac 5 ms); Poisson synapses
~U(0,100) nS with delay 1 step; v(0) ~ U(-60,-50) mV.  Conductances in uS.

A step = one simulation time step (propagate + update); the network is built
on the device by the fixed fan-out generator.  Inputs are larger than L2
(8 GB synapse table); the per-neuron state (16 MB) stays L2-resident across
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
BYTES_PER_EVENT = 8      # int32 target + fp32 weight, delay implied by the bucket
BYTES_PER_NEURON = 48    # 16 B state read + 16 B write + 8 B input read + 8 B clear
# DRAM bytes (read + write) per launch from single ncu captures (cold L2):
# k_update at 1.1M units, the benchmark's unit count; k_propagate at 300k
# neurons x 1000 synapses (152,640 events per launch), scaled by events.
NCU_UPDATE_TRAFFIC = 25_399_040
NCU_PROPAGATE_TRAFFIC_PER_EVENT = 5_706_752 / 152_640
# k_step at 1.1M units and fan-out 100 (245,471 events per launch): 70.7 MB; the per-(spike, delay)
# item traffic is the same at fan-out 1000, each further event adds its 8 B synapse
NCU_STEP_TRAFFIC_FANOUT100 = 70_680_320
NCU_STEP_EVENTS_FANOUT100 = 245_471


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--neurons", type=int, default=1_000_000)
    ap.add_argument("--fanout", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--acc", default="float", choices=["float", "fixed"])
    ap.add_argument("--classic", dest="overlap", action="store_false",
                    help="propagate-then-update order (two launches per step) instead of the overlapped one")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep the default launch shape instead of autotuning after the warm-up")
    ap.add_argument("--tune-after", type=int, default=3000, help="steps simulated before the tuner's replays")
    ap.add_argument("--shape", default=None,
                    help="fixed launch shape 'order,mode,group,blocks,update_block' (order: overlapped|classic) "
                         "instead of the tuner")
    ap.add_argument("--e2e-steps", type=int, default=1000)
    ap.add_argument("--profile-steps", type=int, default=200)
    ap.add_argument("--cpu-neurons", type=int, default=50_000)
    ap.add_argument("--cpu-steps", type=int, default=300)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the batched-sweep and BPTT measurements")
    ap.add_argument("--batch-nets", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=1000)
    ap.add_argument("--bptt-scale", type=float, default=1.0)
    ap.add_argument("--bptt-steps", type=int, default=500)
    return ap.parse_args(argv)


def cond_config(n: int, fanout: int):
    """Generator blocks, populations and initial state of the benchmark network."""
    import szsnn_b200 as sz
    from szsnn_b200.network import GenBlock

    p = n // 10
    D = 64
    ne = int(0.8 * n)
    blocks = [GenBlock(0, ne, 0, n, fanout, 0.0, 0.004, 1.0, 1, D, True, 1),
              GenBlock(ne, n - ne, 0, n, fanout, 0.0, 0.051, -1.0, 1, D, True, 2),
              GenBlock(n, p, 0, n, 100, 0.0, 0.1, 1.0, 1, 1, False, 3)]
    pv = sz.fold_dt(sz.if_params(v_rest=-60, cm=0.2, tau_m=20, tau_refrac=5, tau_syn_E=5, tau_syn_I=10,
                                 v_reset=-60, v_thresh=-50, e_rev_E=0.0, e_rev_I=-80.0), DT_MS)
    pops = [sz.Pop(sz.IF_COND_EXP, 0, n, pv),
            sz.Pop(sz.POISSON, n, n + p, np.array([5.0 * DT_MS * 1e-3], np.float32), seed=20240)]
    return n, p, D, blocks, pops


def init_state(n, p, seed):
    rng = np.random.default_rng(seed)
    v0 = np.concatenate([rng.uniform(-60, -50, n), np.zeros(p)]).astype(np.float32)
    fired = np.concatenate([np.full(n, 1e4), np.zeros(p)]).astype(np.float32)
    return [v0, None, None, fired]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                line = out.stdout.strip().splitlines()[0]
                self.samples.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.1)

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
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower() in ("active", "1")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def net_overlap(net) -> bool:
    """The step order the network runs in (set by --classic or by the tuner)."""
    return bool(net.overlap)


def pinned_words(steps, words):
    """uint32 [steps, words] in page-locked host memory (torch's pinned allocator)."""
    import torch
    return torch.empty((steps, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)


def cpu_baseline(args, n_steps_warm=100):
    """Oracle port, all host threads, on a bounded sample of the same network."""
    import oracle
    import szsnn_b200 as sz  # noqa: F401

    threads = os.cpu_count() or 1
    n, p, D, blocks, pops = cond_config(args.cpu_neurons, args.fanout)
    csr = oracle.generate(blocks, args.seed, n + p, D)
    on = oracle.OracleNet(n, p, D, pops, csr, state=init_state(n, p, args.seed))
    on.run(n_steps_warm, nthreads=threads)
    t0 = time.perf_counter()
    steps = max(args.cpu_steps - n_steps_warm, 50)
    _, ev = on.run(steps, nthreads=threads)
    dt = time.perf_counter() - t0
    return {"value": ev / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} IF_cond_exp neurons x {args.fanout} synapses + {p} Poisson x 100, same weights, "
                      f"delays and rates as the 1M network; {steps} steps after {n_steps_warm} warm-up steps; "
                      f"{ev} events in {dt:.2f} s"}


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
    return {"metric": "nets/s (batched sweep)", "nets": r["nets"], "steps": r["steps"],
            "batched_nets_per_s": r["batched_nets_per_s"], "looped_nets_per_s": r["looped_nets_per_s"],
            "speedup": r["speedup"], "batched_s": r["batched_s"], "looped_s": r["looped_s"],
            "wall_batched_s": r["wall_batched_s"], "wall_looped_s": r["wall_looped_s"],
            "neurons": r["neurons"], "synapses": r["synapses"],
            "syn_events_per_s_batched": r["events_batched"] / r["batched_s"],
            "spike_counts_equal_looped": same, "accumulation": "float",
            "workload": f"{r['nets']} nets, N log-uniform 200..20000, fan-out 100, delays U{{1..20}} steps, "
                        f"w scale 0.5..2.0, Poisson 5..20 Hz, dt 1 ms, {r['steps']} steps"}


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
    net = P.LIFCurrExpRNN(N, M, K, rp, col, beta=10.0, checkpoint_every=50)
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
    return {"metric": "BPTT forward+backward cost / forward cost", "fwd_ms": f_ms, "fwd_bwd_ms": fb_ms,
            "ratio": fb_ms / f_ms, "rate_hz": rate, "loss": float(loss.detach()), "trials": Bt, "steps": T,
            "neurons": N, "inputs": M, "readouts": K, "synapses": int(col.numel()), "w_in_scale": args.bptt_scale,
            "workload": "IF_curr_exp RNN 10,000 neurons (10 % recurrent), 700 Poisson inputs, 20 readouts, "
                        "batch 64, 500 steps, fast-sigmoid slope 10, checkpoints every 50 steps"}


def run_reference(args, rank):
    """The reference arm: the oracle port of the reference's step (all host
    threads) on the bounded CPU sample of the benchmark network.  One bench
    step is S simulation steps of the sample, S = ceil(2000 / K), so the K
    timed steps cover at least 2000 simulation steps and at most K; the W
    warm-up steps (W * S simulation steps, at least 100) fill the delay ring."""
    if rank != 0:
        return
    import oracle
    import szsnn_b200 as sz  # noqa: F401

    K, W = max(1, args.steps), max(1, args.warmup)
    S = max(1, -(-2000 // K))
    threads = os.cpu_count() or 1
    n, p, D, blocks, pops = cond_config(args.cpu_neurons, args.fanout)
    csr = oracle.generate(blocks, args.seed, n + p, D)
    on = oracle.OracleNet(n, p, D, pops, csr, state=init_state(n, p, args.seed))
    on.run(max(W * S, 100), nthreads=threads)
    t0 = time.perf_counter()
    _, ev = on.run(K * S, nthreads=threads)
    dt = time.perf_counter() - t0
    value = ev / dt
    cb = {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
          "sample": f"{n} IF_cond_exp neurons x {args.fanout} synapses + {p} Poisson x 100, same weights, "
                    f"delays and rates as the 1M network; {K} steps of {S} simulation steps after "
                    f"{max(W * S, 100)} warm-up simulation steps; {ev} events in {dt:.2f} s"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": dt / K * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "IF_cond_exp 1M x 1000 syn, Poisson 100k x 100, dt 0.1 ms (bounded CPU sample)",
                       "neurons": args.cpu_neurons, "sim_steps_per_step": S},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


    ctx = sz.Context(local_rank)
    n, p, D, blocks, pops = cond_config(args.neurons, args.fanout)
    acc = L.ACC_FIXED if args.acc == "fixed" else L.ACC_FLOAT
    net = sz.Network(ctx, n, p, D, pops, state=init_state(n, p, args.seed + rank), acc_mode=acc, graph_chunk=100)
    t0 = time.perf_counter()
    net.generate(blocks, seed=args.seed + 1000 * rank)
    net.set_overlap(args.overlap)
    gen_s = time.perf_counter() - t0

    # warm-up (graph instantiation, initial transient), then the launch shape
    # chosen by the autotuner on replays of a warmed-up step (scratch state)
    net.run_device(args.warmup)
    ctx.sync()
    tuning = None
    if args.shape:
        order, mode, group, blocks_, ub = args.shape.split(",")
        net.set_overlap(order == "overlapped")
        net.set_tuning(int(mode), int(group), int(blocks_), int(ub))
        tuning = {"overlap": order == "overlapped", "mode": int(mode), "group": int(group), "blocks": int(blocks_),
                  "update_block": int(ub), "source": "--shape"}
        net.run_device(args.warmup)
        ctx.sync()
    elif args.tune:  # past the start-up transient (v(0) ~ U(-60,-50) fires a first volley)
        from szsnn_b200.autotune import tune
        net.run_device(max(0, args.tune_after - args.warmup))
        ctx.sync()
        ch = tune(net, replays=50, use_cache=False)
        tuning = {k: ch[k] for k in ("overlap", "mode", "group", "blocks", "update_block", "step_us",
                                     "classic_step_us")}
        net.run_device(args.warmup)  # graphs of the chosen shape
        ctx.sync()
    overlap = net_overlap(net)
    s0 = net.stats()
    barrier()
    ctx.sync()
    import ctypes as C
    lib = L.lib()
    # CUDA events on the net's stream, through torch if present, else via the library timing
    with ClockSampler(local_rank) as clk:
        t_wall = time.perf_counter()
        net.run_device(args.steps)
        ctx.sync()
        t_wall = time.perf_counter() - t_wall
        _, _, total_ms = (C.c_double(), C.c_double(), C.c_double())
        pm, um, tm = C.c_double(), C.c_double(), C.c_double()
        lib.szsnn_net_timing(net.h, C.byref(pm), C.byref(um), C.byref(tm))
    barrier()
    s1 = net.stats()
    ms_timed = tm.value if tm.value > 0 else t_wall * 1e3
    events = s1["events"] - s0["events"]
    spikes = s1["spikes"] - s0["spikes"]
    ms_max, ev_tot = reduce_replicas(dist, ms_timed, events)
    value = ev_tot / (ms_max / 1e3)

    # end to end through the public API: host input words in, host raster out,
    # every step, both in page-locked host memory (DMA overlapped with compute)
    e2e_steps = min(args.e2e_steps, args.steps)
    forced, raster = pinned_words(e2e_steps, net.words), pinned_words(e2e_steps, net.words)
    forced[:] = 0
    # untimed warm-up through the same call: the graphs of host-I/O chunks (both
    # stage buffers) are captured and instantiated once, outside the timed run
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
    prop_bytes = ev_launch * BYTES_PER_EVENT
    upd_bytes = n * BYTES_PER_NEURON
    ev_step = events / args.steps
    if overlap:
        # one fused launch per step (k_step): the update of every unit, the
        # delay-1 buckets of its spikes and the delay >= 2 delivery of the next step
        step_bytes = upd_bytes + ev_step * BYTES_PER_EVENT
        dom = {"kernel": "k_step", "achieved": step_bytes / (step_us * 1e-6) / 1e9, "bytes_per_launch": step_bytes,
               "us_per_launch": step_us,
               "traffic": int(NCU_STEP_TRAFFIC_FANOUT100 + max(0.0, ev_step - NCU_STEP_EVENTS_FANOUT100) * 8)
               if n + p == 1_100_000 else None}
    elif prop_us >= upd_us:
        dom = {"kernel": "k_propagate", "achieved": prop_bytes / (prop_us * 1e-6) / 1e9,
               "bytes_per_launch": prop_bytes, "us_per_launch": prop_us,
               "traffic": int(NCU_PROPAGATE_TRAFFIC_PER_EVENT * ev_launch)}
    else:
        dom = {"kernel": "k_update", "achieved": upd_bytes / (upd_us * 1e-6) / 1e9, "bytes_per_launch": upd_bytes,
               "us_per_launch": upd_us, "traffic": NCU_UPDATE_TRAFFIC if n + p == 1_100_000 else None}
    roofline = {"bound": "hbm", "achieved": round(dom["achieved"], 1), "peak": hbm, "unit": "GB/s",
                "frac": round(dom["achieved"] / hbm, 4), "traffic": dom["traffic"], "kernel": dom["kernel"],
                "peak_source": peak_kind,
                "us_per_launch": round(dom["us_per_launch"], 3),
                "algorithmic_bytes_per_launch": int(dom["bytes_per_launch"]),
                "step": {"us": round(step_us, 3), "order": "overlapped" if overlap else "classic"},
                "delivery_alone": {"us_per_launch": round(prop_us, 3),
                                   "gbs": round(prop_bytes / (prop_us * 1e-6) / 1e9, 1),
                                   "events_per_launch": ev_launch,
                                   "delays": "2..64" if overlap else "1..64"},
                "update_alone": {"us_per_launch": round(upd_us, 3),
                                 "gbs": round(upd_bytes / (upd_us * 1e-6) / 1e9, 1)}}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cb = cpu_baseline(args)
        except Exception as e:  # the baseline is reported, not required
            cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}

    n_syn, words = net.n_synapses, net.words
    net.close()  # frees the 8 GB synapse table before the secondary workloads
    batched = bptt = None
    if rank == 0 and world == 1 and not args.no_secondary:
        try:
            batched = bench_batched(ctx, args)
        except Exception as e:  # reported beside the headline, not required for it
            batched = {"error": f"{type(e).__name__}: {e}"}
        try:
            bptt = bench_bptt(args)
        except Exception as e:
            bptt = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        steps = args.steps
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "IF_cond_exp 1M neurons x 1000 synapses (1e9), 100k Poisson x 100, "
                                   "delays U{1..64} steps, dt 0.1 ms",
                       "neurons": n, "sources": p, "synapses": n_syn, "max_delay": D,
                       "accumulation": args.acc, "graph_chunk": 100,
                       "step_order": "overlapped" if overlap else "classic", "tuning": tuning,
                       "l2": "inputs larger than L2 (8 GB synapse table); neuron state L2-resident across steps",
                       "parallelism": f"replicas x{world}"},
            "neuron_updates_per_s": (n + p) * steps * world / (ms_max / 1e3),
            "mean_rate_hz": spikes / max(n + p, 1) / (steps * DT_MS * 1e-3),
            "events_per_step": events / steps,
            "generate_s": gen_s,
            "roofline": roofline,
            "cpu_baseline": cb,
            "e2e": {"value": e2e_tot / e2e_max, "unit": UNIT, "steps": e2e_steps,
                    "h2d_bytes_per_step": int(words * 4), "d2h_bytes_per_step": int(words * 4),
                    "api": "szsnn_net_run (forced-spike words in, raster out, page-locked host arrays)"},
            "gpu_launches": int((1 if overlap else 2) * steps + (steps + 99) // 100),
            "clocks": clk.summary(),
            "batched": batched,
            "bptt": bptt,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
