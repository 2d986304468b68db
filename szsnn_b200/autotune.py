"""Launch-shape autotuner for a Network: step order, delivery variant and
grid, update block.

Candidates are timed with Network.profile_step: replays of the current step on
scratch copies of the state, CUDA events on the launching stream, the network
itself untouched.  The overlapped order (one fused launch per step) is tuned
on the whole-step time over (delivery variant, delivery threads per SM, update
block); the classic order (propagate, then update) tunes its two launches
independently; the faster order wins.  Results are cached in a JSON file keyed
by device and workload shape ($SZSNN_TUNE_CACHE, default
~/.cache/szsnn_b200/tune.json); a hit skips the search.
"""
from __future__ import annotations

import json
import os

PROPAGATE = [(0, 8, 16), (0, 16, 8), (0, 16, 16), (0, 16, 32), (0, 32, 8), (0, 32, 16),
             (1, 8, 8), (1, 8, 16), (1, 16, 16), (1, 16, 32), (1, 32, 16)]  # classic: (mode, group, blocks/SM)
UPDATE = [64, 128, 256]
FAR = [(0, 16), (0, 8), (1, 8), (1, 16), (1, 32)]        # overlapped delivery: (mode, group)
FAR_THREADS_PER_SM = [256, 512, 1024, 2048, 4096]


def _cache_path() -> str:
    return os.environ.get("SZSNN_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "szsnn_b200", "tune.json"))


def workload_key(net, events_per_step: float, sms: int) -> str:
    ev_bucket = int(round(max(events_per_step, 1.0))).bit_length()
    return (f"v2-sms{sms}-U{net.U.bit_length()}-D{net.D}-pops{'many' if len(net.pops) > 8 else 'few'}"
            f"-ev{ev_bucket}")


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only costs the next search


def _apply(net, c: dict) -> None:
    net.set_overlap(c["overlap"])
    net.set_tuning(c["mode"], c["group"], c["blocks"], c["update_block"])


def tune(net, replays: int = 20, sms: int = 148, use_cache: bool = True, cache: dict | None = None) -> dict:
    """Pick and apply the fastest step order and launch shape; returns the
    choice and timings.  `cache`: a dict shared by the calls of one run in
    place of the file cache (workloads of one size bucket tuned once)."""
    ev = net.profile_step(1)["events_per_launch"]
    key = workload_key(net, ev, sms)
    mem = cache is not None
    if mem:
        use_cache = False
    else:
        cache = _load() if use_cache else {}
    if key in cache:
        c = cache[key]
        _apply(net, c)
        return dict(c, cached=True, key=key)
    trials = []
    # classic order: the two launches tuned independently
    net.set_overlap(False)
    best_p = best_u = None
    for mode, group, per_sm in PROPAGATE:
        net.set_tuning(mode, group, per_sm * sms, 256)
        p_ms = net.profile_step(replays)["propagate_ms"]
        trials.append(("classic-propagate", mode, group, per_sm, p_ms / replays))
        if best_p is None or p_ms < best_p[0]:
            best_p = (p_ms, mode, group, per_sm * sms)
    for ub in UPDATE:
        net.set_tuning(best_p[1], best_p[2], best_p[3], ub)
        u_ms = net.profile_step(replays)["update_ms"]
        trials.append(("classic-update", ub, u_ms / replays))
        if best_u is None or u_ms < best_u[0]:
            best_u = (u_ms, ub)
    net.set_tuning(best_p[1], best_p[2], best_p[3], best_u[1])
    classic = dict(overlap=False, mode=best_p[1], group=best_p[2], blocks=best_p[3], update_block=best_u[1],
                   step_us=net.profile_step(replays)["step_ms"] / replays * 1e3)
    # overlapped order: whole-step time of the fused launch
    best = classic
    net.set_overlap(True)
    for ub in UPDATE:
        for mode, group in FAR:
            for tps in FAR_THREADS_PER_SM:
                blocks = max(1, tps * sms // ub)
                net.set_tuning(mode, group, blocks, ub)
                us = net.profile_step(replays)["step_ms"] / replays * 1e3
                trials.append(("overlapped", ub, mode, group, tps, us))
                if us < best["step_us"]:
                    best = dict(overlap=True, mode=mode, group=group, blocks=blocks, update_block=ub, step_us=us)
    choice = dict(best, classic_step_us=classic["step_us"])
    _apply(net, choice)
    if use_cache or mem:
        cache[key] = choice
    if use_cache:
        _store(cache)
    return dict(choice, cached=False, key=key, trials=trials)
