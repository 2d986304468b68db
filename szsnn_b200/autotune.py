"""Launch-shape autotuner for a Network (propagate variant, grid, update block).

Candidates are timed with Network.profile: replays of the current step's
propagate and update launches on scratch copies of the state, CUDA events on
the launching stream, the network itself untouched.  The propagate and update
choices are independent, so each is tuned on its own.  Results are cached in a
JSON file keyed by device and workload shape ($SZSNN_TUNE_CACHE, default
~/.cache/szsnn_b200/tune.json); a hit skips the search.
"""
from __future__ import annotations

import json
import os

PROPAGATE = [(0, 8, 16), (0, 16, 8), (0, 16, 16), (0, 16, 32), (0, 32, 8), (0, 32, 16),
             (1, 8, 8), (1, 8, 16), (1, 16, 16)]          # (mode, group, blocks per SM)
UPDATE = [128, 256, 512]


def _cache_path() -> str:
    return os.environ.get("SZSNN_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "szsnn_b200", "tune.json"))


def workload_key(net, events_per_step: float, sms: int) -> str:
    ev_bucket = int(round(max(events_per_step, 1.0))).bit_length()
    return (f"sms{sms}-U{net.U.bit_length()}-D{net.D}-pops{'many' if len(net.pops) > 8 else 'few'}"
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


def tune(net, replays: int = 20, sms: int = 148, use_cache: bool = True) -> dict:
    """Pick and apply the fastest launch shape; returns the choice and timings."""
    _, _, ev = net.profile(1)
    key = workload_key(net, ev, sms)
    cache = _load() if use_cache else {}
    if key in cache:
        c = cache[key]
        net.set_tuning(c["mode"], c["group"], c["blocks"], c["update_block"])
        return dict(c, cached=True, key=key)
    best_p, best_u = None, None
    trials = []
    for mode, group, per_sm in PROPAGATE:
        net.set_tuning(mode, group, per_sm * sms, 256)
        p_ms, _, _ = net.profile(replays)
        trials.append(("propagate", mode, group, per_sm, p_ms / replays))
        if best_p is None or p_ms < best_p[0]:
            best_p = (p_ms, mode, group, per_sm * sms)
    for ub in UPDATE:
        net.set_tuning(best_p[1], best_p[2], best_p[3], ub)
        _, u_ms, _ = net.profile(replays)
        trials.append(("update", ub, u_ms / replays))
        if best_u is None or u_ms < best_u[0]:
            best_u = (u_ms, ub)
    choice = dict(mode=best_p[1], group=best_p[2], blocks=best_p[3], update_block=best_u[1],
                  propagate_us=best_p[0] / replays * 1e3, update_us=best_u[0] / replays * 1e3)
    net.set_tuning(choice["mode"], choice["group"], choice["blocks"], choice["update_block"])
    if use_cache:
        cache[key] = choice
        _store(cache)
    return dict(choice, cached=False, key=key, trials=trials)
