"""CPU: the benchmark's live choices, against a stand-in network whose device
times are scripted per launch shape and stepping scheme (no GPU).

  * refine_live takes the tuner's best overlapped shapes by replay time
    (distinct shapes, classic trials ignored), times each live and applies
    the fastest;
  * choose_resident keeps resident stepping only when it beats the graphs
    (mode auto), keeps it with its fastest split when forced (mode on), and
    falls back to the graphs when the network does not qualify.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class FakeCtx:
    def sync(self):
        pass


class FakeNet:
    """Device time per step from `times`, keyed by the current shape or the
    resident split; records what was applied."""

    def __init__(self, shape_us=None, graphs_us=20.0, resident_us=None, refuse=False):
        self.shape_us = shape_us or {}
        self.graphs_us = graphs_us
        self.resident_us = resident_us or {}
        self.refuse = refuse
        self.shape = None
        self.resident = (False, 0)
        self.steps = 0

    def set_tuning(self, mode, group, blocks, ub):
        self.shape = (mode, group, blocks, ub)

    def set_resident(self, on, update_warps=0, blocks=0):
        if on and self.refuse:
            raise RuntimeError("resident stepping needs the overlapped step order")
        self.resident = (bool(on), update_warps)

    def run_device(self, steps, current_ptr=None):
        self.steps = steps

    def device_ms(self):
        if self.resident[0]:
            us = self.resident_us[self.resident[1]]
        elif self.shape in self.shape_us:
            us = self.shape_us[self.shape]
        else:
            us = self.graphs_us
        return us * self.steps / 1e3


def _trial(ub, mode, group, tps, us):
    return ("overlapped", ub, mode, group, tps, us)


def test_refine_live_times_the_best_replay_shapes_and_keeps_the_fastest():
    # replay order: A (15.0) < B (15.1) < A again (15.2, same shape) < C (15.3) < D (16.0);
    # live order: C fastest
    trials = [_trial(128, 1, 16, 256, 15.0), _trial(128, 1, 8, 256, 15.1), ("classic-update", 256, 14.0),
              _trial(128, 1, 16, 256, 15.2), _trial(256, 1, 16, 256, 15.3), _trial(64, 0, 16, 256, 16.0)]
    sms = 148
    a, b, c, d = (1, 16, 256 * sms // 128, 128), (1, 8, 256 * sms // 128, 128), (1, 16, 256 * sms // 256, 256), \
        (0, 16, 256 * sms // 64, 64)
    net = FakeNet(shape_us={a: 15.6, b: 15.9, c: 15.2, d: 14.0})
    out = bench.refine_live(net, FakeCtx(), {"trials": trials}, 3)
    assert [tuple(sh) for _, sh in out["candidates_us"]] == [a, b, c]  # distinct, best three by replay
    assert net.shape == c
    assert out["chosen"] == {"mode": 1, "group": 16, "blocks": c[2], "update_block": 256}


def test_choose_resident_keeps_the_graphs_when_faster():
    net = FakeNet(graphs_us=15.5, resident_us={12: 33.0, 16: 27.0, 20: 24.5, 24: 22.4})
    out = bench.choose_resident(net, FakeCtx(), "auto", [12, 16, 20, 24])
    assert out["resident"] is False and net.resident == (False, 0)
    assert out["live_us"]["graphs"] == 15.5 and out["live_us"]["resident_24"] == 22.4


def test_choose_resident_keeps_resident_when_faster_or_forced():
    net = FakeNet(graphs_us=15.5, resident_us={12: 14.0, 16: 12.5})
    out = bench.choose_resident(net, FakeCtx(), "auto", [12, 16])
    assert out["resident"] is True and out["update_warps"] == 16 and net.resident == (True, 16)
    net = FakeNet(graphs_us=15.5, resident_us={12: 30.0, 16: 25.0})
    out = bench.choose_resident(net, FakeCtx(), "on", [12, 16])
    assert out["resident"] is True and out["update_warps"] == 16


def test_choose_resident_falls_back_when_refused():
    net = FakeNet(graphs_us=15.5, refuse=True)
    out = bench.choose_resident(net, FakeCtx(), "auto", [12, 16])
    assert out["resident"] is False and "refused" in out["live_us"]["resident_12"]


@pytest.mark.parametrize("k,least,s", [(20, 20_000, 1000), (3, 2000, 667), (1, 5, 5)])
def test_sim_steps_per_step_covers_the_least(k, least, s):
    assert bench.sim_steps_per_step(k, least) == s and k * s >= least
