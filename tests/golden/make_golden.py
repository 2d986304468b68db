"""Extract golden vectors from the reference's known-answer files.

Run once where the reference tree is present:
    python tests/golden/make_golden.py <reference root>
It writes small .npz fixtures beside this script; the tests only read those.

Sources (paths inside the reference project):
  szsnn1.1/bin/pyNN2neurony.vvv~   1000-step membrane trace of neuron 1 of the
      2-neuron IF_curr_exp test (bin/2_neurony.py:6-31: v_rest -49, tau_m 20,
      cm 1, v_reset -200, v_thresh -50, tau_syn_E 5, v(0) -70, one-to-one
      weight 100 from neuron 0 to neuron 1), written by PyNN/Brian in fp64.
  szsnn1.1/bin/myfile.txt~         SZSNN's own fp32 debug log of a 1000-cycle
      IF_curr_exp run: for neuron 1 of partition 0 the kernel prints, each
      cycle, Ie / Ii with their input sums and V with last value, rest, tau,
      reset, I, cm and delta (IF_curr_exp_update_kernel.cl:241-242,267-269).
  szsnn1.1/bin/izi1.conn~, izi2.conn~   the connection files of the reference's
      100-neuron Izhikevich example (src/main.cpp:139-142): 80 excitatory and
      20 inhibitory sources; copied byte for byte as izi1.conn / izi2.conn.
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def pynn_trace(ref: str) -> np.ndarray:
    path = os.path.join(ref, "szsnn1.1", "bin", "pyNN2neurony.vvv~")
    vals = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            vals.append(float(line.split()[0]))
    return np.array(vals, dtype=np.float64)


_IE = re.compile(r">>>>>>IE (\S+) last(\S+) in(\S+) tau(\S+)")
_II = re.compile(r">>>>>>II (\S+) last(\S+) in(\S+) tau(\S+)")
_V = re.compile(r">>>>>>V (\S+) last(\S+) rest(\S+) tau(\S+) reset(\S+) I(\S+), cm(\S+), delta(\S+)")


def szsnn_log(ref: str) -> dict:
    path = os.path.join(ref, "szsnn1.1", "bin", "myfile.txt~")
    ie, ii, v = [], [], []
    with open(path, errors="replace") as f:
        for line in f:
            m = _IE.search(line)
            if m:
                ie.append([float(x) for x in m.groups()])
                continue
            m = _II.search(line)
            if m:
                ii.append([float(x) for x in m.groups()])
                continue
            m = _V.search(line)
            if m:
                v.append([float(x) for x in m.groups()])
    ie, ii, v = np.array(ie), np.array(ii), np.array(v)
    n = min(len(ie), len(ii), len(v))
    return dict(
        in_exc=ie[:n, 2], in_inh=ii[:n, 2], ie=ie[:n, 0], ii=ii[:n, 0], tau_e=ie[:n, 3], tau_i=ii[:n, 3],
        v=v[:n, 0], v_last=v[:n, 1], v_rest=v[:n, 2], tau_m=v[:n, 3], v_reset=v[:n, 4], I=v[:n, 5],
        cm=v[:n, 6], delta=v[:n, 7])


def main(ref: str) -> None:
    tr = pynn_trace(ref)
    np.savez_compressed(os.path.join(HERE, "pynn_2neuron_v.npz"), v=tr)
    lg = szsnn_log(ref)
    np.savez_compressed(os.path.join(HERE, "szsnn_if_curr_exp_log.npz"), **lg)
    for name in ("izi1", "izi2"):
        with open(os.path.join(ref, "szsnn1.1", "bin", name + ".conn~"), "rb") as f:
            data = f.read()
        with open(os.path.join(HERE, name + ".conn"), "wb") as f:
            f.write(data)
    print(f"pynn trace: {len(tr)} steps; szsnn log: {len(lg['v'])} cycles; izi1/izi2.conn copied")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference root>")
    main(sys.argv[1])
