"""Neuron / source model parameter slots and dt folding.

Slot numbering follows the reference's model classes:
  IF_curr_exp  (szsnn1.1/src/models/IF_curr_exp_NeuronModel.hpp:12-30): params
     v_rest, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, i_offset, v_reset,
     v_thresh; vars v, Ie, Ii, fired (steps since the last spike, init 10000)
  Izhikevich   (models/Izhikevich_NeuronModel.hpp:82-93): params a, b, c, d; vars v, u
  Const_rate   (models/Const_rate_InputModel.hpp:140-147): param rate; var last
New models with no reference class: IF_cond_exp (IF_curr_exp slots + e_rev_E,
e_rev_I; vars v, ge, gi, fired) and Poisson (param p = rate * dt).

The reference kernels assume dt = 1 (IF_curr_exp_update_kernel.cl:230,261,
Izhikevich_update_kernel.cl:259); `fold_dt` turns physical parameters at a
time step dt (ms) into those step units: every time constant and cm divided by
dt, the refractory period in steps.
"""
from __future__ import annotations

import numpy as np

from ._lib import CONST_RATE, IF_COND_EXP, IF_CURR_EXP, IZHIKEVICH, POISSON

IF_SLOTS = ["v_rest", "cm", "tau_m", "tau_refrac", "tau_syn_E", "tau_syn_I", "i_offset", "v_reset",
            "v_thresh", "e_rev_E", "e_rev_I"]
IZH_SLOTS = ["a", "b", "c", "d"]

# defaults of IF_curr_exp_NeuronModel() (IF_curr_exp_NeuronModel.hpp:36-51)
IF_CURR_EXP_DEFAULTS = dict(v_rest=-65.0, cm=1.0, tau_m=20.0, tau_refrac=0.0, tau_syn_E=5.0, tau_syn_I=5.0,
                            i_offset=0.0, v_reset=-65.0, v_thresh=-65.0)
IF_CURR_EXP_VAR_DEFAULTS = dict(v=0.0, Ie=0.0, Ii=0.0, fired=10000.0)
# Izhikevich_NeuronModel() (Izhikevich_NeuronModel.hpp:100-110)
IZH_DEFAULTS = dict(a=0.02, b=0.2, c=-65.0, d=2.0)

PARAM_COUNT = {IF_CURR_EXP: 9, IF_COND_EXP: 11, IZHIKEVICH: 4, POISSON: 1, CONST_RATE: 1}
VAR_COUNT = {IF_CURR_EXP: 4, IF_COND_EXP: 4, IZHIKEVICH: 2, POISSON: 0, CONST_RATE: 1}
MODEL_NAMES = {IF_CURR_EXP: "IF_curr_exp", IF_COND_EXP: "IF_cond_exp", IZHIKEVICH: "Izhikevich",
               POISSON: "Poisson", CONST_RATE: "Const_rate"}


def if_params(**kw) -> np.ndarray:
    """12-slot fp32 parameter vector for IF_curr_exp / IF_cond_exp."""
    p = np.zeros(12, dtype=np.float32)
    vals = dict(IF_CURR_EXP_DEFAULTS)
    vals.update(e_rev_E=0.0, e_rev_I=-70.0)
    vals.update(kw)
    for i, k in enumerate(IF_SLOTS):
        p[i] = np.float32(vals[k])
    return p


def izh_params(a=0.02, b=0.2, c=-65.0, d=2.0) -> np.ndarray:
    p = np.zeros(12, dtype=np.float32)
    p[:4] = np.array([a, b, c, d], dtype=np.float32)
    return p


def fold_dt(params: np.ndarray, dt: float) -> np.ndarray:
    """Physical IF parameters at time step dt (ms) -> the kernels' step units.

    tau_m, tau_syn_E, tau_syn_I and cm are divided by dt (so 1/tau' = dt/tau and
    I/cm' = I*dt/cm), tau_refrac becomes a step count.  Works on a 12-slot
    vector or on a [12, n] per-neuron array."""
    out = np.array(params, dtype=np.float32, copy=True)
    dtf = np.float32(dt)
    for slot in (1, 2, 3, 4, 5):  # cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I
        out[slot] = (out[slot] / dtf).astype(np.float32)
    return out
