"""The reference's network files, read into a native Network.

Formats (restated from the reference's readers; no reference code is used):
  * connection files -- Connection::loadFromFile (szsnn1.1/src/Connection.hpp:71-140):
    two header lines (skipped), then `from to weight delay` per line, whitespace
    separated, indices local to the connection's source / target start ids.  A
    later line for the same (from, to) pair replaces the earlier one (the
    reference keeps a map keyed by the pair, iterated in ascending (from, to)).
    Reading stops at the first line without four values; that is a format error
    unless it is the end of the file.  `from`, `to` and `delay` are read as
    numbers and truncated to integers, as the reference does through float.
  * population files -- Population::loadFromFile / loadFromTemplateFile
    (Population.hpp:118-292): '#' comment lines, then the population size, the
    first neuron id and a label, then the model's parameters and variables:
    once per neuron (full file) or once for all neurons (template file).
    Parameter / variable order is the model's enum order (IF_curr_exp: v_rest,
    cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, i_offset, v_reset, v_thresh /
    v, Ie, Ii, fired; Izhikevich: a, b, c, d / v, u; Const_rate: rate / last;
    models/*_NeuronModel.hpp, Const_rate_InputModel.hpp), which is the native
    slot order.
  * assembly -- NetworkCreator::fillNetworkGraph (NetworkCreator.hpp:110-190):
    neuron id = population first id + index, synapse (from_start + from,
    to_start + to, weight, delay + 1) (NetworkGraph.ipp:416,431,495).  Input
    connections come from input populations (ids after the neurons in the
    native layout).  The reference's loop for input synapses walks the neuron
    connections a second time (NetworkCreator.hpp:167); the builder adds the
    input connections, which is what that loop is for.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .network import Network, Pop, csr_from_synapses

# model -> (parameter count, variable count), the reference's traits
# (models/neuron_model_traits.hpp:90-91,119-120,149-150)
MODEL_SHAPE = {L.IF_CURR_EXP: (9, 4), L.IZHIKEVICH: (4, 2), L.CONST_RATE: (1, 1)}


class NetFileError(ValueError):
    """A network file that does not follow the reference's format."""


@dataclass
class Connections:
    """One connection file: local (from, to) indices, weights and user delays."""
    src: np.ndarray
    tgt: np.ndarray
    w: np.ndarray
    delay: np.ndarray
    from_start: int = 0
    to_start: int = 0


def _int_field(tok: str) -> int:
    v = float(tok)
    if not np.isfinite(v) or v < 0:
        raise ValueError(tok)
    return int(v)


def read_conn(path: str, from_start: int = 0, to_start: int = 0) -> Connections:
    pairs: dict[tuple[int, int], tuple[float, int]] = {}
    with open(path) as f:
        lines = f.read().split("\n")
    body = lines[2:]
    for k, line in enumerate(body):
        vals = line.split()
        if len(vals) != 4:
            rest = [x for x in body[k:] if x.strip()]
            if rest:
                raise NetFileError(f"{path}: wrong format at line #{k + 3}: {len(vals)} values, expected 4")
            break
        try:
            a, b = _int_field(vals[0]), _int_field(vals[1])
            w = float(np.float32(vals[2]))
            d = _int_field(vals[3])
        except ValueError:
            raise NetFileError(f"{path}: wrong format at line #{k + 3}: `{line.strip()}`") from None
        pairs[(a, b)] = (w, d)
    keys = sorted(pairs)
    src = np.array([k[0] for k in keys], np.int64)
    tgt = np.array([k[1] for k in keys], np.int64)
    w = np.array([pairs[k][0] for k in keys], np.float32)
    d = np.array([pairs[k][1] for k in keys], np.int64)
    return Connections(src, tgt, w, d, from_start, to_start)


@dataclass
class PopulationFile:
    model: int
    size: int
    first_id: int
    label: str
    params: np.ndarray   # [param_count][size] fp32
    vars: np.ndarray     # [var_count][size] fp32


def read_population(path: str, model: int, template: bool = False) -> PopulationFile:
    if model not in MODEL_SHAPE:
        raise NetFileError(f"model {model} has no population-file shape")
    npar, nvar = MODEL_SHAPE[model]
    toks = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            toks.extend(s.split())
    try:
        size, first = _int_field(toks[0]), _int_field(toks[1])
        label = toks[2]
        nums = np.array([np.float32(x) for x in toks[3:]], np.float32)
    except (IndexError, ValueError):
        raise NetFileError(f"{path}: wrong header (size, first id, label)") from None
    if size <= 0:
        raise NetFileError(f"{path}: population size must be > 0")
    per = npar + nvar
    need = per if template else per * size
    if nums.size < need:
        raise NetFileError(f"{path}: not enough data: {nums.size} values, {need} needed for {size} neurons")
    rows = np.tile(nums[:per], (size, 1)) if template else nums[:need].reshape(size, per)
    return PopulationFile(model, size, first, label, np.ascontiguousarray(rows[:, :npar].T),
                          np.ascontiguousarray(rows[:, npar:].T))


@dataclass
class NetworkFiles:
    """Populations and connections in the reference's terms, assembled like
    NetworkCreator::fillNetworkGraph."""
    populations: list[PopulationFile] = field(default_factory=list)
    inputs: list[PopulationFile] = field(default_factory=list)
    connections: list[Connections] = field(default_factory=list)
    input_connections: list[Connections] = field(default_factory=list)

    def synapses(self):
        """Global (src unit, tgt neuron, weight, stored delay) arrays; input ids
        follow the neurons."""
        n = self.n_neurons
        parts = []
        for cons, src_off in ((self.connections, 0), (self.input_connections, n)):
            for c in cons:
                parts.append((src_off + c.from_start + c.src, c.to_start + c.tgt, c.w, c.delay + 1))
        if not parts:
            e = np.zeros(0, np.int64)
            return e, e, np.zeros(0, np.float32), e
        return tuple(np.concatenate([p[i] for p in parts]) for i in range(4))

    @property
    def n_neurons(self) -> int:
        return max((p.first_id + p.size for p in self.populations), default=0)

    @property
    def n_inputs(self) -> int:
        return max((p.first_id + p.size for p in self.inputs), default=0)

    def build(self, ctx, acc_mode: int = L.ACC_FLOAT, graph_chunk: int = 100, **kw) -> Network:
        n, p = self.n_neurons, self.n_inputs
        covered = np.zeros(n, bool)
        for pf in self.populations:
            if covered[pf.first_id: pf.first_id + pf.size].any():
                raise NetFileError(f"population `{pf.label}` overlaps another")
            covered[pf.first_id: pf.first_id + pf.size] = True
        if not covered.all():
            raise NetFileError("neuron ids are not contiguous from 0")
        src, tgt, w, d1 = self.synapses()
        if src.size and (tgt.max() >= n or src.max() >= n + p):
            raise NetFileError("a connection names a neuron or input outside the populations")
        D = int(d1.max()) if d1.size else 1
        csr = csr_from_synapses(n + p, D, src, tgt, w, d1.astype(np.uint32))
        pops, state = [], [np.zeros(n + p, np.float32) for _ in range(4)]
        for pf, off in [(x, 0) for x in self.populations] + [(x, n) for x in self.inputs]:
            a = off + pf.first_id
            per_unit = np.zeros((12, pf.size), np.float32)
            per_unit[: pf.params.shape[0]] = pf.params
            shared = bool(np.all(pf.params == pf.params[:, :1]))
            pops.append(Pop(pf.model, a, a + pf.size, per_unit[:, 0].copy(),
                            per_unit=None if shared else per_unit))
            for k in range(pf.vars.shape[0]):
                state[k][a: a + pf.size] = pf.vars[k]
        pops.sort(key=lambda q: q.begin)
        return Network(ctx, n, p, D, pops, csr=csr, state=state, acc_mode=acc_mode, graph_chunk=graph_chunk, **kw)
