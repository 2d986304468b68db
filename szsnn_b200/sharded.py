"""A network sharded by unit ranges across devices, one process per GPU.

No counterpart in the reference, which runs one network on one device with
one in-order queue (Context.cpp:211-213).  For a network larger than one
device holds, the units are split into contiguous ranges (neurons and
sources separately, word-aligned) and each rank keeps:

  * the whole id space (spike ids, ring slots and synapse rows keep their
    global numbering), updating only its own ranges (szsnn_net_set_owned);
  * only the synapses whose target it owns (shard_csr): each rank delivers
    into its own targets;
  * after every step, its own units' spike words go to every other rank (an
    all-gather of U/32 words: N/8 bytes per step) and the words of the other
    ranks are injected into its ring for that step (szsnn_net_inject_spikes),
    which also delivers their delay-1 buckets before the next step.

One exchange per step is what a minimum delay of one step allows; the ranks'
spike rasters together equal the unsharded network's, bit for bit in
fixed-point accumulation.  `exchange` is any callable mapping this rank's
words to the list of every rank's words, in rank order: an all-gather over
torch.distributed (NCCL between GPUs, gloo on CPU) from `dist_exchange`, or
a local stand-in.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class ShardRange:
    rank: int
    n_lo: int
    n_hi: int
    s_lo: int
    s_hi: int

    def owns(self, ids) -> np.ndarray:
        ids = np.asarray(ids)
        return ((ids >= self.n_lo) & (ids < self.n_hi)) | ((ids >= self.s_lo) & (ids < self.s_hi))


def plan(n_neurons: int, n_sources: int, world: int) -> list[ShardRange]:
    """Contiguous neuron and source ranges per rank, neuron boundaries at
    multiples of 32 units, as even as that allows."""
    if world < 1:
        raise ValueError("world must be >= 1")

    def cuts(lo, count, align):
        b = [lo + ((count * r // world) // align) * align for r in range(world)] + [lo + count]
        return b

    nb = cuts(0, n_neurons, 32)
    sb = cuts(n_neurons, n_sources, 1)
    return [ShardRange(r, nb[r], nb[r + 1], sb[r], sb[r + 1]) for r in range(world)]


def shard_csr(csr, n_units: int, max_delay: int, rng: ShardRange):
    """The rows of a delay-bucketed CSR (row_ptr [U*D+1], tgt, w) kept to the
    synapses whose target neuron the shard owns, in their original order."""
    row_ptr, tgt, w = (np.asarray(a) for a in csr)
    keep = (tgt >= rng.n_lo) & (tgt < rng.n_hi)
    counts = np.diff(row_ptr.astype(np.int64))
    bucket = np.repeat(np.arange(n_units * max_delay), counts)
    new_counts = np.bincount(bucket[keep], minlength=n_units * max_delay)
    rp = np.zeros(n_units * max_delay + 1, np.uint64)
    rp[1:] = np.cumsum(new_counts, dtype=np.uint64)
    return rp, np.ascontiguousarray(tgt[keep], np.int32), np.ascontiguousarray(w[keep], np.float32)


def own_words(words: np.ndarray, rng: ShardRange, n_units: int) -> np.ndarray:
    """This shard's spikes among a step's words (other units' bits cleared)."""
    mask = np.zeros(len(words) * 32, bool)
    mask[rng.n_lo:rng.n_hi] = True
    mask[rng.s_lo:rng.s_hi] = True
    mask[n_units:] = False
    m = np.packbits(mask, bitorder="little").view(np.uint32)  # bit k of word w: unit 32 w + k
    return np.asarray(words, np.uint32) & m


def dist_exchange(dist, device: str = "cpu"):
    """An all-gather of one step's words over torch.distributed."""
    import torch

    def ex(words: np.ndarray) -> list[np.ndarray]:
        x = torch.from_numpy(np.ascontiguousarray(words).view(np.int32)).to(device)
        out = [torch.empty_like(x) for _ in range(dist.get_world_size())]
        dist.all_gather(out, x)
        return [o.cpu().numpy().view(np.uint32) for o in out]
    return ex


class ShardedRunner:
    """Steps one shard: `net` has step() -> words and inject_spikes(words)
    (szsnn_b200.Network, or any object with both); returns per step the
    union of all shards' spike words."""

    def __init__(self, net, rng: ShardRange, n_units: int, exchange):
        self.net, self.rng, self.U, self.exchange = net, rng, n_units, exchange

    def step(self) -> np.ndarray:
        mine = own_words(self.net.step(), self.rng, self.U)
        every = self.exchange(mine)
        others = np.zeros_like(mine)
        for r, w in enumerate(every):
            if r != self.rng.rank:
                others |= np.asarray(w, np.uint32)
        self.net.inject_spikes(others)
        return mine | others

    def run(self, steps: int) -> np.ndarray:
        return np.stack([self.step() for _ in range(steps)])
