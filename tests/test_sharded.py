"""CPU: the sharded network's host logic (szsnn_b200.sharded) over gloo,
world size 2, with the oracle standing in for each rank's device.

Each rank owns half the neurons and half the sources (plan), keeps the
synapses into its own targets (shard_csr), steps its shard, all-gathers the
spike words of its own units and injects the other rank's words into its
spike history for that step.  The ranks' union raster must equal the
unsharded oracle run of the same network bit for bit (fixed-point
accumulation), and each rank's own neurons must end in the unsharded state.
The oracle shard updates every unit but its history keeps only its own
units' spikes plus the injected ones, which is what the device shard's
owned ranges and szsnn_net_inject_spikes do."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 80


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _network():
    import szsnn_b200 as sz
    from tests.test_gpu_parity import cond_network
    import oracle
    n, p, D = 3000, 300, 16
    blocks, pops, st = cond_network(n, p, fanout=40, D=D, seed=8)
    csr = oracle.generate(blocks, 77, n + p, D)
    return sz, n, p, D, pops, st, csr


class OracleShard:
    """One rank's shard on the oracle: step() -> this step's words; after the
    exchange, inject_spikes(others) makes the step's history slot hold the
    shard's own spikes and the injected ones."""

    def __init__(self, onet, rng, n_units):
        from szsnn_b200.sharded import own_words
        self.on, self.rng, self.U, self._own = onet, rng, n_units, own_words

    def step(self):
        import oracle
        r, _ = self.on.run(1, acc_mode=oracle.ACC_FIXED)
        return r[0]

    def inject_spikes(self, others):
        t = self.on.t - 1
        W = self.on.W
        slot = self.on.hist[(t % self.on.D) * W:(t % self.on.D + 1) * W]
        slot[:] = self._own(slot, self.rng, self.U) | others


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import oracle
    from szsnn_b200 import sharded as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sz, n, p, D, pops, st, csr = _network()
        rng = S.plan(n, p, world)[rank]
        scsr = S.shard_csr(csr, n + p, D, rng)
        shard = OracleShard(oracle.OracleNet(n, p, D, pops, scsr, state=st), rng, n + p)
        runner = S.ShardedRunner(shard, rng, n + p, S.dist_exchange(dist))
        raster = runner.run(STEPS)
        v_own = shard.on.state[0][rng.n_lo:rng.n_hi].copy()
        q.put((rank, raster, v_own, rng))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_two_ranks_equal_unsharded_oracle():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = dict((r, (ras, v, rng)) for r, ras, v, rng in (q.get(timeout=300) for _ in range(2)))
    for pr in procs:
        pr.join(120)
    assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]

    sys.path.insert(0, ROOT)
    import oracle
    sz, n, p, D, pops, st, csr = _network()
    full = oracle.OracleNet(n, p, D, pops, csr, state=st)
    ref, _ = full.run(STEPS, acc_mode=oracle.ACC_FIXED)
    assert int(np.unpackbits(ref.view(np.uint8)).sum()) > 500
    assert np.array_equal(got[0][0], ref) and np.array_equal(got[1][0], ref)
    for r in (0, 1):
        v, rng = got[r][1], got[r][2]
        assert np.array_equal(v, full.state[0][rng.n_lo:rng.n_hi])


def test_plan_and_shard_csr_partition_the_synapses():
    sys.path.insert(0, ROOT)
    from szsnn_b200 import sharded as S
    sz, n, p, D, pops, st, csr = _network()
    ranges = S.plan(n, p, 3)
    assert ranges[0].n_lo == 0 and ranges[-1].n_hi == n and ranges[0].s_lo == n and ranges[-1].s_hi == n + p
    assert all(r.n_lo % 32 == 0 for r in ranges)
    total = 0
    for r in ranges:
        rp, tg, w = S.shard_csr(csr, n + p, D, r)
        assert rp[-1] == len(tg) and np.all((tg >= r.n_lo) & (tg < r.n_hi))
        total += len(tg)
    assert total == len(csr[1])
