"""CPU: the multi-rank logic of bench.py (replicas only) over gloo, world size 2.

Each rank runs its own replica; the job's value is all ranks' units over the
slowest rank's time.  The ranks here report fixed durations and unit counts,
so the reduction can be checked exactly."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = [12.5, 20.0][rank]           # ms of this rank's timed region
        units = [1000, 3000][rank]       # events this rank processed
        q.put((rank, bench.reduce_replicas(dist, t, units)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reduce_replicas_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got[0] == got[1] == (20.0, 4000.0)


def test_reduce_replicas_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_replicas(None, 7.0, 11) == (7.0, 11.0)


def test_reference_arm_other_ranks_do_nothing(capsys):
    """Under torchrun only rank 0 runs the reference arm; other ranks exit
    without work or output."""
    sys.path.insert(0, ROOT)
    import bench
    bench.run_reference(None, rank=1)
    assert capsys.readouterr().out == ""


def test_reference_arm_reports_the_steps_it_was_given(capsys):
    """The reference arm's line carries the K timed and W warm-up steps of its
    command line, each step S = ceil(2000 / K) simulation steps of the
    network the port runs, and its value is that network's events over the
    timed steps."""
    import json
    sys.path.insert(0, ROOT)
    import bench
    args = bench.parse(["--impl", "reference", "--steps", "3", "--warmup", "4", "--cpu-neurons", "2000"])
    bench.run_reference(args, rank=0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 3 and line["warmup"] == 4
    assert line["sim_steps_per_step"] == 667
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
