"""The multi-rank plumbing of bench.py on the CPU (gloo, world size 2).

The benchmark runs one independent job stream per GPU (replicas, no
collective on the data path); the only exchange is the reduction at the end:
the slowest rank's timed totals and the input bytes of all ranks, from which
rank 0 reports whole-job throughput.  Under torchrun the reference arm runs on
rank 0 alone and the other ranks exit without work.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: timed totals 10(r+1) and 5(r+1) ms, 100(r+1) input bytes
        got = bench.reduce_over_ranks(dist, "cpu", 10.0 * (rank + 1), 5.0 * (rank + 1),
                                      100 * (rank + 1))
        q.put((rank, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get() for _ in range(2))
    # every rank sees the slowest rank's times and the sum of the bytes
    assert res[0] == res[1] == (20.0, 10.0, 300.0)


def test_reduce_over_ranks_single_process():
    assert bench.reduce_over_ranks(None, "cpu", 3.0, 4.0, 7) == (3.0, 4.0, 7.0)


def test_reference_arm_only_on_rank0(capsys):
    # a rank other than 0 returns before reading its arguments or any input
    bench.reference_arm(None, rank=1)
    assert capsys.readouterr().out == ""
