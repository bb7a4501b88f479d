"""The multi-replica path of bench.py on CPU with two gloo ranks: every rank
ends with the slowest rank's time (max over ranks), and under the reference
arm only rank 0 works and prints while the other ranks exit 0 silently."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = 1.5 + rank  # rank 1 is the slow one
        got = bench.max_over_ranks(mine, dist, device="cpu")
        dist.barrier()
        q.put((rank, mine, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[2] for r in res] == [2.5, 2.5]


def test_max_over_ranks_without_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25) == 3.25


def test_reference_arm_nonzero_rank_is_silent(capsys):
    import sys
    from types import SimpleNamespace
    sys.path.insert(0, ROOT)
    import bench
    assert bench.run_reference(SimpleNamespace(steps=1, warmup=0), rank=1, world=2) == 0
    assert capsys.readouterr().out == ""
