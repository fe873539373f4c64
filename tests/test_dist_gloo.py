"""Replica-run plumbing with two gloo ranks on CPU: barrier and max-over-ranks timing."""

import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from asuka_b200.dist import barrier, max_over_ranks, world as w

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert w() == (rank, world)
        barrier()
        out[rank] = max_over_ranks(10.0 + rank)
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert dict(out) == {0: 11.0, 1: 11.0}


def test_single_process_is_identity():
    from asuka_b200.dist import max_over_ranks

    assert max_over_ranks(3.5) == 3.5
