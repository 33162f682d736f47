"""The bench's multi-rank plumbing (barrier, max over ranks, rank-0 output)
on two CPU ranks with the gloo backend."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), GENESIS_DIST_BACKEND="gloo")
    import bench

    d = bench.Dist(world)
    d.barrier()
    m = d.max(10.0 + rank)  # each rank's device time; the job time is the max
    d.barrier()
    d.close()
    out.put((rank, m))


def test_two_rank_max_over_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 11.0, 1: 11.0}


def test_replica_partition_is_disjoint():
    # weak scaling: every rank gets its own replica (different salt) of the workload
    from genesis_b200 import workloads as W

    a = W.C1.scaled(6).generate(salt=0)
    b = W.C1.scaled(6).generate(salt=1)
    assert not (a.pos == b.pos).all()
