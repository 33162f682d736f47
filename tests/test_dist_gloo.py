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


def _sweep_worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), GENESIS_DIST_BACKEND="gloo")
    import numpy as np

    import bench
    from genesis_b200 import sweep

    d = bench.Dist(world)
    wls = sweep.make_replicas(256, seed=0)
    parts = sweep.partition([wl.n_atoms for wl in wls], world)
    # stand-in for this rank's batch: one row per replica it was given
    local = [[float(i), float(wls[i].n_atoms), float(rank), 0.0] for i in parts[rank]]
    stats = sweep.assemble(parts, d.all_gather_object(local))
    t = d.max(float(len(parts[rank])))
    d.close()
    out.put((rank, stats.tolist(), t))


def test_sharded_sweep_gathers_every_replica_once():
    import numpy as np
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_sweep_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    res = {r: (np.array(s), t) for r, s, t in (q.get(timeout=5) for _ in range(2))}
    s0, t0 = res[0]
    assert np.array_equal(s0, res[1][0]) and t0 == res[1][1] == 128.0
    assert np.array_equal(s0[:, 0], np.arange(256))  # every replica back in its place, once
    assert set(np.unique(s0[:, 2])) == {0.0, 1.0}


def test_partition_is_size_balanced():
    from genesis_b200 import sweep

    sizes = [wl.n_atoms for wl in sweep.make_replicas(256, seed=0)]
    for world in (1, 2, 3, 4, 8):
        parts = sweep.partition(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(256))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)  # greedy packing bound
    with pytest.raises(ValueError):
        sweep.assemble([[0, 1], [2]], [[[1.0]], [[2.0]]])
