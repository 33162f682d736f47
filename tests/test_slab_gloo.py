"""One universe over two ranks (gloo on the CPU): z slabs, migration and the
per-tick halo exchange (genesis_b200/slab.py), with the oracle's FP64 force
pass as each rank's force engine.  The decomposed trajectory must follow
the oracle's single-process ticks (the per-atom force sums run in another
order, and the kinetic energy is summed per rank first: 1e-10 relative over
eight ticks), every atom owned by exactly one rank, and atoms must cross
the slab boundaries in the run."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
TICKS = 8


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from genesis_b200 import workloads as W
    wl = W.C1.scaled(12)
    cfg = wl.config()
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 120.0
    cfg.enable_electrostatics = True
    u = wl.generate()
    u.vel *= 3.0  # hot enough that atoms cross the slab boundaries
    return cfg, u


def _worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from genesis_b200 import elements as E
    from genesis_b200 import slab
    from oracle import oracle

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, u = _case()
        rc = E.LJ_CUTOFF_FACTOR * max(cfg.sigma)
        sl = slab.Slabs(cfg.size, rc, rank, world, dist)
        wrapped = np.mod(u.pos, np.asarray(cfg.size)) - 0.5 * np.asarray(cfg.size)  # only to pick owners
        mine = sl.owner(wrapped[:, 2]) == rank
        own = slab.Owned(u.pos[mine], u.vel[mine], np.zeros((int(mine.sum()), 3)), u.elem[mine], u.charge[mine],
                         u.mass[mine], np.nonzero(mine)[0])

        def force(pos, elem, charge, mass):
            return oracle.forces(cfg, pos, elem, charge, mass)[0]

        migrated = 0
        for _ in range(TICKS):
            before = set(own.ids.tolist())
            own, K, lam = slab.tick(sl, own, force, cfg, u.n)
            migrated += len(set(own.ids.tolist()) - before)
        out.put((rank, own.ids, own.pos, own.vel, own.acc, K, lam, migrated))
    finally:
        dist.destroy_process_group()


def test_two_slabs_follow_the_single_process_ticks():
    import torch.multiprocessing as mp

    sys.path.insert(0, str(ROOT))
    from oracle import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=300)
        res[r[0]] = r
    for p in ps:
        p.join(60)
    assert all(p.exitcode == 0 for p in ps)
    cfg, u = _case()
    p_ref, v_ref, a_ref, st_ref = oracle.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, TICKS)
    ids = np.concatenate([res[0][1], res[1][1]])
    assert np.array_equal(np.sort(ids), np.arange(u.n))  # every atom owned exactly once
    pos = np.empty_like(p_ref)
    vel = np.empty_like(v_ref)
    acc = np.empty_like(a_ref)
    for r in (0, 1):
        pos[res[r][1]] = res[r][2]
        vel[res[r][1]] = res[r][3]
        acc[res[r][1]] = res[r][4]
    for x, y in ((pos, p_ref), (vel, v_ref), (acc, a_ref)):
        assert np.linalg.norm(x - y) <= 1e-10 * np.linalg.norm(y)
    # the all-reduced kinetic energy before the scale, times lambda^2, is the oracle's after it
    assert abs(res[0][5] * res[0][6] ** 2 - st_ref[-1, 0]) <= 1e-10 * abs(st_ref[-1, 0])
    assert res[0][6] == res[1][6] and abs(res[0][6] - st_ref[-1, 3]) <= 1e-12  # the same lambda on both
    assert res[0][7] + res[1][7] > 0  # atoms crossed the slab boundaries


def test_slab_geometry_rejects_narrow_slabs():
    import pytest

    sys.path.insert(0, str(ROOT))
    from genesis_b200 import slab
    with pytest.raises(ValueError):
        slab.Slabs((20.0, 20.0, 20.0), 5.75, 0, 2)  # 10-wide slabs < 2 r_c
    s = slab.Slabs((60.0, 60.0, 60.0), 5.75, 1, 3)
    assert s.peers() == [0, 2]
    assert list(s.owner(np.array([-30.0, -10.0, 0.0, 10.0, 29.99]))) == [0, 1, 1, 2, 2]
