"""gx_snapshot_world: the snapshot's Vec<EntitySnapshot> encoded on the
device, byte for byte against the CPU restatement (oracle/snapshot.py), on a
state the device has re-sorted (so every column goes through the slot map)
and with observed bonds."""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W
from oracle import snapshot as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_world_bytes_match_the_restatement(gpu, precision):
    from genesis_b200._lib import Handle
    wl = W.C2.scaled(10)
    cfg, u = wl.config(), wl.generate()
    ent = (np.arange(u.n, dtype=np.uint32) * 3 + 5).astype(np.uint32)
    u.entity = ent
    gen = (np.arange(u.n) % 4).astype(np.uint32)
    with Handle(cfg, precision) as h:
        h.set_universe(u)
        for t in range(1, 61):
            h.step(1)
            h.bond_observe(cfg.bond_k_bind, 0.1, t)
        bonds = h.get_bonds()
        assert len(bonds) > 0
        pos, vel, acc = h.get_state()
        got = h.snapshot_world(gen)
        got0 = h.snapshot_world()
    want = S.encode_world(pos, vel, acc, u.mass, u.charge, u.elem, ent, gen, bonds)
    assert got == want
    recs = S.decode_world(got0)
    assert all(r["generation"] == 0 for r in recs) and [r["index"] for r in recs] == list(ent)


def test_world_bytes_of_the_quench_lattice(gpu):
    from genesis_b200._lib import Handle
    wl = W.C3.scaled(48)
    cfg, u = wl.config(), wl.generate()
    with Handle(cfg, "mixed") as h:
        h.set_universe(u)
        h.step(3)
        pos, vel, acc = h.get_state()
        got = h.snapshot_world()
    assert len(got) == 8 + S.RECORD_FIXED * u.n
    want = S.encode_world(pos, vel, acc, u.mass, u.charge, u.elem)
    assert got == want
