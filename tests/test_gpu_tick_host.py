"""gx_tick_host: one tick against host ECS columns.

The call must give the same bits as the three calls it replaces
(gx_set_dynamic, gx_step(h, 1, stats, 1), gx_get_state): on the list path
with its rebuilds and the thermostat's pending scale, on the FP64 list path
and on the per-tick cell path, with pinned and with pageable columns, and
when the host moves atoms between ticks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _lattice(n_side=14, temperature=300.0, coul=True, thermo=True, seed=0):
    wl = W.Workload("tick host", n_side=n_side, temperature=temperature, steps=10, seed=seed,
                    electrostatics=coul)
    cfg = wl.config()
    if thermo:
        cfg.enable_thermostat = True
        cfg.thermostat_temperature = 60.0
    return cfg, wl.generate()


def _columns(u, pinned):
    if not pinned:
        return [np.ascontiguousarray(a, dtype=np.float64).copy() for a in (u.pos, u.vel, np.zeros_like(u.pos))]
    import torch
    out = []
    for a in (u.pos, u.vel, np.zeros_like(u.pos)):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = a
        out.append(t)
    return out


def _run_pair(cfg, u, precision, variant, ticks, pinned, move=None, bonds=None):
    from genesis_b200._lib import Handle
    keep = _columns(u, pinned)  # torch tensors stay alive while their arrays are used
    cols = [c.numpy() if hasattr(c, "numpy") else c for c in keep]
    ref = [c.copy() for c in cols]
    ha, hb = Handle(cfg, precision), Handle(cfg, precision)
    for h in (ha, hb):
        h.set_kernel_variant(variant)
        h.set_universe(u)
        if bonds is not None:
            h.set_bonds(bonds)
    rec_a, rec_b = [], []
    for t in range(ticks):
        if move is not None and t == move:  # the host moves one atom by a box quarter
            for c in (cols, ref):
                c[0][7] += 0.25 * np.asarray(cfg.size)
        rec_a.append(ha.tick_host(*cols))
        hb.set_dynamic(*ref)
        rec_b.append(hb.step(1, graph=True))
        hb.get_state_into(*ref)
    out = (cols, ref, np.concatenate(rec_a), np.concatenate(rec_b), ha.list_rebuilds(), hb.list_rebuilds())
    ha.close()
    hb.close()
    del keep
    return out


@pytest.mark.parametrize("pinned", [True, False])
def test_list_path_matches_the_three_calls(gpu, pinned):
    cfg, u = _lattice()
    cols, ref, ra, rb, na, nb = _run_pair(cfg, u, "mixed", 6, 24, pinned)
    for x, y in zip(cols, ref):
        assert np.array_equal(x, y)
    assert np.array_equal(ra, rb)
    assert na == nb and na >= 2  # the ticks include list rebuilds


def test_fp64_list_path_matches_the_three_calls(gpu):
    cfg, u = _lattice(12)
    cols, ref, ra, rb, _, _ = _run_pair(cfg, u, "fp64", 0, 10, True)
    for x, y in zip(cols, ref):
        assert np.array_equal(x, y)
    assert np.array_equal(ra, rb)


def test_cell_path_matches_the_three_calls(gpu):
    # variant 1 re-sorts every tick into the other buffer: the positions
    # follow the tick instead of overlapping the pair pass
    cfg, u = _lattice(12)
    cols, ref, ra, rb, _, _ = _run_pair(cfg, u, "mixed", 1, 8, True)
    for x, y in zip(cols, ref):
        assert np.array_equal(x, y)
    assert np.array_equal(ra, rb)


def test_host_moves_between_ticks(gpu):
    cfg, u = _lattice(12, temperature=60.0, thermo=False)
    cols, ref, ra, rb, na, nb = _run_pair(cfg, u, "mixed", 6, 8, True, move=4)
    for x, y in zip(cols, ref):
        assert np.array_equal(x, y)
    assert np.array_equal(ra, rb)
    assert na == nb


def test_spring_and_collisions_on_the_list_path(gpu):
    # the spring and the collision pass run after the positions-final event:
    # they write forces and velocities only
    cfg, u = _lattice(12, temperature=300.0)
    cfg.enable_bond_interaction = True
    cfg.enable_collisions = True
    cfg.particle_radius = 1.3  # contact 2.6, below the lattice spacing: neighbours touch
    bonds = np.array([[2 * k, 2 * k + 1] for k in range(60)], dtype=np.uint32)
    cols, ref, ra, rb, na, nb = _run_pair(cfg, u, "mixed", 6, 12, True, bonds=bonds)
    for x, y in zip(cols, ref):
        assert np.array_equal(x, y)
    assert np.array_equal(ra, rb)
    assert np.any(ra["bond_energy"] != 0.0)


def test_tick_host_then_step_then_tick_host(gpu):
    # the positions-final event joins the captured ticks once; plain steps
    # in between keep giving the bits of a handle that never used it
    from genesis_b200._lib import Handle
    cfg, u = _lattice(12)
    cols = _columns(u, False)
    ha, hb = Handle(cfg, "mixed"), Handle(cfg, "mixed")
    for h in (ha, hb):
        h.set_kernel_variant(6)
        h.set_universe(u)
    ha.tick_host(*cols)
    ha.step(9, graph=True)
    p, v, a = ha.get_state()
    cols = [p, v, a]
    ha.tick_host(*cols)
    hb.step(11, graph=True)
    for x, y in zip(cols, hb.get_state()):
        assert np.array_equal(x, y)
    ha.close()
    hb.close()


def test_tick_host_rejects_missing_columns(gpu):
    from genesis_b200._lib import GxError, Handle
    cfg, u = _lattice(8)
    with Handle(cfg, "mixed") as h:
        h.set_universe(u)
        pos = np.ascontiguousarray(u.pos, dtype=np.float64).copy()
        with pytest.raises(ValueError):
            h.tick_host(pos, pos[:-1].copy(), pos.copy())
        rc = h.lib.gx_tick_host(h.h, pos.ctypes.data_as(C.POINTER(C.c_double)), None, None, None)
        assert rc != 0
        with pytest.raises(GxError):
            h._check(rc)
