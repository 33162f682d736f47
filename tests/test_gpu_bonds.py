"""Bond observation on the device (gx_bond_observe) against the oracle's
restatement of PairTracker + BondObservationSystem, tick by tick.

Exact: the summary (bonded pairs and atoms, coordination, bonds formed and
their summed lifetimes, open and completed episodes, the species matrix)
and the persistent pairs, which become the handle's bond list.
"""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

KEYS = ("bonded_pairs", "bonded_entities", "mean_coordination", "bonds_formed", "lifetime_sum_ticks",
        "open_episodes", "completed_episodes", "completed_ticks")


def _ionic(n_side=10, temperature=300.0):
    wl = W.Workload("bond check", n_side=n_side, temperature=temperature, steps=10, seed=5, electrostatics=True,
                    thermostat=True, thermostat_temperature=temperature, bond_observation=True,
                    bond_interaction=True, species=(E.by_name("Na"), E.by_name("O")),
                    fixed_fractions={E.by_name("Na"): 0.5, E.by_name("O"): 0.5})
    return wl.config(), wl.generate()


@pytest.mark.parametrize("precision,min_periods", [("fp64", 0.2), ("mixed", 0.2), ("mixed", 10.0)])
def test_observation_matches_oracle_tick_by_tick(gpu, orc, precision, min_periods):
    from genesis_b200._lib import Handle
    cfg, u = _ionic()
    h = Handle(cfg, precision)
    h.set_universe(u)
    ref = orc.BondTracker(cfg, debounce=E.DEBOUNCE, min_periods=min_periods)
    seen_formed = 0
    for tick in range(1, 121):
        h.step(1)
        bound = h.bound_pairs(cfg.bond_k_bind)  # entity = slot here
        got = h.bond_observe(cfg.bond_k_bind, min_periods, tick)
        want, pers = ref.observe(bound, u.elem, tick)
        assert got["bound_pairs"] == len(bound)
        for k in KEYS:
            assert got[k] == want[k], (tick, k, got[k], want[k])
        assert np.array_equal(got["species_matrix"], want["species_matrix"])
        bonds = h.get_bonds()
        assert np.array_equal(np.sort(bonds.view(np.uint64).ravel()), np.sort(pers.view(np.uint64).ravel()))
        seen_formed = got["bonds_formed"]
    if min_periods < 1.0:
        assert got["bonded_pairs"] > 0 and seen_formed > 0  # both persistence and breaking were exercised


def test_observed_bonds_drive_the_spring(gpu, orc):
    # after an observation with apply_bonds the next force pass applies the
    # spring to exactly the observed pairs (src/systems/forces.rs:305-317)
    from genesis_b200._lib import Handle
    cfg, u = _ionic(n_side=8)
    h = Handle(cfg, "fp64")
    h.set_universe(u)
    for tick in range(1, 400):
        h.step(1)
        if h.bond_observe(cfg.bond_k_bind, 0.2, tick)["bonded_pairs"] > 0 and tick > 20:
            break
    bonds = h.get_bonds()
    assert len(bonds) > 0
    pos, vel, acc = h.get_state()
    V, Vb, _ = h.forces()
    acc_ref, V_ref, Vb_ref, _ = orc.forces(cfg, pos, u.elem, u.charge, u.mass, bonds=bonds)
    _, _, acc = h.get_state()
    assert np.linalg.norm(acc - acc_ref) <= 1e-12 * np.linalg.norm(acc_ref)
    assert abs(Vb - Vb_ref) <= 1e-12 * max(abs(Vb_ref), 1e-300) and Vb_ref != 0.0


def test_lifetime_and_species_matrix_on_device(gpu, orc):
    # src/systems/bonds.rs:263-341 replayed on the device: an H-H pair at 1.0
    # held past its threshold, then separated
    from genesis_b200._lib import Handle
    from genesis_b200.config import default_config
    cfg = default_config()
    cfg.size = (30.0, 30.0, 30.0)
    hh = E.by_name("H")
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    h = Handle(cfg, "fp64")
    h.set_state(pos, np.zeros((2, 3)), np.array([hh, hh], dtype=np.uint8))
    thr = orc.BondTracker(cfg).threshold(hh, hh)
    tick = 0
    for _ in range(thr + 500):
        tick += 1
        st = h.bond_observe(cfg.bond_k_bind, cfg.bond_min_periods, tick)
    assert st["bonded_pairs"] == 1 and st["bonds_formed"] == 0
    assert st["species_matrix"][hh, hh] == 2
    h.set_dynamic(pos=np.array([[0.0, 0.0, 0.0], [6.0, 0.0, 0.0]]))
    for _ in range(E.DEBOUNCE + 2):
        tick += 1
        st = h.bond_observe(cfg.bond_k_bind, cfg.bond_min_periods, tick)
    assert st["bonded_pairs"] == 0 and st["bonds_formed"] == 1
    assert st["lifetime_sum_ticks"] == 502.0


def test_reset_and_new_state_start_afresh(gpu):
    from genesis_b200._lib import Handle
    cfg, u = _ionic(n_side=8)
    h = Handle(cfg, "mixed")
    h.set_universe(u)
    for tick in range(1, 20):
        h.step(1)
        st = h.bond_observe(cfg.bond_k_bind, 0.2, tick)
    assert st["open_episodes"] > 0
    h.bond_tracker_reset()
    st = h.bond_observe(cfg.bond_k_bind, 0.2, 20)
    assert st["completed_episodes"] == 0 and st["bonds_formed"] == 0 and st["bonded_pairs"] == 0
    h.set_universe(u)
    st = h.bond_observe(cfg.bond_k_bind, 0.2, 1)
    assert st["completed_episodes"] == 0 and st["open_episodes"] == st["bound_pairs"]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _initial_bonds(orc, cfg, u):
    bonds = orc.bound_pairs(u.pos, u.elem, u.entity, cfg.size, cfg.bond_k_bind, cfg.sigma)
    return np.ascontiguousarray(bonds, dtype=np.uint32).reshape(-1, 2)


@pytest.mark.parametrize("variant", [5, 6])
def test_list_path_spring_matches_oracle(gpu, orc, variant):
    # the persistent-list passes apply the spring too (one occurrence per
    # pair: the list grid, and so the force grid, has at least 3 cells per axis)
    from genesis_b200._lib import Handle
    cfg, u = _ionic()
    bonds = _initial_bonds(orc, cfg, u)
    assert len(bonds) > 0
    h = Handle(cfg, "mixed")
    h.set_kernel_variant(variant)
    h.set_universe(u)
    h.set_bonds(bonds)
    st = h.step(1)
    assert h.list_rebuilds() >= 1  # the list path ran
    _, _, acc = h.get_state()
    _, _, acc_ref, st_ref = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, 1, bonds=bonds)
    assert _rel(acc, acc_ref) <= 1e-5
    vb, vb_ref = st["bond_energy"][0], st_ref[0, 2]
    assert vb_ref != 0.0 and abs(vb - vb_ref) <= 1e-6 * abs(vb_ref) + 1e-7


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("mixed", 1), ("mixed", 5), ("mixed", 6)])
def test_bond_count_changes_inside_captured_ticks(gpu, orc, precision, variant):
    # the spring reads the bond count on the device: captured ticks follow a
    # list that shrinks, empties and refills in place exactly as eager ticks do
    from genesis_b200._lib import Handle
    cfg, u = _ionic()
    bonds = _initial_bonds(orc, cfg, u)
    runs = []
    for graph in (False, True):
        h = Handle(cfg, precision)
        h.set_kernel_variant(variant)
        h.set_universe(u)
        sts = []
        for sel in (bonds, bonds[: len(bonds) // 2], bonds[:0], bonds[::3]):
            h.set_bonds(np.ascontiguousarray(sel))
            sts.append(h.step(4, graph=graph))
        runs.append((h.get_state(), sts))
    (s0, t0), (s1, t1) = runs
    assert np.all(t0[2]["bond_energy"] == 0.0) and np.all(t0[0]["bond_energy"] != 0.0)
    if precision == "mixed":  # order-independent fixed-point sums: bit-identical
        for x, y in zip(s0, s1):
            assert np.array_equal(x, y)
        for a, b in zip(t0, t1):
            assert np.array_equal(a, b)
    else:  # FP64 spring forces meet at an atom through atomics
        for x, y in zip(s0, s1):
            assert _rel(x, y) <= 1e-13
        for a, b in zip(t0, t1):
            assert np.allclose(a["bond_energy"], b["bond_energy"], rtol=1e-13, atol=0.0)


def test_observed_bonds_drive_the_list_path(gpu):
    # bond observation feeding the spring on the default mixed path (the
    # persistent list): captured and eager ticks agree bit for bit
    from genesis_b200._lib import Handle
    cfg, u = _ionic(n_side=8)
    out = []
    for graph in (False, True):
        h = Handle(cfg, "mixed")
        h.set_universe(u)
        most, obs = 0, []
        for tick in range(1, 81):
            h.step(1, stats=False, graph=graph)
            ob = h.bond_observe(cfg.bond_k_bind, 0.1, tick)
            most = max(most, ob["bonded_pairs"])
            obs.append(tuple(ob[k] for k in KEYS))
        assert h.list_rebuilds() >= 1 and most > 0
        out.append((h.get_state(), obs, h.get_bonds()))
    for x, y in zip(out[0][0], out[1][0]):
        assert np.array_equal(x, y)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])


def test_list_candidates_match_the_bond_grid(gpu):
    """On the mixed neighbour-list path the observation takes its candidates
    from the list; rewriting the same positions from the host (which leaves
    the list unproven for them) sends it through the bond grid instead.  Two
    handles on one NVE trajectory, one each way: the same summaries and
    bonds every tick."""
    from genesis_b200._lib import Handle
    cfg, u = _ionic()
    cfg.enable_thermostat = False  # a host rewrite voids a pending Berendsen scale
    ha, hb = Handle(cfg, "mixed"), Handle(cfg, "mixed")
    ha.set_universe(u)
    hb.set_universe(u)
    seen = 0
    for tick in range(1, 81):
        ha.step(1)
        hb.step(1)
        hb.set_dynamic(hb.get_state()[0])
        prof = tick == 30
        if prof:
            ha.profile(True)
            hb.profile(True)
        oa = ha.bond_observe(cfg.bond_k_bind, 0.2, tick)
        ob = hb.bond_observe(cfg.bond_k_bind, 0.2, tick)
        if prof:
            pa, pb = ha.profile_read(), hb.profile_read()
            ha.profile(False)
            hb.profile(False)
            assert "bound_pairs" in pa and "bond_grid" not in pa  # the list path
            assert "bond_grid" in pb
        for k in ("bound_pairs",) + KEYS:
            assert oa[k] == ob[k], (tick, k, oa[k], ob[k])
        assert np.array_equal(oa["species_matrix"], ob["species_matrix"])
        assert np.array_equal(ha.get_bonds(), hb.get_bonds()) or np.array_equal(
            np.sort(ha.get_bonds().view(np.uint64).ravel()), np.sort(hb.get_bonds().view(np.uint64).ravel()))
        assert np.array_equal(ha.get_state()[0], hb.get_state()[0])
        seen = max(seen, oa["bound_pairs"])
    assert seen > 0


def test_positions_moved_outside_a_tick_leave_the_list_out(gpu):
    """After gx_drift or gx_set_dynamic the list is not proven for the new
    positions: the observation bins the bond grid again."""
    from genesis_b200._lib import Handle
    cfg, u = _ionic()
    h = Handle(cfg, "mixed")
    h.set_universe(u)
    h.step(2)
    for tick, move in ((3, None), (4, "drift"), (5, "set_dynamic")):
        if move == "drift":
            h.drift()
        elif move == "set_dynamic":
            h.set_dynamic(h.get_state()[0])
        h.profile(True)
        h.bond_observe(cfg.bond_k_bind, 0.2, tick, apply_bonds=False)
        prof = h.profile_read()
        h.profile(False)
        assert ("bond_grid" in prof) == (move is not None), (move, sorted(prof))
