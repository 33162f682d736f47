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
