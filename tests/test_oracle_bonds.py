"""The oracle's bond observation (oracle/oracle_bonds.cpp) against the
reference's own tests of PairTracker and BondObservationSystem."""
from __future__ import annotations

import numpy as np

from genesis_b200 import elements as E
from genesis_b200.config import default_config

P = [(1, 2)]  # one slot pair


def _elem(*names):
    return np.array([E.by_name(n) for n in names], dtype=np.uint8)


def test_tracker_counts_episodes_and_debounce(orc):
    # src/analysis/pairs.rs:230-263
    cfg = default_config()
    t = orc.BondTracker(cfg, debounce=1)
    elem = _elem("H", "H", "H")
    for k in range(5):
        st, _ = t.observe(P, elem, k + 1)
    st, _ = t.observe([], elem, 6)
    assert st["completed_episodes"] == 1 and st["completed_ticks"] == 5 and st["open_episodes"] == 0
    for k in range(3):
        st, _ = t.observe(P, elem, 7 + k)
    t.close_all()
    st, _ = t.observe([], elem, 10)
    assert st["completed_episodes"] == 2 and st["completed_ticks"] == 8

    t2 = orc.BondTracker(cfg, debounce=3)
    for k in range(5):
        st, _ = t2.observe(P, elem, k + 1)
    st, _ = t2.observe([], elem, 6)
    assert st["completed_episodes"] == 0 and st["open_episodes"] == 1
    t2.observe([], elem, 7)
    st, _ = t2.observe([], elem, 8)
    assert st["completed_episodes"] == 1 and st["completed_ticks"] == 5


def test_debounce_two_absorbs_a_one_tick_gap(orc):
    # src/systems/bonds.rs:210-236 (C-C at 2.0 < 1.5 * 1.9 is bound)
    cfg = default_config()
    t = orc.BondTracker(cfg, debounce=E.DEBOUNCE)
    elem = _elem("C", "C")
    for k in range(50):
        t.observe([(0, 1)], elem, k + 1)
    st, _ = t.observe([], elem, 51)
    assert st["open_episodes"] == 1
    st, _ = t.observe([], elem, 52)
    assert st["open_episodes"] == 0


def test_persistence_threshold_is_per_pair(orc):
    # src/systems/bonds.rs:238-261
    cfg = default_config()
    t = orc.BondTracker(cfg)
    h, fe = E.by_name("H"), E.by_name("Fe")
    assert t.threshold(h, h) < t.threshold(fe, fe)


def test_lifetime_and_species_matrix(orc):
    # src/systems/bonds.rs:263-341: a persistent H-H pair, then separated
    cfg = default_config()
    t = orc.BondTracker(cfg)
    elem = _elem("H", "H")
    h = E.by_name("H")
    thr = t.threshold(h, h)
    tick = 0
    for _ in range(thr + 500):
        tick += 1
        st, pers = t.observe([(0, 1)], elem, tick)
    assert st["bonded_pairs"] == 1 and st["bonds_formed"] == 0
    assert st["species_matrix"][h, h] == 2
    assert pers.tolist() == [[0, 1]]
    for _ in range(E.DEBOUNCE + 2):
        tick += 1
        st, pers = t.observe([], elem, tick)
    assert st["bonded_pairs"] == 0 and st["bonds_formed"] == 1
    assert st["lifetime_sum_ticks"] >= 400.0
    # persistent from tick thr, broken when the episode closes at thr + 502
    assert st["lifetime_sum_ticks"] == 502.0


def test_persistent_pairs_are_sorted_and_deduplicated(orc):
    cfg = default_config()
    t = orc.BondTracker(cfg, debounce=2, min_periods=0.0)  # threshold ceil(0.1 period / dt) ticks
    elem = _elem("O", "Na", "O", "Na")
    bound = [(1, 0), (0, 1), (3, 2), (2, 1)]
    for k in range(200):
        st, pers = t.observe(bound, elem, k + 1)
    assert pers.tolist() == [[0, 1], [1, 2], [2, 3]]
    assert st["bonded_entities"] == 4 and st["mean_coordination"] == 1.5
