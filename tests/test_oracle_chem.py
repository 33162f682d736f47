"""The oracle's bond-graph chemistry lens (oracle/chemistry.py) against the
reference's own tests of bond_components / formula
(src/analysis/mod.rs:588-681) and BondStructureSystem
(src/systems/bond_structure.rs:268-411)."""
from __future__ import annotations

import numpy as np

from genesis_b200 import elements as E
from genesis_b200.config import default_config
from oracle import chemistry as X

H, C, O, NA, FE, S = (E.by_name(s) for s in ("H", "C", "O", "Na", "Fe", "S"))


def test_dimers_and_their_compositions():
    comps = X.bond_components([(0, H), (1, H), (2, NA), (3, O)], [(0, 1), (2, 3)])
    assert len(comps) == 2 and all(c["size"] == 2 for c in comps)
    assert comps[0]["formula"] == "H2" and comps[1]["formula"] == "Na-O"


def test_chain_has_stoichiometry():
    comps = X.bond_components([(0, NA), (1, O), (2, NA)], [(0, 1), (1, 2)])
    assert len(comps) == 1 and comps[0]["size"] == 3 and comps[0]["formula"] == "Na2-O"


def test_duplicates_and_dangling_edges_are_ignored():
    comps = X.bond_components([(0, H), (1, H)], [(0, 1), (1, 0), (7, 0), (9, 9)])
    assert len(comps) == 1 and comps[0]["formula"] == "H2" and comps[0]["size"] == 2


def test_cycle_is_one_component_and_empty_graph_is_empty():
    comps = X.bond_components([(0, C), (1, C), (2, C)], [(0, 1), (1, 2), (2, 0)])
    assert len(comps) == 1 and comps[0]["size"] == 3 and comps[0]["formula"] == "C3"
    assert X.bond_components([], []) == []


def test_formula_orders_multiplicity_then_symbol():
    comp = [0] * 10
    comp[H], comp[C] = 6, 2
    assert X.formula(comp) == "H6-C2"
    comp = [0] * 10
    comp[NA], comp[O] = 2, 1
    assert X.formula(comp) == "Na2-O"
    comp = [0] * 10
    comp[FE], comp[S] = 1, 2
    assert X.formula(comp) == "S2-Fe"


def _two_dimers_and_monomer():
    elem = np.array([NA, O, NA, O, NA])
    pos = np.array([[0.0, 0, 0], [2.0, 0, 0], [5.0, 0, 0], [7.0, 0, 0], [10.0, 0, 0]])
    return elem, pos, [(0, 1), (2, 3)]


def _fused_ring():
    elem = np.array([NA, O, NA, O, NA])
    pos = np.array([[0.0, 0, 0], [1.2, 0, 0], [5.0, 0, 0], [6.2, 0, 0], [10.0, 0, 0]])
    return elem, pos, [(0, 1), (1, 2), (2, 3), (0, 3)]


def test_first_sample_records_new_aggregates_with_negative_binding():
    cfg = default_config()
    cfg.enable_bond_observation = True
    cfg.enable_electrostatics = True
    elem, pos, bonds = _two_dimers_and_monomer()
    cs = X.BondStructure().sample(5, elem, bonds, pos, cfg)
    assert (cs["aggregates"], cs["monomers"], cs["largest"]) == (2, 1, 2)
    assert (cs["appeared"], cs["disappeared"], cs["fusions"]) == (2, 0, 0)
    na_o = [c for c in cs["compositions"] if c[0] == "Na-O"][0]
    assert na_o[1] == 2 and na_o[2] < 0.0


def test_affinity_table_tunes_binding_energy():
    cfg = default_config()
    charged = X.pair_potential_raw(cfg.sigma, cfg.epsilon_k, cfg.charge, 0.01, NA, O, 2.0, 1.0, True, False)
    q = list(cfg.charge)
    q[NA] = q[O] = 0.0
    neutral = X.pair_potential_raw(cfg.sigma, cfg.epsilon_k, q, 0.01, NA, O, 2.0, 1.0, True, False)
    assert charged < neutral < 0.0


def test_fusion_from_dimers_to_ring():
    cfg = default_config()
    cfg.enable_bond_observation = True
    lens = X.BondStructure()
    e, p, b = _two_dimers_and_monomer()
    assert lens.sample(5, e, b, p, cfg)["appeared"] == 2
    e, p, b = _fused_ring()
    cs = lens.sample(5, e, b, p, cfg)
    assert (cs["aggregates"], cs["disappeared"], cs["appeared"], cs["fusions"]) == (1, 2, 1, 1)
    assert cs["reactions"] == [(["Na-O", "Na-O"], ["Na2-O2"], 1)]


def test_scission_from_ring_to_dimers():
    cfg = default_config()
    cfg.enable_bond_observation = True
    lens = X.BondStructure()
    e, p, b = _fused_ring()
    assert lens.sample(5, e, b, p, cfg)["aggregates"] == 1
    e, p, b = _two_dimers_and_monomer()
    cs = lens.sample(5, e, b, p, cfg)
    assert (cs["aggregates"], cs["disappeared"], cs["appeared"], cs["scissions"]) == (2, 1, 2, 1)
    assert cs["reactions"] == [(["Na2-O2"], ["Na-O", "Na-O"], 1)]


def test_min_image_rounds_half_away_from_zero():
    assert X._round_half_away(0.5) == 1.0 and X._round_half_away(-0.5) == -1.0
    assert X._round_half_away(0.49999999999999994) == 0.0
    assert X.pair_distance([0.0, 0, 0], [9.0, 0, 0], (10.0, 10.0, 10.0)) == 1.0
