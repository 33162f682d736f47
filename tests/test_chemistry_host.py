"""The chemistry lens's host side (genesis_b200/chemistry.py) against the
oracle's restatement of BondStructureSystem, fed the same labels and bond
energies the device produces (computed here by the oracle)."""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import chemistry as G
from genesis_b200.config import default_config
from oracle import chemistry as X


def _labels(n, bonds):
    lab = np.full(n, G.NO_COMPONENT, dtype=np.uint32)
    ents = sorted({a for a, b in bonds} | {b for a, b in bonds})
    for c in X.bond_components([(e, 0) for e in ents], bonds):
        lab[c["members"]] = min(c["members"])
    return lab


def _energies(bonds, elem, pos, cfg):
    return np.array([X.pair_potential_raw(cfg.sigma, cfg.epsilon_k, cfg.charge, cfg.thermal_constant, int(elem[a]),
                                          int(elem[b]), X.pair_distance(pos[a], pos[b], cfg.size),
                                          cfg.coulomb_constant, cfg.enable_electrostatics,
                                          cfg.enable_bond_interaction) for a, b in bonds])


def _random_graph(rng, n, m):
    bonds = []
    while len(bonds) < m:
        a, b = rng.integers(0, n, 2)
        if a != b:
            bonds.append((int(min(a, b)), int(max(a, b))))
    return bonds


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_lens_matches_oracle_over_samples(seed):
    rng = np.random.default_rng(seed)
    cfg = default_config()
    cfg.enable_electrostatics = True
    cfg.enable_bond_interaction = True
    n = 60
    elem = rng.integers(0, 10, n)
    lens, ref = G.BondStructureLens(), X.BondStructure()
    bonds = _random_graph(rng, n, 25)
    for step in range(6):
        pos = rng.uniform(-60, 60, (n, 3))
        # evolve the graph: drop some bonds, add some (fusions and scissions happen)
        if step:
            keep = [b for b in bonds if rng.random() > 0.3]
            bonds = keep + _random_graph(rng, n, 8)
        got = lens.sample(_labels(n, bonds), elem, np.array(bonds), _energies(bonds, elem, pos, cfg), n)
        want = ref.sample(n, elem, bonds, pos, cfg)
        for k in ("aggregates", "bound_entities", "monomers", "largest", "appeared", "disappeared", "fusions",
                  "scissions", "reactions"):
            assert got[k] == want[k], (step, k, got[k], want[k])
        assert [c[:2] for c in got["compositions"]] == [c[:2] for c in want["compositions"]]
        for g, w in zip(got["compositions"], want["compositions"]):
            assert g[2] == pytest.approx(w[2], rel=1e-12, abs=1e-12)


def test_duplicate_and_reversed_bonds_count_once():
    cfg = default_config()
    elem = np.array([5, 4, 5, 4])
    pos = np.array([[0.0, 0, 0], [2.0, 0, 0], [5.0, 0, 0], [7.0, 0, 0]])
    bonds = [(0, 1), (1, 0), (2, 3), (0, 1)]
    e = _energies(bonds, elem, pos, cfg)
    got = G.BondStructureLens().sample(_labels(4, bonds), elem, np.array(bonds), e, 4)
    assert got["compositions"] == [("Na-O", 2, pytest.approx((e[0] + e[2]) / 2, rel=1e-15))]


def test_no_bonds_is_all_monomers():
    got = G.BondStructureLens().sample(np.full(5, G.NO_COMPONENT, dtype=np.uint32), np.zeros(5, dtype=int),
                                       np.zeros((0, 2)), np.zeros(0), 5)
    assert got["aggregates"] == 0 and got["monomers"] == 5 and got["largest"] == 0 and got["compositions"] == []
