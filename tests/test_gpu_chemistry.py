"""The bond-graph chemistry lens on the device (gx_bond_components) and in
the System mirror (bond-structure) against the oracle's restatement
(oracle/chemistry.py): component labels exactly, each bond's raw energy
bit for bit, the ChemicalStructure resource at every sample."""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _ionic(n_side=8, temperature=300.0):
    wl = W.Workload("chem check", n_side=n_side, temperature=temperature, steps=10, seed=5, electrostatics=True,
                    thermostat=True, thermostat_temperature=temperature, bond_observation=True,
                    bond_interaction=True, species=(E.by_name("Na"), E.by_name("O")),
                    fixed_fractions={E.by_name("Na"): 0.5, E.by_name("O"): 0.5})
    return wl.config(), wl.generate()


def _oracle_labels(n, bonds):
    from oracle import chemistry as X
    lab = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
    ents = sorted({int(a) for a, b in bonds} | {int(b) for a, b in bonds})
    for c in X.bond_components([(e, 0) for e in ents], [(int(a), int(b)) for a, b in bonds]):
        lab[c["members"]] = min(c["members"])
    return lab


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_components_and_bond_energies_match_oracle(gpu, orc, precision):
    from genesis_b200._lib import Handle
    from oracle import chemistry as X
    cfg, u = _ionic(10)
    h = Handle(cfg, precision)
    h.set_universe(u)
    h.step(5)
    pos = h.get_state()[0]
    bonds = orc.bound_pairs(pos, u.elem, u.entity, cfg.size, cfg.bond_k_bind, cfg.sigma)
    h.set_bonds(np.ascontiguousarray(bonds, dtype=np.uint32))
    labels, energy = h.bond_components()
    assert len(bonds) > 100 and np.array_equal(labels, _oracle_labels(u.n, bonds))
    want = np.array([X.pair_potential_raw(cfg.sigma, cfg.epsilon_k, cfg.charge, cfg.thermal_constant,
                                          int(u.elem[a]), int(u.elem[b]), X.pair_distance(pos[a], pos[b], cfg.size),
                                          cfg.coulomb_constant, cfg.enable_electrostatics,
                                          cfg.enable_bond_interaction) for a, b in h.get_bonds()])
    assert np.array_equal(energy, want)


def test_no_bonds_gives_only_monomers(gpu):
    from genesis_b200._lib import Handle
    cfg, u = _ionic(6)
    h = Handle(cfg, "fp64")
    h.set_universe(u)
    labels, energy = h.bond_components()
    assert np.all(labels == 0xFFFFFFFF) and len(energy) == 0


def test_bond_structure_system_matches_oracle_lens(gpu):
    from genesis_b200.systems import GpuUniverse
    from oracle import chemistry as X
    cfg, u = _ionic(8)
    cfg.bond_min_periods = 0.1
    cfg.structure_interval = 20
    gu = GpuUniverse(cfg, u, "fp64")
    ref = X.BondStructure()
    seen_aggregates = 0
    for _ in range(6):
        gu.run_ticks(20)
        w = gu.sync()
        cs = gu.resources["ChemicalStructure"]
        bonds = [(int(a), int(b)) for a, b in gu.gpu.h.get_bonds()]
        want = ref.sample(u.n, u.elem, bonds, w.pos, cfg)
        for k in ("aggregates", "bound_entities", "monomers", "largest", "appeared", "disappeared", "fusions",
                  "scissions", "reactions"):
            assert cs[k] == want[k], (k, cs[k], want[k])
        assert [c[:2] for c in cs["compositions"]] == [c[:2] for c in want["compositions"]]
        for g, r in zip(cs["compositions"], want["compositions"]):
            assert g[2] == pytest.approx(r[2], rel=1e-12, abs=1e-12)
        seen_aggregates = max(seen_aggregates, cs["aggregates"])
    assert seen_aggregates > 0  # bonds persisted and formed aggregates during the run
