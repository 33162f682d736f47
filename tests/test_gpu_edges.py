"""Edge cases of the boundary on the GPU: an empty universe (ForceSystem::run
returns without work when N = 0, src/systems/forces.rs:201-203), one atom
(no pair), and one pair against the oracle in both precisions."""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cfg():
    cfg = W.C1.config()
    cfg.enable_electrostatics = True
    return cfg


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_empty_universe_steps_without_work(gpu, precision):
    from genesis_b200._lib import Handle
    z = np.zeros((0, 3))
    with Handle(_cfg(), precision) as h:
        h.set_state(z, z, np.zeros(0, dtype=np.uint8))
        V, Vb, npairs = h.forces()
        assert (V, Vb, npairs) == (0.0, 0.0, 0)
        st = h.step(3, graph=True)
        assert np.all(st["kinetic"] == 0.0) and np.all(st["pairs"] == 0)
        pos, vel, acc = h.get_state()
        assert pos.shape == (0, 3) and vel.shape == (0, 3) and acc.shape == (0, 3)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_one_atom_feels_no_force(gpu, precision):
    from genesis_b200._lib import Handle
    pos = np.array([[1.0, -2.0, 3.0]])
    vel = np.array([[0.1, 0.2, -0.3]])
    with Handle(_cfg(), precision) as h:
        h.set_state(pos, vel, np.array([E.by_name("Na")], dtype=np.uint8))
        V, _, npairs = h.forces()
        _, _, acc = h.get_state()
    assert V == 0.0 and npairs == 0
    assert np.array_equal(acc, np.zeros((1, 3)))


@pytest.mark.parametrize("precision,rel", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_one_pair_matches_the_oracle(gpu, orc, precision, rel):
    from genesis_b200._lib import Handle
    cfg = _cfg()
    pos = np.array([[0.3, 0.1, -0.2], [3.1, 0.4, 0.5]])
    elem = np.array([E.by_name("Na"), E.by_name("O")], dtype=np.uint8)
    charge = np.array([E.CHARGE[e] for e in elem])
    mass = np.array([E.MASS[e] for e in elem])
    with Handle(cfg, precision) as h:
        h.set_state(pos, np.zeros_like(pos), elem, charge=charge, mass=mass)
        V, _, npairs = h.forces()
        _, _, acc = h.get_state()
    a_ref, V_ref, _, np_ref = orc.forces(cfg, pos, elem, charge, mass)
    assert npairs == np_ref == 1
    assert np.linalg.norm(acc - a_ref) <= rel * np.linalg.norm(a_ref)
    assert abs(V - V_ref) <= rel * abs(V_ref)
    f = acc * mass[:, None]  # Newton's third law: the pair's forces cancel
    assert np.linalg.norm(f.sum(0)) <= 1e-12 * np.linalg.norm(f)
