"""The oracle's CollisionSystem (orc_collisions) against the reference's
elastic_pair tests (src/physics/collision.rs:35-100), through two-particle
states whose normal is the one those tests use."""
from __future__ import annotations

import numpy as np

from genesis_b200.config import default_config


def _cfg():
    cfg = default_config()
    cfg.size = (32.0, 32.0, 32.0)
    cfg.enable_collisions = True
    return cfg


def test_equal_masses_swap_velocities(orc):
    # particle 1 at the origin, particle 2 to its right: n = (p1 - p2)/d = (-1, 0, 0)
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0]])
    vel = np.array([[1.0, 0.0, 0.0], [-1.0, 0.0, 0.0]])
    v, c = orc.collisions(_cfg(), pos, vel, np.array([1.0, 1.0]))
    assert c == 1 and v.tolist() == [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]]


def test_conserves_momentum_and_energy(orc):
    m = np.array([1.0, 3.0])
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0]])
    vel = np.array([[2.0, -1.0, 0.5], [0.0, 1.0, -0.5]])
    v, c = orc.collisions(_cfg(), pos, vel, m)
    assert c == 1 and not np.array_equal(v, vel)
    p0, p1 = (vel * m[:, None]).sum(0), (v * m[:, None]).sum(0)
    assert np.linalg.norm(p0 - p1) < 1e-12
    e0 = 0.5 * (m * (vel ** 2).sum(1)).sum()
    e1 = 0.5 * (m * (v ** 2).sum(1)).sum()
    assert abs(e0 - e1) < 1e-12


def test_separating_and_massless_pairs_do_not_impulse(orc):
    pos = np.array([[0.5, 0.0, 0.0], [0.0, 0.0, 0.0]])  # n = (+1, 0, 0)
    vel = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])  # vrel . n > 0: separating
    v, c = orc.collisions(_cfg(), pos, vel, np.array([1.0, 1.0]))
    assert c == 0 and np.array_equal(v, vel)
    vel = np.array([[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    v, c = orc.collisions(_cfg(), pos, vel, np.array([0.0, 1.0]))
    assert c == 0 and np.array_equal(v, vel)


def test_out_of_contact_pairs_do_not_collide(orc):
    cfg = _cfg()
    pos = np.array([[0.0, 0.0, 0.0], [2.0 * cfg.particle_radius + 1e-9, 0.0, 0.0]])
    vel = np.array([[1.0, 0.0, 0.0], [-1.0, 0.0, 0.0]])
    v, c = orc.collisions(cfg, pos, vel, np.array([1.0, 1.0]))
    assert c == 0 and np.array_equal(v, vel)
