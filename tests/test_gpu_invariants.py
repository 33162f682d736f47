"""The reference's system-level invariant tests, run on the GPU paths.

ForceSystem's NVE tests (src/systems/forces.rs:369-431: energy drift below
1e-3 relative and momentum drift below 1e-6 over 2,000 ticks after 300
warm-up ticks, 512 atoms in a 24^3 box, LJ alone and LJ + Coulomb + gravity)
and ThermostatSystem's (src/systems/thermostat.rs:95-116: Berendsen brings
the system to 60 +- 10 K and to 180 +- 10 K in 2,500 ticks), with the sizes
and thresholds transcribed in tests/golden/reference_known_answers.json.
The reference's rand stream cannot be reproduced, so the atoms come from this
project's lattice generator, as in the oracle's versions of these tests.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from genesis_b200 import synth
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = {c["id"]: c for c in json.loads(
    (Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())["cases"]}


def _lattice(t, seed=0):
    return synth.lattice(8, 3.0, 0.02, t, 0.01, seed)


def _nve(cid, precision, coul_grav=False):
    from genesis_b200._lib import Handle
    c = CASES[cid]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    if coul_grav:
        cfg.enable_electrostatics = True
        cfg.enable_gravity = True
        cfg.gravity_constant = c["gravity_constant"]
    u = _lattice(c["temperature"])
    assert u.n == c["atoms"]
    with Handle(cfg, precision) as h:
        h.set_universe(u)
        st = h.step(c["warm"], graph=True)
        e_ref = st["kinetic"][-1] + st["potential"][-1]
        st = h.step(c["ticks"], graph=True)
        e1 = st["kinetic"][-1] + st["potential"][-1]
        _, vel, _ = h.get_state()
    return c, u, e_ref, e1, vel


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_nve_energy_and_momentum(gpu, precision):
    c, u, e_ref, e1, vel = _nve("nve_drift", precision)
    assert abs(e1 - e_ref) / abs(e_ref) < c["energy_rel"]
    p0 = (u.vel * u.mass[:, None]).sum(0)
    dp = np.linalg.norm((vel * u.mass[:, None]).sum(0) - p0)
    assert dp < c["momentum_rel"] * max(np.linalg.norm(p0), 1.0)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_nve_with_coulomb_and_gravity(gpu, precision):
    c, _, e_ref, e1, _ = _nve("nve_drift_coulomb_gravity", precision, coul_grav=True)
    assert abs(e1 - e_ref) / abs(e_ref) < c["energy_rel"]


@pytest.mark.parametrize("cid", ["thermostat_cools", "thermostat_heats"])
def test_thermostat_reaches_target(gpu, cid):
    from genesis_b200._lib import Handle
    c = CASES[cid]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = c["target"]
    cfg.thermostat_tau = c["tau"]
    u = _lattice(c["t0"])
    with Handle(cfg, "mixed") as h:
        h.set_universe(u)
        st = h.step(c["ticks"], graph=True)
    t = (2.0 / 3.0) * (st["kinetic"][-1] / u.n) / cfg.thermal_constant
    assert abs(t - c["target"]) < c["tol"]
