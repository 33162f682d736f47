"""The System/Scheduler mirror (genesis_b200/systems.py) on the GPU: the
reference's force schedule (src/universe/mod.rs:355-392) run through the
C ABI, against the oracle running the same ticks.

FP64 path: states within 1e-10 relative after the run (the per-atom sums
run in a different order than the reference's pair list, 1e-16 per tick);
the bond observation summary, whose persistent pairs feed the next tick's
spring on both sides, exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_schedule_order_matches_build_schedule(gpu):
    from genesis_b200.systems import GpuUniverse
    cfg = W.C2.scaled(6).config()
    gu = GpuUniverse(cfg, W.C2.scaled(6).generate(), "fp64")
    # build_schedule's order (src/universe/mod.rs:355-392)
    assert gu.scheduler.names() == ["velocity_half_kick", "position_drift", "boundary", "forces",
                                    "velocity_half_kick", "thermostat", "bond-observation", "bond-structure",
                                    "structure", "stats"]


def test_plain_schedule_matches_oracle_ticks(gpu, orc):
    from genesis_b200.systems import GpuUniverse
    wl = W.C1.scaled(10)
    cfg, u = wl.config(), wl.generate()
    gu = GpuUniverse(cfg, u, "fp64")
    gu.run_ticks(20)
    w = gu.sync()
    pos, vel, acc, st = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, 20)
    assert _rel(w.pos, pos) <= 1e-10 and _rel(w.vel, vel) <= 1e-10 and _rel(w.acc, acc) <= 1e-10
    assert abs(gu.resources["PotentialEnergy"] - st[-1, 1]) <= 1e-10 * abs(st[-1, 1])


def test_ionic_schedule_with_bond_observation_matches_oracle(gpu, orc):
    from genesis_b200.systems import GpuUniverse
    wl = W.Workload("ionic check", n_side=8, temperature=300.0, steps=10, seed=5, electrostatics=True,
                    thermostat=True, thermostat_temperature=300.0, bond_observation=True, bond_interaction=True,
                    species=(E.by_name("Na"), E.by_name("O")),
                    fixed_fractions={E.by_name("Na"): 0.5, E.by_name("O"): 0.5})
    cfg, u = wl.config(), wl.generate()
    cfg.bond_min_periods = 0.1  # the floor: Na-O persists after ~32 ticks, so the spring acts in the run
    ticks = 80
    gu = GpuUniverse(cfg, u, "fp64")
    gu.run_ticks(ticks)
    w = gu.sync()
    # the oracle: one tick of the force schedule with the bonds observed on the
    # previous tick, then the observation of this tick
    tr = orc.BondTracker(cfg, debounce=E.DEBOUNCE)
    pos, vel, acc = u.pos, u.vel, np.zeros_like(u.pos)
    bonds = np.zeros((0, 2), dtype=np.uint32)
    most = 0
    for t in range(1, ticks + 1):
        pos, vel, acc, st = orc.ticks(cfg, pos, vel, acc, u.elem, u.charge, u.mass, 1, bonds=bonds)
        bp = orc.bound_pairs(pos, u.elem, u.entity, cfg.size, cfg.bond_k_bind, cfg.sigma)
        obs, bonds = tr.observe(bp, u.elem, t)
        most = max(most, len(bonds))
    assert _rel(w.pos, pos) <= 1e-10 and _rel(w.vel, vel) <= 1e-10
    bo = gu.resources["BondObservation"]
    for k in ("bonded_pairs", "bonded_entities", "mean_coordination", "bonds_formed", "lifetime_sum_ticks"):
        assert bo[k] == obs[k], (k, bo[k], obs[k])
    assert np.array_equal(bo["species_matrix"], obs["species_matrix"])
    assert most > 0  # the spring acted on observed bonds during the run
    n_host = sum(len(v) for v in w.bonds.values())
    assert n_host == 2 * obs["bonded_pairs"]


def test_stats_snapshot_csv_rows_and_frames(gpu, orc, tmp_path):
    """StatsSystem's full snapshot from the GPU schedule, written as the
    metrics CSV (export::append_csv) every tick and as an XYZ frame."""
    from genesis_b200 import export as X
    from genesis_b200.systems import GpuUniverse
    wl = W.Workload("ionic csv", n_side=8, temperature=300.0, steps=10, seed=5, electrostatics=True,
                    thermostat=True, thermostat_temperature=300.0, bond_observation=True, bond_interaction=True,
                    species=(E.by_name("Na"), E.by_name("O")),
                    fixed_fractions={E.by_name("Na"): 0.5, E.by_name("O"): 0.5})
    cfg, u = wl.config(), wl.generate()
    cfg.bond_min_periods = 0.1
    cfg.structure_interval = 10
    gu = GpuUniverse(cfg, u, "fp64")
    nsys = len(gu.scheduler.systems)
    path = tmp_path / "metrics.csv"
    for t in range(1, 41):
        gu.tick()
        gu.append_csv(path)
        s = gu.stats.snapshot
        assert s["tick"] == t and s["entities"] == len(u.elem) and s["systems_run"] == (t - 1) * nsys
        assert abs(s["time"] - t * cfg.dt) <= 1e-12 * t
        assert s["energy_total"] == s["kinetic"] + s["energy_potential"] + s["bond_energy"]
        assert (s["structure"] is not None) == (t >= 10) and (s["chemical"] is not None) == (t >= 10)
    lines = path.read_text().splitlines()
    assert lines[0] == X.CSV_HEADER and len(lines) == 41
    assert all(len(r.split(",")) == 30 for r in lines[1:])
    assert lines[-1] == X.csv_row(gu.stats.snapshot)
    last = lines[-1].split(",")
    assert last[0] == "40" and last[2] == str(len(u.elem)) and int(last[18]) == gu.stats.snapshot["bonded_pairs"]
    assert len(gu.stats.history) == 40
    frame = gu.write_frame(tmp_path / "frame")
    assert frame.endswith("frame_00000040.xyz")
    w = gu.sync()
    assert open(frame, "rb").read() == orc.xyz_frame(40, w.pos, w.elem)
