"""Writes reference_known_answers.json: the known-answer vectors of the
reference's own unit tests for the hot path, transcribed with their file:line.

The reference is Rust and cannot run here, so its tests' inputs and expected
values are restated as data.  When the reference tree is present, each entry's
`check` token is looked up in the cited lines to catch transcription slips:

    python tests/golden/make_known_answers.py [--reference-root PATH]
"""
from __future__ import annotations

import argparse
import os
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent

CASES = [
    {"id": "lj_minimum", "cite": "src/physics/forces.rs:395-405", "check": "2.0f64.powf(1.0 / 6.0)",
     "pair": ["H", "H"], "v_plus_eps_tol_rel": 1e-12, "force_abs_tol": 1e-9},
    {"id": "lj_sign", "cite": "src/physics/forces.rs:408-420", "check": "0.8 * p.sigma",
     "pair": ["C", "C"], "repulsive_at": 0.8, "attractive_at": 1.5, "zero_force_tol": 1e-9},
    {"id": "lb_mixing", "cite": "src/physics/forces.rs:423-432", "check": "(12.0f64 * 80.0).sqrt()",
     "pair": ["H", "C"], "thermal_constant": 0.01, "eps_expected": "0.01*sqrt(12*80)", "tol": 1e-12},
    {"id": "bond_fd", "cite": "src/physics/forces.rs:435-459", "check": "[2.0, 2.1, 2.3, 2.5, 2.59]",
     "k": 5.0, "r_eq": 2.0, "r_on": 2.0, "rc": 2.6, "h": 1e-6, "r": [2.0, 2.1, 2.3, 2.5, 2.59], "tol_rel": 1e-4},
    {"id": "switch_at_cutoff", "cite": "src/physics/forces.rs:462-475", "check": "0.8 * t.r_on",
     "pair": ["O", "O"], "inner_frac_of_r_on": 0.8, "tol": 1e-12},
    {"id": "well_curvature_fd", "cite": "src/physics/forces.rs:478-490", "check": "let eps = 0.8;",
     "eps": 0.8, "sigma": 1.9, "h": 1e-5, "tol_rel": 1e-4},
    {"id": "vib_period_order", "cite": "src/physics/forces.rs:493-521", "check": "(1.0..20.0)",
     "range": [1.0, 20.0], "cc_hh_min_gap": 0.5},
    {"id": "smooth_endpoints", "cite": "src/physics/forces.rs:524-535", "check": "(2.0, 3.0)",
     "r_on": 2.0, "rc": 3.0, "mid": 2.5, "tol": 1e-12},
    {"id": "coulomb_values", "cite": "src/physics/forces.rs:538-550", "check": "-0.25",
     "cases": [{"args": [1.0, 1.0, -1.0, 2.0], "f": -0.25, "v": -0.5},
               {"args": [1.0, 1.0, 1.0, 4.0], "f": 0.0625}], "tol": 1e-12},
    {"id": "gravity_values", "cite": "src/physics/forces.rs:553-558", "check": "-1.5",
     "args": [1.0, 2.0, 3.0, 2.0], "f": -1.5, "v": -3.0, "tol": 1e-12},
    {"id": "charges", "cite": "src/physics/forces.rs:561-566", "check": "AtomType::Sodium), 1.0",
     "expect": {"Na": 1.0, "O": -1.0, "H": 0.0, "He": 0.0}},
    {"id": "override_na", "cite": "src/physics/forces.rs:569-594", "check": "epsilon_k: Some(50.0)",
     "symbol": "Na", "sigma": 1.0, "epsilon_k": 50.0, "eps_pair_expected": 0.5, "tol": 1e-12},
    {"id": "override_keeps_fields", "cite": "src/physics/forces.rs:597-613", "check": "charge: Some(-2.0)",
     "symbol": "O", "charge": -2.0},
    {"id": "grid_brute_force", "cite": "src/physics/grid.rs:342-355", "check": "Vec3::new(64.0, 64.0, 64.0)",
     "world": [64.0, 64.0, 64.0], "radius": 1.0, "npoints": 400},
    {"id": "grid_degenerate_nz1", "cite": "src/physics/grid.rs:358-375", "check": "Vec3::new(16.0, 16.0, 2.0)",
     "world": [16.0, 16.0, 2.0], "radius": 0.6, "npoints": 300, "nz": 1},
    {"id": "grid_single_cell", "cite": "src/physics/grid.rs:378-388", "check": "Vec3::new(-0.5, 1.5, 0.0)",
     "world": [3.0, 3.0, 3.0], "radius": 5.0,
     "points": [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [-0.5, 1.5, 0.0]]},
    {"id": "min_image_border", "cite": "src/physics/grid.rs:391-401", "check": "Vec3::new(31.5, 0.0, 0.0)",
     "size": [64.0, 64.0, 64.0], "a": [-31.0, 0.0, 0.0], "b": [31.5, 0.0, 0.0], "dx": 1.5, "d2": 2.25,
     "tol": 1e-9},
    {"id": "gr_pair_peak", "cite": "src/analysis/mod.rs:455-468", "check": "let d = 1.7;",
     "world": [32.0, 32.0, 32.0], "d": 1.7, "r_max": 4.0, "nbins": 400, "dr": 0.01, "window": [0.5, 3.0],
     "peak_tol": 0.03, "g_min": 1000.0},
    {"id": "gr_random_gas", "cite": "src/analysis/mod.rs:471-488", "check": "(0.8..=1.2)",
     "world": [32.0, 32.0, 32.0], "npoints": 400, "r_max": 8.0, "nbins": 32, "mean_range": [0.8, 1.2]},
    {"id": "gr_partial", "cite": "src/analysis/mod.rs:491-532", "check": "gp_cc > 500.0",
     "world": [32.0, 32.0, 32.0], "n_h": 2000, "cc_d": 1.8, "r_max": 4.0, "nbins": 400, "g_cc_min": 500.0,
     "hh_mean_range": [0.9, 1.15], "cc_over_ch_min": 100.0},
    {"id": "gr_partial_empty", "cite": "src/analysis/mod.rs:535-544", "check": "AtomType::Sodium, AtomType::Sodium",
     "world": [16.0, 16.0, 16.0], "points": [[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]], "r_max": 4.0, "nbins": 100},
    {"id": "fof_dimers", "cite": "src/analysis/mod.rs:547-567", "check": "hydrogen_at(Vec3::new(5.0, 50.0, 50.0))",
     "world": [64.0, 64.0, 64.0],
     "points": [[10, 10, 10], [12, 10, 10], [30, 10, 10], [32, 10, 10], [50, 50, 50], [5, 50, 50]],
     "aggregates": 2, "monomers": 2, "largest": 2, "bound_pairs": 2, "mean_size": 1.5},
    {"id": "fof_isolated", "cite": "src/analysis/mod.rs:570-586", "check": "hydrogen_at(Vec3::new(50.0, 50.0, 50.0))",
     "world": [64.0, 64.0, 64.0], "points": [[10, 10, 10], [50, 50, 50]], "monomers": 2, "aggregates": 0,
     "bound_pairs": 0},
    {"id": "bound_pair_thresholds", "cite": "src/analysis/pairs.rs:196-227", "check": "Vec3::new(3.3, 0.0, 0.0)",
     "world": [64.0, 64.0, 64.0], "k_bind": 1.5,
     "cases": [{"pair": ["H", "H"], "d": 2.0, "bound": 1}, {"pair": ["Si", "Si"], "d": 3.3, "bound": 1},
               {"pair": ["H", "H"], "d": 3.3, "bound": 0}]},
    {"id": "tracker_debounce", "cite": "src/analysis/pairs.rs:230-263", "check": "PairTracker::new(3)",
     "bound_ticks": 5, "rebind_ticks": 3},
    {"id": "persistence_per_pair", "cite": "src/systems/bonds.rs:238-261", "check": "t_hh < t_fefe"},
    {"id": "nve_drift", "cite": "src/systems/forces.rs:368-401", "check": "rel < 1e-3",
     "atoms": 512, "world": [24.0, 24.0, 24.0], "temperature": 100.0, "warm": 300, "ticks": 2000,
     "energy_rel": 1e-3, "momentum_rel": 1e-6},
    {"id": "nve_drift_coulomb_gravity", "cite": "src/systems/forces.rs:403-431", "check": "gravity_constant = 1e-3",
     "atoms": 512, "world": [24.0, 24.0, 24.0], "temperature": 100.0, "warm": 300, "ticks": 2000,
     "gravity_constant": 1e-3, "energy_rel": 1e-3},
    {"id": "thermostat_cools", "cite": "src/systems/thermostat.rs:94-103", "check": "hot_config(60.0)",
     "atoms": 512, "world": [24.0, 24.0, 24.0], "t0": 300.0, "target": 60.0, "tau": 10.0, "ticks": 2500, "tol": 10.0},
    {"id": "thermostat_heats", "cite": "src/systems/thermostat.rs:105-116", "check": "hot_config(180.0)",
     "atoms": 512, "world": [24.0, 24.0, 24.0], "t0": 20.0, "target": 180.0, "tau": 10.0, "ticks": 2500, "tol": 10.0},
    {"id": "fixed_bond_nve", "cite": "src/systems/forces.rs:453-538", "check": "r_eq * 0.5 + 0.15",
     "world": [32.0, 32.0, 32.0], "stretch": 0.15, "relax": 100, "window": 100, "gap": 1500, "energy_rel": 1e-3},
    {"id": "quench_bonds_appear", "cite": "src/systems/forces.rs:433-451", "check": "u.run_ticks(6000);",
     "atoms": 216, "world": [24.0, 24.0, 24.0], "t0": 300.0, "target": 80.0, "ticks": 6000},
]


def verify(root: Path) -> list[str]:
    bad = []
    for c in CASES:
        path, span = c["cite"].split(":")
        lo, hi = (int(x) for x in span.split("-"))
        lines = (root / path).read_text().splitlines()[lo - 1:hi]
        if c["check"] not in "\n".join(lines):
            bad.append(f"{c['id']}: `{c['check']}` not found in {c['cite']}")
    return bad


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=os.environ.get("GENESIS_REFERENCE_ROOT"),
                    help="checkout of the reference repository whose text each citation is checked "
                         "against (or set GENESIS_REFERENCE_ROOT)")
    a = ap.parse_args()
    if not a.reference_root:
        raise SystemExit("give --reference-root or set GENESIS_REFERENCE_ROOT")
    root = Path(a.reference_root)
    bad = verify(root)
    if bad:
        raise SystemExit("\n".join(bad))
    (HERE / "reference_known_answers.json").write_text(json.dumps({"cases": CASES}, indent=1) + "\n")


if __name__ == "__main__":
    main()
