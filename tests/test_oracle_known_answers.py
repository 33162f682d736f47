"""The oracle against the reference's own known-answer and invariant tests
(tests/golden/reference_known_answers.json, each entry citing file:line)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import synth
from genesis_b200 import workloads as W
from genesis_b200.config import Config

CASES = {c["id"]: c for c in json.loads(
    (Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())["cases"]}
IDX = {s: i for i, s in enumerate(E.SYMBOLS)}


def table(orc, cfg=None):
    return orc.lj_table(cfg or Config())


def test_lj_minimum(orc):
    c = CASES["lj_minimum"]
    ps, pe, _, _ = table(orc)
    i = IDX[c["pair"][0]]
    s, e = ps[i, i], pe[i, i]
    m, v = orc.lj_raw(s, e, s * 2.0 ** (1.0 / 6.0))
    assert abs(v + e) < c["v_plus_eps_tol_rel"] * max(e, 1.0)
    assert abs(m) < c["force_abs_tol"]


def test_lj_force_sign(orc):
    c = CASES["lj_sign"]
    ps, pe, _, _ = table(orc)
    i = IDX["C"]
    s, e = ps[i, i], pe[i, i]
    assert orc.lj_raw(s, e, c["repulsive_at"] * s)[0] > 0
    assert orc.lj_raw(s, e, c["attractive_at"] * s)[0] < 0
    assert abs(orc.lj_raw(s, e, s * 2 ** (1 / 6))[0]) < c["zero_force_tol"]


def test_lb_mixing(orc):
    c = CASES["lb_mixing"]
    ps, pe, _, _ = table(orc)
    h, cc = IDX["H"], IDX["C"]
    assert ps[h, cc] == ps[cc, h] and pe[h, cc] == pe[cc, h]
    assert abs(pe[h, cc] - 0.01 * math.sqrt(12 * 80)) < c["tol"]


def test_bond_term_is_exact_derivative(orc):
    c = CASES["bond_fd"]
    k, req, ron, rc, h = c["k"], c["r_eq"], c["r_on"], c["rc"], c["h"]

    def vsw(x):
        _, v = orc.bond_harmonic_raw(k, req, x)
        sw, _ = orc.smooth_cutoff(x, ron, rc)
        return v * sw

    for r in c["r"]:
        m, v = orc.bond_harmonic_raw(k, req, r)
        sw, dsw = orc.smooth_cutoff(r, ron, rc)
        f, _ = orc.switched(m, v, sw, dsw)
        num = -(vsw(r + h) - vsw(r - h)) / (2 * h)
        assert abs(f - num) < c["tol_rel"] * max(abs(f), 1.0)


def test_switch_vanishes_at_cutoff(orc):
    c = CASES["switch_at_cutoff"]
    ps, pe, rc, ron = table(orc)
    o = IDX["O"]
    m, v = orc.force_switched_scalar(ps[o, o], pe[o, o], rc, ron, rc)
    assert m == 0.0 and v == 0.0
    r_in = c["inner_frac_of_r_on"] * ron
    m_in, _ = orc.force_switched_scalar(ps[o, o], pe[o, o], r_in, ron, rc)
    assert abs(m_in - orc.lj_raw(ps[o, o], pe[o, o], r_in)[0]) < c["tol"]


def test_well_curvature(orc):
    c = CASES["well_curvature_fd"]
    e, s, h = c["eps"], c["sigma"], c["h"]
    rm = s * 2 ** (1 / 6)
    v = lambda r: orc.lj_raw(s, e, r)[1]  # noqa: E731
    num = (v(rm + h) + v(rm - h) - 2 * v(rm)) / (h * h)
    assert abs(num - orc.well_curvature(e, s)) / num < c["tol_rel"]


def test_vib_period_order(orc):
    c = CASES["vib_period_order"]
    lo, hi = c["range"]

    def per(sym):
        i = IDX[sym]
        return orc.vib_period(0.01 * E.EPSILON_K[i], E.SIGMA[i], E.MASS[i] / 2)

    t_cc, t_hh, t_fe = per("C"), per("H"), per("Fe")
    assert lo <= t_cc < hi and lo <= t_hh < hi and lo <= t_fe < hi
    assert abs(t_cc - t_hh) > c["cc_hh_min_gap"]


def test_smooth_endpoints(orc):
    c = CASES["smooth_endpoints"]
    assert orc.smooth_cutoff(c["r_on"], c["r_on"], c["rc"]) == (1.0, 0.0)
    sw, dsw = orc.smooth_cutoff(c["rc"], c["r_on"], c["rc"])
    assert abs(sw) < c["tol"] and abs(dsw) < c["tol"]
    mid, _ = orc.smooth_cutoff(c["mid"], c["r_on"], c["rc"])
    assert 0 < mid < 1


def test_coulomb_and_gravity_values(orc):
    for case in CASES["coulomb_values"]["cases"]:
        f, v = orc.coulomb_raw(*case["args"])
        assert abs(f - case["f"]) < 1e-12
        if "v" in case:
            assert abs(v - case["v"]) < 1e-12
    c = CASES["gravity_values"]
    f, v = orc.gravity_raw(*c["args"])
    assert abs(f - c["f"]) < c["tol"] and abs(v - c["v"]) < c["tol"]


def test_element_charges():
    for sym, q in CASES["charges"]["expect"].items():
        assert E.CHARGE[IDX[sym]] == q


def test_affinity_overrides(orc):
    from genesis_b200.config import ConfigError, from_toml
    base = """
[universe]
name = "t"
size = { x = 10.0, y = 10.0, z = 10.0 }
dt = 0.02
initial_atoms = 100
stats_history = 256
[rng]
seed = 1
[physics]
initial_temperature = 300.0
speed_limit = 1000.0
gravity_constant = 6.674e-11
"""
    cfg = from_toml(base + "[physics.elements]\nNa = { sigma = 1.0, epsilon_k = 50.0 }\nO = { charge = -2.0 }\n"
                    "[systems]\nenable_electrostatics = true\n")
    na, o = IDX["Na"], IDX["O"]
    assert cfg.sigma[na] == 1.0 and cfg.epsilon_k[na] == 50.0
    ps, pe, _, _ = orc.lj_table(cfg)
    assert ps[na, na] == 1.0 and abs(pe[na, na] - 0.5) < 1e-12
    m, v = orc.lj_raw(1.0, pe[na, na], 2 ** (1 / 6))
    assert abs(v + pe[na, na]) < 1e-12 * pe[na, na]
    assert cfg.charge[o] == -2.0 and cfg.sigma[o] == E.SIGMA[o] and cfg.epsilon_k[o] == E.EPSILON_K[o]
    with pytest.raises(ConfigError, match="Faux"):
        from_toml(base + "[physics.elements]\nFaux = { charge = -2.0 }\n[systems]\n")


def _brute(pos, box, cutoff):
    out = []
    n = len(pos)
    for i in range(n):
        d = pos[i] - pos[i + 1:]
        d = d - box * np.round(d / box)
        d2 = (d * d).sum(1)
        for j in np.nonzero(d2 < cutoff * cutoff)[0]:
            out.append((i, i + 1 + j))
    return sorted(out)


def _grid_pairs(orc, pos, box, cutoff):
    p = orc.neighbors(pos, box, cutoff, cutoff)
    return sorted((int(min(a, b)), int(max(a, b))) for a, b in p)


@pytest.mark.parametrize("cid,seed", [("grid_brute_force", 1234), ("grid_degenerate_nz1", 99)])
def test_grid_matches_brute_force(orc, cid, seed):
    c = CASES[cid]
    box = np.array(c["world"])
    u = synth.uniform_box(c["npoints"], tuple(box), seed=seed)
    cutoff = 2 * c["radius"]
    if "nz" in c:
        assert orc.grid_dims(box, cutoff)[2] == c["nz"]
    assert _grid_pairs(orc, u.pos, box, cutoff) == _brute(u.pos, box, cutoff)


def test_single_cell_universe(orc):
    c = CASES["grid_single_cell"]
    pos = np.array(c["points"], dtype=float)
    box = np.array(c["world"])
    cutoff = 2 * c["radius"]
    assert _grid_pairs(orc, pos, box, cutoff) == _brute(pos, box, cutoff)


def test_min_image_across_border(orc):
    c = CASES["min_image_border"]
    d = orc.min_image(np.array(c["a"]) - np.array(c["b"]), c["size"])
    assert abs(d[0] - c["dx"]) < c["tol"] and abs((d * d).sum() - c["d2"]) < c["tol"]


def test_two_cell_axes_repeat_pairs_in_the_reference(orc):
    # Not a reference test: documents the 2-cell multiplicity the GPU reproduces.
    box = np.array([16.0, 16.0, 16.0])
    u = synth.uniform_box(200, tuple(box), seed=5)
    assert orc.grid_dims(box, 5.75) == (2, 2, 2)
    p = orc.neighbors(u.pos, box, 5.75, 5.75)
    uniq = {(int(min(a, b)), int(max(a, b))) for a, b in p}
    assert len(p) > len(uniq)
    assert sorted(uniq) == _brute(u.pos, box, 5.75)


def test_gr_pair_peak(orc):
    c = CASES["gr_pair_peak"]
    pos = np.array([[0.0, 0, 0], [c["d"], 0, 0]])
    counts, bins, rm, dr, rc = orc.radial_distribution(pos, c["world"], c["r_max"], c["nbins"])
    assert abs(dr - c["dr"]) < 1e-12
    r = (np.arange(len(bins)) + 0.5) * dr
    win = (r >= c["window"][0]) & (r <= c["window"][1])
    k = np.argmax(np.where(win, bins, -np.inf))
    assert abs(r[k] - c["d"]) < c["peak_tol"] and bins[k] > c["g_min"]


def test_gr_random_gas(orc):
    # The reference draws one gas from its rand stream (seed 7), which cannot be
    # reproduced here; the property is checked on the mean over eight seeded gases.
    c = CASES["gr_random_gas"]
    means = []
    for seed in range(1, 9):
        u = synth.uniform_box(c["npoints"], tuple(c["world"]), seed=seed)
        _, bins, _, _, _ = orc.radial_distribution(u.pos, c["world"], c["r_max"], c["nbins"])
        means.append(bins.mean())
    lo, hi = c["mean_range"]
    assert lo <= float(np.mean(means)) <= hi


def test_gr_partial(orc):
    c = CASES["gr_partial"]
    u = synth.uniform_box(c["n_h"], tuple(c["world"]), seed=11, species=(IDX["H"],))
    pos, elem = u.pos.copy(), u.elem.copy()
    pos[0] = [0, 0, 0]
    pos[1] = [c["cc_d"], 0, 0]
    elem[0] = elem[1] = IDX["C"]

    def peak(b, dr):
        r = (np.arange(len(b)) + 0.5) * dr
        w = (r >= 0.5) & (r <= 3.0)
        return b[w].max() if w.any() else 0.0

    _, g_cc, _, dr, _ = orc.radial_distribution(pos, c["world"], c["r_max"], c["nbins"], elem, (IDX["C"], IDX["C"]))
    _, g_hh, _, _, _ = orc.radial_distribution(pos, c["world"], c["r_max"], c["nbins"], elem, (IDX["H"], IDX["H"]))
    _, g_ch, _, _, _ = orc.radial_distribution(pos, c["world"], c["r_max"], c["nbins"], elem, (IDX["C"], IDX["H"]))
    assert peak(g_cc, dr) > c["g_cc_min"]
    lo, hi = c["hh_mean_range"]
    assert lo <= g_hh.mean() <= hi
    assert peak(g_cc, dr) / peak(g_ch, dr) > c["cc_over_ch_min"]
    ce = CASES["gr_partial_empty"]
    _, g, _, _, _ = orc.radial_distribution(np.array(ce["points"]), ce["world"], ce["r_max"], ce["nbins"],
                                            np.array([0, 0]), (IDX["Na"], IDX["Na"]))
    assert np.all(g == 0)


@pytest.mark.parametrize("cid", ["fof_dimers", "fof_isolated"])
def test_fof(orc, cid):
    c = CASES[cid]
    pos = np.array(c["points"], dtype=float) - 32.0  # the reference test places atoms in [0, 64)
    elem = np.zeros(len(pos), dtype=np.uint8)
    _, st = orc.clusters(pos, elem, c["world"], E.BOND_FACTOR, E.SIGMA)
    for k in ("aggregates", "monomers", "largest", "bound_pairs", "mean_size"):
        if k in c:
            assert st[k] == c[k], k


def test_fof_empty(orc):
    _, st = orc.clusters(np.zeros((0, 3)), np.zeros(0, dtype=np.uint8), [64.0] * 3, E.BOND_FACTOR, E.SIGMA)
    assert st["largest"] == 0 and st["mean_size"] == 0.0


def test_bound_pair_thresholds(orc):
    c = CASES["bound_pair_thresholds"]
    for case in c["cases"]:
        a, b = (IDX[s] for s in case["pair"])
        pos = np.array([[0.0, 0, 0], [case["d"], 0, 0]])
        got = orc.bound_pairs(pos, np.array([a, b]), None, c["world"], c["k_bind"], E.SIGMA)
        assert len(got) == case["bound"]


def _lattice(t, seed=0):
    return synth.lattice(8, 3.0, 0.02, t, 0.01, seed)


def test_nve_energy_and_momentum(orc):
    c = CASES["nve_drift"]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    u = _lattice(c["temperature"])
    p0 = (u.vel * u.mass[:, None]).sum(0)
    pos, vel, acc, st = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, c["warm"])
    e_ref = st[-1, 0] + st[-1, 1]
    pos, vel, acc, st = orc.ticks(cfg, pos, vel, acc, u.elem, u.charge, u.mass, c["ticks"])
    e1 = st[-1, 0] + st[-1, 1]
    assert abs(e1 - e_ref) / abs(e_ref) < c["energy_rel"]
    dp = np.linalg.norm((vel * u.mass[:, None]).sum(0) - p0)
    assert dp < c["momentum_rel"] * max(np.linalg.norm(p0), 1.0)


def test_nve_with_coulomb_and_gravity(orc):
    c = CASES["nve_drift_coulomb_gravity"]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    cfg.enable_electrostatics = True
    cfg.enable_gravity = True
    cfg.gravity_constant = c["gravity_constant"]
    u = _lattice(c["temperature"])
    pos, vel, acc, st = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, c["warm"])
    e_ref = st[-1, 0] + st[-1, 1]
    pos, vel, acc, st = orc.ticks(cfg, pos, vel, acc, u.elem, u.charge, u.mass, c["ticks"])
    assert abs(st[-1, 0] + st[-1, 1] - e_ref) / abs(e_ref) < c["energy_rel"]


@pytest.mark.parametrize("cid", ["thermostat_cools", "thermostat_heats"])
def test_thermostat_reaches_target(orc, cid):
    c = CASES[cid]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = c["target"]
    cfg.thermostat_tau = c["tau"]
    u = _lattice(c["t0"])
    _, vel, _, st = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, c["ticks"])
    t = (2.0 / 3.0) * (st[-1, 0] / u.n) / cfg.thermal_constant
    assert abs(t - c["target"]) < c["tol"]


def test_fixed_bond_conserves_energy(orc):
    c = CASES["fixed_bond_nve"]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    cfg.enable_bond_interaction = True
    ci = IDX["C"]
    ps, pe, _, _ = orc.lj_table(cfg)
    r_eq = ps[ci, ci] * 2 ** (1 / 6)
    half = r_eq * 0.5 + c["stretch"]
    pos = np.array([[-half, 0, 0], [half, 0, 0], [13, 13, 13], [13, 13, -13], [13, -13, 13], [13, -13, -13],
                    [-13, 13, 13], [-13, 13, -13]], dtype=float)
    elem = np.full(8, ci, dtype=np.uint8)
    mass = np.full(8, E.MASS[ci])
    vel = np.zeros_like(pos)
    bonds = np.array([[0, 1]], dtype=np.uint32)
    q = np.zeros(8)
    pos, vel, acc, _ = orc.ticks(cfg, pos, vel, None, elem, q, mass, c["relax"], bonds)

    def window(pos, vel, acc):
        pos, vel, acc, st = orc.ticks(cfg, pos, vel, acc, elem, q, mass, c["window"], bonds)
        return pos, vel, acc, (st[:, 0] + st[:, 1] + st[:, 2]).mean(), st

    pos, vel, acc, e_ref, _ = window(pos, vel, acc)
    pos, vel, acc, _ = orc.ticks(cfg, pos, vel, acc, elem, q, mass, c["gap"], bonds)
    pos, vel, acc, e_end, st = window(pos, vel, acc)
    assert abs(e_end - e_ref) / abs(e_ref) < c["energy_rel"]
    assert st[-1, 2] > 0.0


def test_threaded_forces_match_sequential(orc):
    cfg = W.C1.config()
    cfg.enable_electrostatics = True
    u = W.C1.scaled(10).generate()
    a1, v1, _, n1 = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass, nthreads=1)
    a4, v4, _, n4 = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass, nthreads=4)
    assert n1 == n4
    assert np.array_equal(a1, a4)  # per-atom sums run in pair-list order on every split
    assert abs(v1 - v4) <= 1e-12 * abs(v1)


def test_quench_bonds_appear(orc):
    """A cold quench of a 6^3 lattice jams it: persistent pairs appear within
    6,000 ticks (bond observation every tick, Berendsen to 80 K)."""
    c = CASES["quench_bonds_appear"]
    cfg = W.C1.config()
    cfg.size = tuple(c["world"])
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = c["target"]
    n_side = round(c["atoms"] ** (1.0 / 3.0))
    u = synth.lattice(n_side, c["world"][0] / n_side, 0.02, c["t0"], 0.01, 0)
    assert u.n == c["atoms"]
    tracker = orc.BondTracker(cfg)
    pos, vel, acc = u.pos, u.vel, None
    for tick in range(1, c["ticks"] + 1):
        pos, vel, acc, _ = orc.ticks(cfg, pos, vel, acc, u.elem, u.charge, u.mass, 1)
        bound = orc.bound_pairs(pos, u.elem, None, cfg.size, cfg.bond_k_bind, cfg.sigma)
        st, _ = tracker.observe(bound, u.elem, tick)
    assert st["bonded_pairs"] > 0
