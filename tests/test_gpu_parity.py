"""Parity of the sm_100a path against the CPU oracle, through the C ABI.

Bit-exact: cell assignment, neighbour pair multisets, bound pairs, FoF labels,
g(r) bin counts, kick/drift/wrap.  FP64 path: forces, energies, K and lambda
within 1e-12 relative (norm-wise for vectors).  Mixed path: force relative RMS
<= 1e-5 (the mixed path's accuracy bound), deterministic across runs.
"""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import synth
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
MIXED_RMS = 1e-5


def _handle(cfg, precision="fp64"):
    from genesis_b200._lib import Handle
    return Handle(cfg, precision)


def _pairset(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    a = np.minimum(p[:, 0], p[:, 1])
    b = np.maximum(p[:, 0], p[:, 1])
    key = a * (1 << 32) + b
    return np.sort(key)


def _relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _c1(n_side=16, **kw):
    wl = W.C1.scaled(n_side)
    for k, v in kw.items():
        setattr(wl, k, v)
    return wl, wl.config(), wl.generate()


def _small_ionic(n_side=10):
    wl = W.C2.scaled(n_side)
    return wl, wl.config(), wl.generate()


# ---------------------------------------------------------------- bit-exact grid


@pytest.mark.parametrize("min_cell", [5.75, 3.45, 17.25, 1.0])
def test_cell_assignment_bit_exact(gpu, orc, min_cell):
    wl, cfg, u = _c1()
    h = _handle(cfg)
    h.set_universe(u)
    got = h.cell_assign(min_cell)
    ref = orc.cell_of(u.pos, cfg.size, min_cell)
    assert np.array_equal(got, ref)


def _boxes():
    # (box, min_cell, cutoff, npoints): the force grid, a 2-cell axis (the
    # reference reports such pairs more than once), nz = 1, a single cell.
    return [((44.16, 44.16, 44.16), 5.75, 5.75, 4096),
            ((16.0, 16.0, 16.0), 5.75, 5.75, 600),
            ((16.0, 16.0, 2.0), 1.2, 1.2, 300),
            ((3.0, 3.0, 3.0), 10.0, 10.0, 40),
            ((24.0, 13.0, 30.0), 4.0, 4.0, 900)]


@pytest.mark.parametrize("case", range(5))
def test_neighbor_multiset_bit_exact(gpu, orc, case):
    box, min_cell, cutoff, npts = _boxes()[case]
    u = synth.uniform_box(npts, box, seed=1234 + case)
    cfg = W.C1.config()
    cfg.size = box
    h = _handle(cfg)
    h.set_universe(u)
    ref = orc.neighbors(u.pos, box, min_cell, cutoff)
    got = h.neighbors(min_cell, cutoff, cap=len(ref) + 16)
    assert len(got) == len(ref)
    assert np.array_equal(_pairset(got), _pairset(ref))


def test_two_cell_axis_repeats_pairs(gpu, orc):
    # dims (2,2,2): the reference's canonical-offset filter reports cross-cell
    # pairs twice; the GPU enumeration must do the same.
    box = (16.0, 16.0, 16.0)
    u = synth.uniform_box(200, box, seed=5)
    ref = orc.neighbors(u.pos, box, 5.75, 5.75)
    uniq = np.unique(_pairset(ref))
    assert len(ref) > len(uniq)
    cfg = W.C1.config()
    cfg.size = box
    h = _handle(cfg)
    h.set_universe(u)
    assert np.array_equal(_pairset(h.neighbors(5.75, 5.75)), _pairset(ref))


# ---------------------------------------------------------------- integrator


def test_kick_drift_wrap_bit_exact(gpu, orc):
    wl, cfg, u = _c1()
    rng = np.random.default_rng(3)
    acc = rng.normal(size=u.pos.shape)
    h = _handle(cfg)
    h.set_universe(u, acc=acc)
    h.half_kick()
    v_ref = orc.half_kick(u.vel, acc, cfg.dt)
    pos, vel, a = h.get_state()
    assert np.array_equal(vel, v_ref)
    h.drift()
    p_ref = orc.drift(u.pos, v_ref, cfg.dt)
    pos, vel, a = h.get_state()
    assert np.array_equal(pos, p_ref)
    h.wrap()
    w_ref = orc.wrap(p_ref, cfg.size)
    pos, vel, a = h.get_state()
    assert np.array_equal(pos, w_ref)


def test_thermostat_matches(gpu, orc):
    wl, cfg, u = _c1()
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 20.0
    h = _handle(cfg)
    h.set_universe(u)
    K, lam = h.thermostat()
    v_ref, K_ref, lam_ref, applied = orc.thermostat(u.vel, u.mass, cfg.thermal_constant, 20.0, cfg.thermostat_tau)
    assert applied
    assert abs(K - K_ref) <= FP64_REL * abs(K_ref)
    assert abs(lam - lam_ref) <= FP64_REL * abs(lam_ref)
    _, vel, _ = h.get_state()
    assert _relnorm(vel, v_ref) <= FP64_REL


# ---------------------------------------------------------------- force pass


def test_forces_fp64_c1(gpu, orc):
    wl, cfg, u = _c1()
    h = _handle(cfg)
    h.set_universe(u)
    V, Vb, npairs = h.forces()
    acc_ref, V_ref, Vb_ref, np_ref = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass)
    _, _, acc = h.get_state()
    assert npairs == np_ref
    assert _relnorm(acc, acc_ref) <= FP64_REL
    assert abs(V - V_ref) <= FP64_REL * abs(V_ref)
    assert Vb == 0.0


def test_forces_fp64_ionic_with_bonds(gpu, orc):
    wl, cfg, u = _small_ionic()
    bp = orc.bound_pairs(u.pos, u.elem, None, cfg.size, cfg.bond_k_bind, cfg.sigma)
    bonds = np.unique(np.sort(bp, axis=1), axis=0)
    assert len(bonds) > 0
    h = _handle(cfg)
    h.set_universe(u)
    h.set_bonds(bonds)
    V, Vb, npairs = h.forces()
    acc_ref, V_ref, Vb_ref, np_ref = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass, bonds)
    _, _, acc = h.get_state()
    assert npairs == np_ref
    assert _relnorm(acc, acc_ref) <= FP64_REL
    assert abs(V - V_ref) <= FP64_REL * abs(V_ref)
    assert abs(Vb - Vb_ref) <= FP64_REL * max(abs(Vb_ref), 1e-300)


def test_forces_fp64_two_cell_box(gpu, orc):
    # A box with two force-grid cells per axis: the reference counts each
    # cross-cell pair twice in its force pass; so must the GPU.
    box = (12.0, 12.0, 12.0)
    u = synth.lattice(4, 3.0, 0.02, 60.0, 0.01, seed=2)
    cfg = W.C1.config()
    cfg.size = box
    h = _handle(cfg)
    h.set_universe(u)
    V, Vb, npairs = h.forces()
    acc_ref, V_ref, _, np_ref = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass)
    _, _, acc = h.get_state()
    assert npairs == np_ref
    assert _relnorm(acc, acc_ref) <= FP64_REL
    assert abs(V - V_ref) <= FP64_REL * abs(V_ref)


@pytest.mark.parametrize("nticks", [1, 25])
def test_ticks_fp64(gpu, orc, nticks):
    wl, cfg, u = _c1(n_side=12)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 30.0
    cfg.enable_electrostatics = True
    h = _handle(cfg)
    h.set_universe(u)
    st = h.step(nticks)
    pos, vel, acc = h.get_state()
    p_ref, v_ref, a_ref, st_ref = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, nticks)
    tol = FP64_REL if nticks == 1 else 1e-9  # trajectories separate slowly from ulp-level sums
    assert _relnorm(pos, p_ref) <= tol
    assert _relnorm(vel, v_ref) <= tol
    assert _relnorm(acc, a_ref) <= tol
    assert np.all(st["pairs"] == st_ref[:, 4].astype(np.uint64))
    assert np.allclose(st["potential"], st_ref[:, 1], rtol=tol, atol=0)
    assert np.allclose(st["kinetic"], st_ref[:, 0], rtol=tol, atol=0)
    assert np.allclose(st["lambda"], st_ref[:, 3], rtol=tol, atol=0)


@pytest.mark.parametrize("nticks", [1, 25])
def test_fp64_list_path_matches_oracle(gpu, orc, nticks):
    # the plain FP64 path's default tick runs on the persistent full list
    # (k_nl_force64): the reference's per-pair arithmetic, sums in list order
    wl, cfg, u = _c1(n_side=14)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 30.0
    cfg.enable_electrostatics = True
    h = _handle(cfg)
    h.set_universe(u)
    st = h.step(nticks, graph=True)
    assert h.list_rebuilds() >= 1
    pos, vel, acc = h.get_state()
    p_ref, v_ref, a_ref, st_ref = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, nticks)
    tol = FP64_REL if nticks == 1 else 1e-9
    assert _relnorm(pos, p_ref) <= tol
    assert _relnorm(vel, v_ref) <= tol
    assert _relnorm(acc, a_ref) <= tol
    assert np.all(st["pairs"] == st_ref[:, 4].astype(np.uint64))
    assert np.allclose(st["potential"], st_ref[:, 1], rtol=tol, atol=0)
    assert np.allclose(st["lambda"], st_ref[:, 3], rtol=tol, atol=0)


def test_fp64_list_overflow_scans_cells(gpu, orc):
    # a dense clump overflows the per-atom lists; those atoms scan their cells
    wl, cfg, u = _c1(n_side=12)
    rng = np.random.default_rng(4)
    pos = u.pos.copy()
    k = 300
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos[:k] = d * (4.0 * rng.random(k) ** (1.0 / 3.0) + 0.3)[:, None]
    u2 = synth.Universe(box=u.box, pos=pos, vel=u.vel, elem=u.elem, charge=u.charge, mass=u.mass, entity=u.entity)
    h = _handle(cfg)
    h.set_universe(u2)
    st = h.step(1)
    assert h.list_stats()[1] > 0  # some lists overflowed
    _, _, acc = h.get_state()
    _, _, a_ref, st_ref = orc.ticks(cfg, u2.pos, u2.vel, None, u2.elem, u2.charge, u2.mass, 1)
    assert _relnorm(acc, a_ref) <= FP64_REL
    assert int(st["pairs"][0]) == int(st_ref[0, 4])


def test_step_matches_granular_calls(gpu):
    # the per-tick re-sort path (variant 1) runs the same force pass as gx_forces
    wl, cfg, u = _c1(n_side=10)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 30.0
    a = _handle(cfg)
    a.set_kernel_variant(1)
    a.set_universe(u)
    a.step(3)
    b = _handle(cfg)
    b.set_universe(u)
    for _ in range(3):
        b.half_kick()
        b.drift()
        b.wrap()
        b.forces()
        b.half_kick()
        b.thermostat()
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


# ---------------------------------------------------------------- mixed path


@pytest.mark.parametrize("ionic", [False, True])
def test_mixed_force_accuracy(gpu, orc, ionic):
    wl, cfg, u = _small_ionic(14) if ionic else _c1(n_side=20)
    h = _handle(cfg, "mixed")
    h.set_universe(u)
    V, Vb, npairs = h.forces()
    acc_ref, V_ref, _, np_ref = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass)
    _, _, acc = h.get_state()
    rms = _relnorm(acc, acc_ref)
    assert rms <= MIXED_RMS, rms
    assert abs(V - V_ref) <= 1e-5 * abs(V_ref)
    assert abs(int(npairs) - np_ref) <= max(2, np_ref // 100000)


@pytest.mark.parametrize("ionic", [False, True])
def test_mixed_kernel_variants_bit_identical(gpu, ionic):
    # thread-per-atom (reference half shell) and tiled (row half shell,
    # shared-memory staging, compaction) must give the same fixed-point sums
    wl, cfg, u = _small_ionic(16) if ionic else _c1(n_side=20)
    out = []
    for variant in (1, 2, 3, 4):
        h = _handle(cfg, "mixed")
        h.set_kernel_variant(variant)
        h.set_universe(u)
        V, _, npairs = h.forces()
        st = h.step(4)
        out.append((V, npairs, h.get_state(), st))
    for o in out[1:]:
        assert out[0][0] == o[0] and out[0][1] == o[1]
        for x, y in zip(out[0][2], o[2]):
            assert np.array_equal(x, y)
        assert np.array_equal(out[0][3], o[3])


@pytest.mark.parametrize("prec,variant", [("fp64", 0), ("mixed", 1), ("mixed", 5), ("mixed", 6)])
def test_graph_replay_matches_eager_ticks(gpu, prec, variant):
    wl, cfg, u = _c1(n_side=12)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 30.0
    cfg.enable_electrostatics = True
    res = []
    for graph in (False, True):
        h = _handle(cfg, prec)
        h.set_kernel_variant(variant)
        h.set_universe(u)
        parts = [h.step(3, graph=graph), h.step(6, graph=graph)]
        h.step(1, stats=False, graph=graph)
        parts.append(h.step(4, graph=graph))
        st = np.concatenate(parts)
        res.append((h.get_state(), st))
    for x, y in zip(res[0][0], res[1][0]):
        assert np.array_equal(x, y)
    assert np.array_equal(res[0][1], res[1][1])


def test_autotune_leaves_state_unchanged(gpu):
    wl, cfg, u = _c1(n_side=14)
    a = _handle(cfg, "mixed")
    a.set_universe(u)
    a.step(2)
    before = a.get_state()
    best, ms = a.autotune(reps=2)
    assert best in ms and best in (1, 2, 3, 4, 5, 6, 7, 8)
    assert all(v in ms for v in (0, 5, 6, 7, 8))  # the list paths were timed against the best pass tick
    if best >= 5:  # the skin was chosen among 0.05, 0.1, 0.15, 0.2 r_c
        skin, _ = a.list_config()
        rc = E.LJ_CUTOFF_FACTOR * max(cfg.sigma)
        assert min(abs(skin - f * rc) for f in (0.05, 0.1, 0.15, 0.2)) <= 1e-12 * rc
    after = a.get_state()
    for x, y in zip(before, after):
        assert np.array_equal(x, y)


def test_mixed_is_deterministic(gpu):
    wl, cfg, u = _c1(n_side=14)
    cfg.enable_electrostatics = True
    runs = []
    for _ in range(2):
        h = _handle(cfg, "mixed")
        h.set_universe(u)
        st = h.step(5)
        runs.append((h.get_state(), st))
    for x, y in zip(runs[0][0], runs[1][0]):
        assert np.array_equal(x, y)
    assert np.array_equal(runs[0][1], runs[1][1])


# ---------------------------------------------------------------- lenses


@pytest.mark.parametrize("n_side,r_max,nbins", [(16, 17.25, 256), (22, 17.25, 256), (12, 100.0, 512)])
def test_gr_counts_bit_exact(gpu, orc, n_side, r_max, nbins):
    wl, cfg, u = _c1(n_side=n_side)
    h = _handle(cfg)
    h.set_universe(u)
    counts, bins, rmo, dro = h.radial_distribution(r_max, nbins, E.G_SAMPLE_CAP)
    # oracle applies the same subsample internally
    c_ref, b_ref, rm_ref, dr_ref, rc = orc.radial_distribution(u.pos, cfg.size, r_max, nbins)
    assert rc == 0
    assert rmo == rm_ref and dro == dr_ref
    assert np.array_equal(counts, c_ref)
    assert np.array_equal(bins, b_ref)


def test_partial_gr_counts_bit_exact(gpu, orc):
    wl, cfg, u = _c1(n_side=16)
    h = _handle(cfg)
    h.set_universe(u)
    for ta, tb in [(2, 2), (0, 6), (9, 4)]:
        counts, bins, _, _ = h.radial_distribution(10.0, 200, E.G_SAMPLE_CAP, between=(ta, tb))
        c_ref, b_ref, _, _, _ = orc.radial_distribution(u.pos, cfg.size, 10.0, 200, elem=u.elem, between=(ta, tb))
        assert np.array_equal(counts, c_ref)
        assert np.array_equal(bins, b_ref)


def test_fof_labels_bit_exact(gpu, orc):
    wl, cfg, u = _c1(n_side=14)
    h = _handle(cfg)
    h.set_universe(u)
    h.step(20, stats=False)
    pos, _, _ = h.get_state()
    labels, st = h.clusters(E.BOND_FACTOR)
    l_ref, st_ref = orc.clusters(pos, u.elem, cfg.size, E.BOND_FACTOR, cfg.sigma)
    assert np.array_equal(labels, l_ref)
    assert st == st_ref


def test_bound_pairs_bit_exact(gpu, orc):
    wl, cfg, u = _small_ionic(12)
    ent = (np.arange(u.n, dtype=np.uint32) * 7 + 3).astype(np.uint32)
    u.entity = ent
    h = _handle(cfg)
    h.set_universe(u)
    got = h.bound_pairs(cfg.bond_k_bind)
    ref = orc.bound_pairs(u.pos, u.elem, ent, cfg.size, cfg.bond_k_bind, cfg.sigma)
    assert np.array_equal(_pairset(got), _pairset(ref))


def test_nonfinite_position_is_reported(gpu):
    from genesis_b200._lib import GxError
    wl, cfg, u = _c1(n_side=8)
    u.pos[5, 1] = np.nan
    for prec in ("fp64", "mixed"):
        h = _handle(cfg, prec)
        h.set_universe(u)
        with pytest.raises(GxError) as e:
            h.forces()
        assert e.value.status == -6


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("mixed", 1), ("mixed", 6)])
def test_gravity_matches_fp64_oracle(gpu, orc, precision, variant):
    # gravity in the FP32 pair law (-G m_i m_j / r^2 with its own switch);
    # with per-atom masses off the element table the kinds carry the mass
    import dataclasses
    wl = W.Workload("gravity check", n_side=12, temperature=60.0, steps=10, seed=3, electrostatics=True)
    cfg, u = wl.config(), wl.generate()
    cfg.enable_gravity = True
    cfg.gravity_constant = 5.0
    if precision == "mixed":  # 10 elements x 2 masses: more kinds than the FP32 table holds
        rng = np.random.default_rng(1)
        u2 = dataclasses.replace(u, mass=u.mass * np.where(rng.random(u.n) < 0.5, 1.0, 1.5))
        with pytest.raises(Exception, match="kinds"):
            _handle(cfg, "mixed").set_universe(u2)
    u = dataclasses.replace(u, mass=u.mass * 1.3)  # masses off the element table, one per element
    h = _handle(cfg, precision)
    if variant:
        h.set_kernel_variant(variant)
    h.set_universe(u)
    st = h.step(1)
    _, _, acc = h.get_state()
    _, _, acc_ref, st_ref = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, 1)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.linalg.norm(acc - acc_ref) / np.linalg.norm(acc_ref) <= tol
    assert abs(st["potential"][0] - st_ref[0, 1]) <= tol * abs(st_ref[0, 1])
    # the gravity term is really in play
    cfg0 = dataclasses.replace(cfg, enable_gravity=False)
    _, _, acc0, _ = orc.ticks(cfg0, u.pos, u.vel, None, u.elem, u.charge, u.mass, 1)
    assert np.linalg.norm(acc0 - acc_ref) / np.linalg.norm(acc_ref) > 1e-3
    if variant == 6:
        assert h.list_rebuilds() >= 1  # the neighbour-list path ran


def test_async_steps_report_errors_at_the_next_wait(gpu):
    from genesis_b200._lib import GxError
    wl, cfg, u = _c1(n_side=8)
    u.pos[5, 1] = np.nan
    for prec in ("fp64", "mixed"):
        h = _handle(cfg, prec)
        h.set_universe(u)
        h.set_step_async(True)
        h.step(1, stats=False)  # queued: returns without waiting
        with pytest.raises(GxError) as e:
            h.synchronize()
        assert e.value.status == -6
        h.synchronize()  # reported once


def test_async_steps_give_the_same_ticks(gpu):
    wl, cfg, u = _c1(n_side=10)
    out = []
    for asyn in (False, True):
        h = _handle(cfg, "mixed")
        h.set_universe(u)
        h.set_step_async(asyn)
        for _ in range(15):
            h.step(2, stats=False, graph=True)
        h.synchronize()
        out.append(h.get_state())
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_async_step_error_is_not_lost_to_a_lens_call(gpu):
    """A queued tick that saturates the fixed-point sums, then g(r): the lens
    clears the device error word for its own use, so it must report the
    queued tick's error first; a clean queued tick afterwards reports none."""
    from genesis_b200._lib import GxError
    import dataclasses
    wl, cfg, u = _small_ionic(n_side=8)
    cfg = dataclasses.replace(cfg, coulomb_constant=1e12, enable_bond_observation=False,
                              enable_bond_interaction=False, enable_thermostat=False)
    hot = synth.Universe(box=u.box, pos=u.pos.copy(), vel=u.vel, elem=u.elem, charge=u.charge.copy(),
                         mass=u.mass, entity=u.entity)
    hot.charge[:] = 0.0
    hot.charge[:2] = 1.0
    hot.pos[1] = hot.pos[0] + np.array([0.3, 0.0, 0.0])  # k_e q^2 / 0.5^2 = 4e12 >> 2^31
    clean = synth.Universe(box=u.box, pos=u.pos, vel=u.vel, elem=u.elem, charge=np.zeros_like(u.charge),
                           mass=u.mass, entity=u.entity)
    h = _handle(cfg, "mixed")
    h.set_universe(hot)
    h.set_step_async(True)
    h.step(1, stats=False)  # queued
    with pytest.raises(GxError) as e:
        h.radial_distribution(10.0, 64)
    assert e.value.status == -5
    h.set_universe(clean)
    h.step(1, stats=False)
    h.synchronize()  # the earlier error was reported once, this tick has none
    h.close()
