"""Oracle parity at the benchmarked sizes, through the C ABI.

The other parity tests run on 8^3-22^3 states.  These run the two measured
workloads at their full size against the same CPU oracle:

* the condensation quench, 128^3 = 2,097,152 atoms (61^3 force grid, about
  nine atoms per cell, Coulomb on): cell assignment, one FP64 force pass
  (<= 1e-12), the mixed neighbour-list tick after 20 ticks that include list
  rebuilds (force relative RMS <= 1e-5), and the g(r) bins, FoF labels and
  bound pairs, which are integers and must match exactly;
* the ionic Na/O system, 32^3 = 32,768 atoms, with bond observation every
  tick for 40 ticks (persistence after 0.1 vibration periods, so bonds form
  and the spring runs), tick by tick against the oracle's tracker in both
  precisions, then the forces with the observed bonds;
* the 256-replica temperature sweep (1.13M atoms) in batch mode 4, every
  replica's forces after 30 ticks of persistent neighbour lists.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import synth
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
MIXED_RMS = 1e-5
THREADS = os.cpu_count() or 1


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _pairset(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return np.sort(np.minimum(p[:, 0], p[:, 1]) * (1 << 32) + np.maximum(p[:, 0], p[:, 1]))


@pytest.fixture(scope="module")
def quench():
    wl = W.C3
    assert wl.n_atoms == 2_097_152
    return wl.config(), wl.generate()


# ---------------------------------------------------------------- 2,097,152 atoms


def test_quench_cell_assignment_on_the_force_grid(gpu, orc, quench):
    from genesis_b200._lib import Handle
    cfg, u = quench
    rc = E.LJ_CUTOFF_FACTOR * max(cfg.sigma)
    with Handle(cfg, "fp64") as h:
        h.set_universe(u)
        got = h.cell_assign(rc)
    ref = orc.cell_of(u.pos, cfg.size, rc)
    assert orc.grid_dims(cfg.size, rc) == (61, 61, 61)
    assert np.array_equal(got, ref)


def test_quench_fp64_forces(gpu, orc, quench):
    from genesis_b200._lib import Handle
    cfg, u = quench
    with Handle(cfg, "fp64") as h:
        h.set_universe(u)
        V, Vb, npairs = h.forces()
        _, _, acc = h.get_state()
    acc_ref, V_ref, _, np_ref = orc.forces(cfg, u.pos, u.elem, u.charge, u.mass, nthreads=THREADS)
    assert npairs == np_ref
    assert _rel(acc, acc_ref) <= FP64_REL
    # per atom as well: the largest deviation against that atom's own force
    dev = np.linalg.norm(acc - acc_ref, axis=1) / np.maximum(np.linalg.norm(acc_ref, axis=1), 1e-300)
    assert float(np.quantile(dev, 0.999)) <= 1e-9
    assert abs(V - V_ref) <= FP64_REL * abs(V_ref)


def test_quench_mixed_list_ticks_then_lenses(gpu, orc, quench):
    """20 mixed ticks on the half neighbour list (Berendsen towards 20 K from
    300 K): the acceleration the last tick left is the force at the final
    positions, compared with the oracle's force pass there; then the FP64
    pass at the same positions, and the lenses on that state."""
    from genesis_b200._lib import Handle
    cfg, u = quench
    with Handle(cfg, "mixed") as h:
        h.set_kernel_variant(6)
        h.set_universe(u)
        st = h.step(20, graph=True)
        rebuilds = h.list_rebuilds()
        pos, vel, acc = h.get_state()
    assert rebuilds >= 2  # the build on the first tick and at least one displacement-triggered rebuild
    acc_ref, V_ref, _, np_ref = orc.forces(cfg, pos, u.elem, u.charge, u.mass, nthreads=THREADS)
    rms = _rel(acc, acc_ref)
    assert rms <= MIXED_RMS, rms
    assert abs(float(st["potential"][-1]) - V_ref) <= 1e-5 * abs(V_ref)
    assert abs(int(st["pairs"][-1]) - np_ref) <= max(2, np_ref // 100000)

    with Handle(cfg, "fp64") as h:
        h.set_universe(synth.Universe(box=u.box, pos=pos, vel=vel, elem=u.elem, charge=u.charge, mass=u.mass,
                                      entity=u.entity))
        V, _, npairs = h.forces()
        _, _, acc64 = h.get_state()
        assert npairs == np_ref
        assert _rel(acc64, acc_ref) <= FP64_REL
        assert abs(V - V_ref) <= FP64_REL * abs(V_ref)

        # g(r) of the reference's call: 256 bins to 3 r_c, the 8,192-atom subsample
        counts, bins, rmo, dro = h.radial_distribution(17.25, 256, E.G_SAMPLE_CAP)
        c_ref, b_ref, rm_ref, dr_ref, rc = orc.radial_distribution(pos, cfg.size, 17.25, 256)
        assert rc == 0 and counts.sum() > 0
        assert rmo == rm_ref and dro == dr_ref
        assert np.array_equal(counts, c_ref)
        assert np.array_equal(bins, b_ref)

        labels, fst = h.clusters(E.BOND_FACTOR)
        l_ref, fst_ref = orc.clusters(pos, u.elem, cfg.size, E.BOND_FACTOR, cfg.sigma)
        assert np.array_equal(labels, l_ref)
        assert fst == fst_ref

        got = h.bound_pairs(cfg.bond_k_bind)
        ref = orc.bound_pairs(pos, u.elem, u.entity, cfg.size, cfg.bond_k_bind, cfg.sigma)
        assert len(ref) > 3_000_000
        assert np.array_equal(_pairset(got), _pairset(ref))


# ---------------------------------------------------------------- 32,768 Na/O atoms


KEYS = ("bonded_pairs", "bonded_entities", "mean_coordination", "bonds_formed", "lifetime_sum_ticks",
        "open_episodes", "completed_episodes", "completed_ticks")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ionic_observation_tick_by_tick(gpu, orc, precision):
    from genesis_b200._lib import Handle
    wl = W.C2
    assert wl.n_atoms == 32_768
    cfg, u = wl.config(), wl.generate()
    min_periods = 0.1  # the reference's floor: Na/O pairs persist after ~32 ticks
    h = Handle(cfg, precision)
    h.set_universe(u)
    ref = orc.BondTracker(cfg, debounce=E.DEBOUNCE, min_periods=min_periods)
    bonds = np.zeros((0, 2), dtype=np.uint32)
    for tick in range(1, 41):
        h.step(1)
        pos, _, acc = h.get_state()
        if tick in (1, 20, 40):
            # the tick's force pass against the oracle with the bonds it used
            acc_ref, _, _, _ = orc.forces(cfg, pos, u.elem, u.charge, u.mass, bonds=bonds if len(bonds) else None,
                                          nthreads=THREADS)
            assert _rel(acc, acc_ref) <= (FP64_REL if precision == "fp64" else MIXED_RMS)
        bound = h.bound_pairs(cfg.bond_k_bind)  # entity = slot here
        if tick in (1, 40):
            want_bound = orc.bound_pairs(pos, u.elem, u.entity, cfg.size, cfg.bond_k_bind, cfg.sigma)
            assert np.array_equal(_pairset(bound), _pairset(want_bound))
        got = h.bond_observe(cfg.bond_k_bind, min_periods, tick)
        want, pers = ref.observe(bound, u.elem, tick)
        for k in KEYS:
            assert got[k] == want[k], (tick, k, got[k], want[k])
        assert np.array_equal(got["species_matrix"], want["species_matrix"])
        bonds = h.get_bonds()
        assert np.array_equal(np.sort(bonds.view(np.uint64).ravel()), np.sort(pers.view(np.uint64).ravel()))
    assert got["bonded_pairs"] > 100  # bonds formed, and the last ticks ran the spring on them
    # the spring with the observed bonds, against the oracle at the final state
    pos, _, _ = h.get_state()
    V, Vb, _ = h.forces()
    _, _, acc = h.get_state()
    acc_ref, V_ref, Vb_ref, _ = orc.forces(cfg, pos, u.elem, u.charge, u.mass, bonds=bonds, nthreads=THREADS)
    tol = FP64_REL if precision == "fp64" else MIXED_RMS
    assert _rel(acc, acc_ref) <= tol
    assert Vb_ref != 0.0 and abs(Vb - Vb_ref) <= tol * abs(Vb_ref)
    h.close()


# ---------------------------------------------------------------- 256 sweep replicas


def test_sweep_replicas_on_neighbour_lists_match_the_oracle(gpu, orc):
    """The benchmarked sweep (256 replicas, 1.13M atoms) in batch mode 4:
    after 30 ticks (the first rebuilds every list, later ones as atoms move)
    every replica's accelerations against the oracle's forces at its own
    positions."""
    from genesis_b200 import sweep
    from genesis_b200._lib import Batch
    wls = sweep.make_replicas(256, seed=0)
    assert sweep.atoms(wls) > 1_000_000
    base = wls[0].config()
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_mode(4)
    us = [wl.generate() for wl in wls]
    b.set_universes(us)
    b.step(30)
    assert b.list_rebuilds() >= 2
    out = b.get_state()
    b.close()
    worst = 0.0
    for (pos, _, acc), wl, u in zip(out, wls, us):
        acc_ref, _, _, _ = orc.forces(wl.config(), pos, u.elem, u.charge, u.mass, nthreads=THREADS)
        worst = max(worst, _rel(acc, acc_ref))
    assert worst <= MIXED_RMS, worst
