"""The persistent neighbour-list passes (kernel variants 5: full list, 6:
half list with far-end atomics, 7: the half list with in-cutoff entries
collected in shared memory before the pair law, 8: the half list brick by
brick with the brick's neighbourhood staged in shared memory) against the
oracle, each other and the per-tick re-sort variants.

Variants 5-8 evaluate the same pair set {d < r_c} as every other variant, in a
cell-local frame anchored at the last rebuild, so its FP32 forces can differ
from variants 1-4 in the last bits: the checks are the mixed path's error
bound against the FP64 oracle (force rel-RMS <= 1e-5), agreement of whole
trajectories with variant 1, exact pair counts, determinism, and the
overflow fallback (atoms whose list overflows scan their cells directly).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

MIXED_RMS = 1e-5


def _handle(cfg, variant=5):
    from genesis_b200._lib import Handle
    h = Handle(cfg, "mixed")
    h.set_kernel_variant(variant)
    return h


def _lattice(n_side=16, temperature=60.0, coul=False, seed=0):
    wl = W.Workload("nl check", n_side=n_side, temperature=temperature, steps=10, seed=seed,
                    electrostatics=coul)
    return wl.config(), wl.generate()


def _relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("coul,variant", [(False, 5), (True, 5), (False, 6), (True, 6), (True, 7), (True, 8)])
def test_first_tick_forces_match_fp64_oracle(gpu, orc, coul, variant):
    cfg, u = _lattice(18, coul=coul)
    h = _handle(cfg, variant)
    h.set_universe(u)
    st = h.step(1)
    _, _, acc = h.get_state()
    _, _, acc_ref, st_ref = orc.ticks(cfg, u.pos, u.vel, None, u.elem, u.charge, u.mass, 1)
    assert _relnorm(acc, acc_ref) <= MIXED_RMS
    assert abs(st["potential"][0] - st_ref[0, 1]) <= 1e-5 * abs(st_ref[0, 1])
    assert abs(int(st["pairs"][0]) - int(st_ref[0, 4])) <= 2


@pytest.mark.parametrize("thermo", [False, True])
def test_full_and_half_lists_are_bit_identical(gpu, thermo):
    cfg, u = _lattice(14, temperature=150.0, coul=True)
    if thermo:
        cfg.enable_thermostat = True
        cfg.thermostat_temperature = 40.0
    out = []
    for variant, opt in ((5, 0), (6, 0), (7, 16), (7, 8), (8, 4), (8, 8)):
        h = _handle(cfg, variant)
        if variant == 7:
            h.set_list_stash(opt)
        if variant == 8:
            h.set_list_brick(opt)
        h.set_universe(u)
        st = h.step(25, graph=True)
        out.append((h.get_state(), st, h.list_rebuilds()))
    for o in out[1:]:
        for x, y in zip(out[0][0], o[0]):
            assert np.array_equal(x, y)
        assert np.array_equal(out[0][1], o[1])
        assert out[0][2] == o[2]


def test_brick_list_build_writes_the_same_lists(gpu):
    # variant 8 builds its half lists brick by brick from shared memory;
    # the entry counts equal variant 6's after every tick of a run with
    # rebuilds, and the trajectories are the same bits
    cfg, u = _lattice(14, temperature=200.0, coul=True)
    hs = []
    for variant in (6, 8):
        h = _handle(cfg, variant)
        h.set_universe(u)
        hs.append(h)
    for _ in range(12):
        st = [h.step(2) for h in hs]
        e6, e8 = hs[0].list_stats(), hs[1].list_stats()
        assert e6 == e8 and e6[0] > 0
        assert np.array_equal(st[0], st[1])
    assert hs[1].list_rebuilds() >= 2
    for x, y in zip(hs[0].get_state(), hs[1].get_state()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("thermo", [False, True])
def test_trajectory_follows_per_tick_variant(gpu, thermo):
    cfg, u = _lattice(16, temperature=120.0, coul=True)
    if thermo:
        cfg.enable_thermostat = True
        cfg.thermostat_temperature = 40.0
    out = []
    for variant in (1, 5):
        h = _handle(cfg, variant)
        h.set_universe(u)
        st = h.step(40)
        out.append((h.get_state(), st, h))
    (p1, v1, a1), s1, _ = out[0]
    (p5, v5, a5), s5, h5 = out[1]
    assert np.max(np.abs(p1 - p5)) <= 1e-6
    assert _relnorm(v5, v1) <= 1e-5
    assert np.max(np.abs(s5["potential"] - s1["potential"]) / np.abs(s1["potential"])) <= 1e-5
    assert np.max(np.abs(s5["pairs"].astype(np.int64) - s1["pairs"].astype(np.int64))) <= 2
    if thermo:
        assert np.max(np.abs(s5["lambda"] - s1["lambda"])) <= 1e-6
    assert h5.list_rebuilds() >= 1


@pytest.mark.parametrize("variant", [5, 6])
def test_threads_per_atom_are_bit_identical(gpu, variant):
    # lanes per atom, and for one lane the block of the shared far-end sums
    cfg, u = _lattice(14, temperature=150.0, coul=True)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 40.0
    out = []
    for tpp, block in ((1, 0), (1, 128), (1, 256), (2, 0), (4, 0), (8, 0)):
        h = _handle(cfg, variant)
        h.set_list_block(block)
        h.set_list_threads(tpp)
        h.set_universe(u)
        st = h.step(12, graph=True)
        assert h.list_config()[1] == tpp
        shape = h.list_shape()
        assert (shape["threads_per_atom"], shape["block"]) == (tpp, block)
        out.append((h.get_state(), st))
    for o in out[1:]:
        for x, y in zip(out[0][0], o[0]):
            assert np.array_equal(x, y)
        assert np.array_equal(out[0][1], o[1])


def test_zero_skin_rebuilds_every_tick(gpu):
    cfg, u = _lattice(12)
    h = _handle(cfg)
    h.set_list_skin(0.0)
    h.set_universe(u)
    h.step(7)
    assert h.list_rebuilds() == 7


def test_default_skin_reuses_the_list(gpu):
    cfg, u = _lattice(14, temperature=20.0)
    h = _handle(cfg)
    h.set_universe(u)
    h.step(30)
    assert 1 <= h.list_rebuilds() < 30


def test_list_path_is_deterministic_and_graph_invariant(gpu):
    cfg, u = _lattice(14, coul=True)
    runs = []
    for graph in (False, True, True):
        h = _handle(cfg)
        h.set_universe(u)
        st = h.step(12, graph=graph)
        runs.append((h.get_state(), st))
    for r in runs[1:]:
        for x, y in zip(runs[0][0], r[0]):
            assert np.array_equal(x, y)
        assert np.array_equal(runs[0][1], r[1])


@pytest.mark.parametrize("variant", [5, 6, 7, 8])
def test_overflowing_lists_fall_back_to_cell_scans(gpu, orc, variant):
    # a dense clump far above the average density overflows the per-atom lists
    cfg, u = _lattice(12, temperature=10.0)
    rng = np.random.default_rng(4)
    pos = u.pos.copy()
    k = 300
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = 4.0 * rng.random(k) ** (1.0 / 3.0) + 0.3
    pos[:k] = d * r[:, None]
    u2 = dataclasses.replace(u, pos=pos)
    h = _handle(cfg, variant)
    h.set_universe(u2)
    st = h.step(1)
    _, _, acc = h.get_state()
    _, _, acc_ref, st_ref = orc.ticks(cfg, u2.pos, u2.vel, None, u2.elem, u2.charge, u2.mass, 1)
    assert _relnorm(acc, acc_ref) <= MIXED_RMS
    assert abs(int(st["pairs"][0]) - int(st_ref[0, 4])) <= 2


def test_state_round_trip_after_list_ticks(gpu):
    # set_dynamic after list ticks writes through the list-grid order
    cfg, u = _lattice(12)
    h = _handle(cfg)
    h.set_universe(u)
    h.step(5)
    pos, vel, acc = h.get_state()
    h.set_dynamic(pos, vel, acc)
    p2, v2, a2 = h.get_state()
    assert np.array_equal(pos, p2) and np.array_equal(vel, v2) and np.array_equal(acc, a2)


@pytest.mark.parametrize("variant", [5, 6, 7, 8])
def test_captured_rebuilds_run_only_when_flagged(gpu, variant):
    # a captured tick holds the rebuild in a conditional graph node set from
    # the displacement flag: the same ticks and rebuilds as eager execution,
    # with the rebuild kernels launched only on the ticks that rebuild
    cfg, u = _lattice(14, temperature=300.0, coul=True)
    out = []
    for graph in (False, True):
        h = _handle(cfg, variant)  # the default skin, 0.1 r_c: a rebuild every few ticks at 300 K
        h.set_universe(u)
        l0 = h.launches
        st = h.step(40, graph=graph)
        rb = h.list_rebuilds()
        out.append((h.get_state(), st, rb, h.launches - l0))
    (s0, t0, r0, n0), (s1, t1, r1, n1) = out
    for x, y in zip(s0, s1):
        assert np.array_equal(x, y)
    assert np.array_equal(t0, t1)
    assert r0 == r1 and 3 <= r0 < 40
    assert n1 < n0  # eager launches every gated rebuild kernel on every tick


def test_zero_skin_captured_rebuild_every_tick(gpu):
    cfg, u = _lattice(12)
    h = _handle(cfg)
    h.set_list_skin(0.0)
    h.set_universe(u)
    h.step(7, graph=True)
    assert h.list_rebuilds() == 7


@pytest.mark.parametrize("variant", [5, 6])
def test_ticks_without_records_give_the_same_state(gpu, variant):
    # a tick that records nothing skips the potential and the pair count in
    # the list pass; the forces, and so the trajectory, are the same bits
    cfg, u = _lattice(14, temperature=200.0, coul=True)
    cfg.enable_thermostat = True
    cfg.thermostat_temperature = 60.0
    out = []
    for stats in (True, False):
        h = _handle(cfg, variant)
        h.set_universe(u)
        h.step(30, stats=stats, graph=True)
        out.append(h.get_state())
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)


def test_bricks_beyond_the_staging_capacity_read_global_memory(gpu):
    # a dense clump puts more than the 1024-atom staging capacity of a
    # 4-cell brick into its neighbourhood: those bricks read global memory,
    # with the same forces as variant 6
    cfg, u = _lattice(16, temperature=10.0)
    rng = np.random.default_rng(9)
    pos = u.pos.copy()
    k = 1500
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos[:k] = d * (6.0 * rng.random(k) ** (1.0 / 3.0) + 0.2)[:, None]
    u2 = dataclasses.replace(u, pos=pos)
    out = []
    for variant, brick in ((6, 0), (8, 4), (8, 8)):
        h = _handle(cfg, variant)
        if brick:
            h.set_list_brick(brick)
        h.set_universe(u2)
        st = h.step(2)
        out.append((h.get_state(), st))
    for o in out[1:]:
        for x, y in zip(out[0][0], o[0]):
            assert np.array_equal(x, y)
        assert np.array_equal(out[0][1], o[1])


def test_pass_timing_inside_captured_ticks(gpu):
    # events captured around the pair pass time the replayed tick's own pass
    cfg, u = _lattice(14, temperature=150.0, coul=True)
    h = _handle(cfg)
    h.set_universe(u)
    h.step(3, graph=True)
    h.set_pass_timing(True)
    h.step(2, graph=True)
    t_graph = h.pass_ms()
    h.step(1, graph=False)
    t_eager = h.pass_ms()
    h.set_pass_timing(False)
    assert 0.0 < t_graph < 50.0 and 0.0 < t_eager < 50.0
    st = h.step(2, graph=True)  # timing off again: the ticks re-capture without the events
    assert len(st["pairs"]) == 2
