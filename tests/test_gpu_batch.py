"""Batched replicas (persistent launches and the all-replica graph) against
one gx_handle per replica."""
from __future__ import annotations

import numpy as np
import pytest

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _replicas(thermo: bool):
    reps = [W.Replica(n_side=n, temperature=t, seed=11 + k)
            for k, (n, t) in enumerate([(8, 40.0), (11, 90.0), (9, 25.0), (13, 110.0)])]
    wls = [W.replica_workload(r) for r in reps]
    for wl in wls:
        wl.thermostat = thermo
    return wls


def _single(wl, steps, variant=1):
    from genesis_b200._lib import Handle
    cfg = wl.config()
    h = Handle(cfg, "mixed")
    h.set_kernel_variant(variant)  # modes 1-3 re-sort every tick, like variants 1-4; mode 4 keeps lists, like 6
    u = wl.generate()
    h.set_universe(u)
    st = h.step(steps)
    out = h.get_state()
    h.close()
    return out, st


def _batch(wls, steps, mode=2):
    from genesis_b200._lib import Batch
    base = wls[0].config()
    base.enable_thermostat = wls[0].thermostat
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_mode(mode)
    b.set_universes([wl.generate() for wl in wls])
    st, ms = b.step(steps)
    out = b.get_state()
    b.close()
    return out, st, ms


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_batch_nve_matches_single_universes_bit_for_bit(gpu, mode):
    wls = _replicas(thermo=False)
    out, st, ms = _batch(wls, 6, mode)
    assert ms > 0
    for k, wl in enumerate(wls):
        ref, rst = _single(wl, 6)
        for x, y in zip(out[k], ref):
            assert np.array_equal(x, y)
        assert st[k, 3] == rst["pairs"][-1]
        assert st[k, 1] == rst["potential"][-1]


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_batch_nvt_matches_single_universes(gpu, mode):
    wls = _replicas(thermo=True)
    out, st, _ = _batch(wls, 5, mode)
    for k, wl in enumerate(wls):
        ref, rst = _single(wl, 5)
        for x, y in zip(out[k], ref):
            assert np.linalg.norm(x - y) <= 1e-12 * np.linalg.norm(y)
        assert abs(st[k, 0] - rst["kinetic"][-1]) <= 1e-12 * abs(rst["kinetic"][-1])
        assert abs(st[k, 2] - rst["lambda"][-1]) <= 1e-12


def test_persistent_mode_rejects_oversized_replica_grid(gpu):
    from genesis_b200._lib import Batch, GxError
    wl = W.Replica(n_side=8, temperature=40.0, seed=3)
    u = W.replica_workload(wl).generate()
    base = W.C1.config()
    b = Batch(base, [(500.0, 500.0, 500.0)], [50.0])  # 86^3 force cells > 4096
    b.set_universes([u])
    b.set_mode(1)
    with pytest.raises(GxError) as e:
        b.step(1)
    assert e.value.status == -4
    b.set_mode(2)  # the all-replica graph has no per-replica cell limit
    b.step(2)
    b.close()


def test_batch_modes_agree_and_autotune_restores_state(gpu):
    wls = _replicas(thermo=True)
    a, sa, _ = _batch(wls, 8, mode=1)
    c, sc, _ = _batch(wls, 8, mode=2)
    for x, y in zip(a, c):
        for p, q in zip(x, y):
            assert np.linalg.norm(p - q) <= 1e-12 * max(np.linalg.norm(q), 1e-300)
    from genesis_b200._lib import Batch
    base = wls[0].config()
    base.enable_thermostat = True
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_universes([wl.generate() for wl in wls])
    before = b.get_state()
    mode, ms = b.autotune(ticks=3)
    assert mode in (1, 2, 3, 4) and ms[1] > 0 and ms[2] > 0 and ms[3] > 0 and ms[4] > 0
    after = b.get_state()
    for x, y in zip(before, after):
        for p, q in zip(x, y):
            assert np.array_equal(p, q)
    b.close()


def test_cooperative_launch_matches_the_graph_bit_for_bit(gpu):
    # mode 3 runs mode 2's phases inside one launch: the same bits, thermostat
    # on, over step calls of several lengths (the last tick of each reports)
    wls = _replicas(thermo=True)
    runs = []
    for mode in (2, 3):
        from genesis_b200._lib import Batch
        base = wls[0].config()
        base.enable_thermostat = True
        b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
        b.set_mode(mode)
        b.set_universes([wl.generate() for wl in wls])
        sts = [b.step(k)[0] for k in (1, 7, 30)]
        runs.append((b.get_state(), sts))
        b.close()
    for x, y in zip(runs[0][0], runs[1][0]):
        for p, q in zip(x, y):
            assert np.array_equal(p, q)
    for a, c in zip(runs[0][1], runs[1][1]):
        assert np.array_equal(a, c)


# ---------------------------------------------------------------- mode 4: neighbour lists


def test_list_mode_single_replica_matches_list_handle_bit_for_bit(gpu):
    # one replica rebuilds on the handle's own schedule, in the same frames,
    # with the same per-pair operations and integer sums
    from genesis_b200._lib import Batch, Handle
    wl = W.replica_workload(W.Replica(n_side=12, temperature=150.0, seed=5))
    wl.thermostat = False
    cfg = wl.config()
    skin = 0.15 * 5.75
    b = Batch(cfg, [cfg.size], [wl.thermostat_temperature])
    b.set_mode(4)
    b.set_list_skin(skin)
    b.set_universes([wl.generate()])
    st, _ = b.step(25)
    out = b.get_state()
    b.close()
    h = Handle(cfg, "mixed")
    h.set_kernel_variant(6)
    h.set_list_skin(skin)
    h.set_universe(wl.generate())
    rst = h.step(25)
    ref = h.get_state()
    h.close()
    for x, y in zip(out[0], ref):
        assert np.array_equal(x, y)
    assert st[0, 3] == rst["pairs"][-1]
    assert st[0, 1] == rst["potential"][-1]


def test_list_mode_follows_the_graph_mode_and_rebuilds(gpu):
    from genesis_b200._lib import Batch
    wls = _replicas(thermo=True)
    runs = []
    for mode in (2, 4):
        base = wls[0].config()
        base.enable_thermostat = True
        b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
        b.set_mode(mode)
        b.set_universes([wl.generate() for wl in wls])
        sts = [b.step(k)[0] for k in (1, 9, 30)]
        runs.append((b.get_state(), sts, b.list_rebuilds() if mode == 4 else None))
        b.close()
    assert runs[1][2] >= 2  # the first tick and at least one displacement-triggered rebuild
    # the two frames differ in the last FP32 bits of each pair's displacement:
    # forces by ~3e-6 relative (the mixed path's error against FP64 is of the
    # same size), positions far less over 40 ticks
    for x, y in zip(runs[0][0], runs[1][0]):
        for p, q, tol in zip(x, y, (1e-7, 1e-5, 1e-5)):
            assert np.linalg.norm(p - q) <= tol * max(np.linalg.norm(q), 1e-300)
    for a, c in zip(runs[0][1], runs[1][1]):
        assert np.allclose(a[:, 0], c[:, 0], rtol=1e-6, atol=0)  # K
        assert np.allclose(a[:, 1], c[:, 1], rtol=1e-5, atol=0)  # V
        assert np.all(np.abs(a[:, 3] - c[:, 3]) <= 2)            # pairs


def test_list_mode_forces_match_the_oracle(gpu, orc):
    from genesis_b200._lib import Batch
    wls = _replicas(thermo=True)
    base = wls[0].config()
    base.enable_thermostat = True
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_mode(4)
    us = [wl.generate() for wl in wls]
    b.set_universes(us)
    b.step(12)
    out = b.get_state()
    b.close()
    for (pos, _, acc), wl, u in zip(out, wls, us):
        acc_ref, _, _, _ = orc.forces(wl.config(), pos, u.elem, u.charge, u.mass)
        assert np.linalg.norm(acc - acc_ref) <= 1e-5 * np.linalg.norm(acc_ref)


def test_list_mode_rebuilds_after_a_new_state_and_is_deterministic(gpu):
    from genesis_b200._lib import Batch
    wls = _replicas(thermo=True)
    base = wls[0].config()
    base.enable_thermostat = True
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_mode(4)
    first = None
    for _ in range(2):  # the same state uploaded again: the lists restart from it
        b.set_universes([wl.generate() for wl in wls])
        r0 = b.list_rebuilds()
        b.step(6)
        assert b.list_rebuilds() > r0
        got = b.get_state()
        if first is None:
            first = got
    for x, y in zip(first, got):
        for p, q in zip(x, y):
            assert np.array_equal(p, q)
    mode, ms = b.autotune(ticks=3)
    assert mode in (1, 2, 3, 4) and ms[4] > 0
    b.close()


def test_list_mode_rejects_small_replicas(gpu):
    from genesis_b200._lib import Batch, GxError
    wl = W.replica_workload(W.Replica(n_side=4, temperature=40.0, seed=3))  # 64 atoms
    base = wl.config()
    b = Batch(base, [wl.config().size], [40.0])
    b.set_universes([wl.generate()])
    b.set_mode(4)
    with pytest.raises(GxError):
        b.step(1)
    b.close()


def test_list_mode_overflowing_lists_scan_their_cells(gpu, orc):
    # a dense clump in one replica overflows the per-slot lists (sized for the
    # densest replica on average); those slots scan their cells directly
    import dataclasses
    from genesis_b200._lib import Batch
    wls = _replicas(thermo=False)
    us = [wl.generate() for wl in wls]
    rng = np.random.default_rng(4)
    pos = us[3].pos.copy()
    k = 300
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos[:k] = d * (4.0 * rng.random(k) ** (1.0 / 3.0) + 0.3)[:, None]
    us[3] = dataclasses.replace(us[3], pos=pos, vel=us[3].vel * 0.0)
    base = wls[0].config()
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls])
    b.set_mode(4)
    b.set_universes(us)
    b.step(1)
    entries, overflowed = b.list_stats()
    assert entries > 0 and overflowed > 0
    out = b.get_state()
    b.close()
    for (p_, _, acc), wl, u in zip(out, wls, us):
        acc_ref, _, _, _ = orc.forces(wl.config(), p_, u.elem, u.charge, u.mass)
        assert np.linalg.norm(acc - acc_ref) <= 1e-5 * np.linalg.norm(acc_ref)
