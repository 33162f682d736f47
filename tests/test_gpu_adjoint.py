"""The adjoint (gx_adjoint_forward / gx_adjoint_backward) on the GPU.

* The forward's V_t and g_k match the oracle's FP64 tick and the plain FP64
  gx_step path (summation order differs: <= 1e-10 relative).
* The gradients match the dual-number oracle (exact derivatives of the same
  discrete map) to 1e-7 relative, and central finite differences of the
  FP64 forward at the full C5 size (8,000 atoms, 200 ticks, checkpoint
  every 20) to 1e-4 relative, step 1e-5 x parameter.
* Checkpoint spacing does not change the result (the recomputation is
  deterministic), and the gradient with respect to the initial state
  matches finite differences.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import pytest

from genesis_b200 import adjoint as A
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

GR = dict(gr_bins=40, gr_every=2, gr_rmax=4.8, gr_width=0.115, gr_support=6.0)


def _small(n_side=8, coul=False, grav=False, seed=3):
    wl = W.Workload("adjoint check", n_side=n_side, temperature=60.0, steps=10, seed=seed, electrostatics=coul)
    cfg = wl.config()
    if grav:
        cfg.enable_gravity = True
        cfg.gravity_constant = 0.05
        cfg.gravity_cutoff = 2.5
    return cfg, wl.generate()


def _handle(cfg, u):
    from genesis_b200._lib import Handle
    h = Handle(cfg, "fp64")
    h.set_universe(u)
    return h


def _close(a, b, rel, floor):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all(np.abs(a - b) <= rel * np.abs(b) + floor * np.abs(b).max()))


def test_forward_matches_oracle(gpu, orc):
    cfg, u = _small(coul=True)
    T = 30
    with _handle(cfg, u) as h:
        V, g = h.adjoint_forward(T, checkpoint_every=7, **GR)
    Vo, go, _, _ = orc.adjoint_forward(cfg, u.pos, u.vel, np.zeros_like(u.pos), u.elem, u.charge, u.mass, T,
                                       nthreads=4, **GR)
    assert np.max(np.abs(V - Vo) / np.abs(Vo)) <= 1e-10
    assert np.max(np.abs(g - go)) <= 1e-9 * np.max(np.abs(go))


def test_forward_leaves_handle_state_unchanged(gpu):
    cfg, u = _small()
    with _handle(cfg, u) as h:
        before = h.get_state()
        h.adjoint_forward(5, checkpoint_every=2)
        after = h.get_state()
    for x, y in zip(before, after):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("coul,grav", [(False, False), (True, False), (True, True)])
def test_gradients_match_dual_oracle(gpu, orc, coul, grav):
    cfg, u = _small(coul=coul, grav=grav)
    T = 40
    w = np.random.default_rng(2).normal(size=GR["gr_bins"])
    with _handle(cfg, u) as h:
        V, g = h.adjoint_forward(T, checkpoint_every=7, **GR)
        gsV, geV = h.adjoint_backward(dl_dpotential=np.full(T, 1.0 / T))
        gsG, geG = h.adjoint_backward(dl_dgr=w)
    _, _, dV, dg = orc.adjoint_forward(cfg, u.pos, u.vel, np.zeros_like(u.pos), u.elem, u.charge, u.mass, T,
                                       nthreads=os.cpu_count() or 4, dual=True, **GR)
    refV, refG = dV.mean(0), w @ dg
    assert _close(np.r_[gsV, geV], refV, 1e-7, 1e-9)
    assert _close(np.r_[gsG, geG], refG, 1e-6, 1e-8)


def test_checkpoint_spacing_does_not_change_gradients(gpu):
    cfg, u = _small()
    T = 24
    res = []
    for K in (1, 5, 24, 100):
        with _handle(cfg, u) as h:
            h.adjoint_forward(T, checkpoint_every=K, **GR)
            gs, ge, st = h.adjoint_backward(np.full(T, 1.0 / T), np.ones(GR["gr_bins"]), initial_state=True)
        res.append((gs, ge) + st)
    for r in res[1:]:
        for x, y in zip(res[0], r):
            assert np.array_equal(x, y)


def test_initial_state_gradient_matches_finite_differences(gpu):
    cfg, u = _small(coul=True)
    T = 15
    with _handle(cfg, u) as h:
        h.adjoint_forward(T, checkpoint_every=4)
        _, _, (gx, gv, ga) = h.adjoint_backward(np.full(T, 1.0 / T), initial_state=True)
    rng = np.random.default_rng(5)
    for field, grad in (("pos", gx), ("vel", gv)):
        for _ in range(3):
            i, k = int(rng.integers(u.n)), int(rng.integers(3))
            step = 1e-6 if field == "pos" else 1e-5
            vals = []
            for s in (+1, -1):
                arr = getattr(u, field).copy()
                arr[i, k] += s * step
                u2 = dataclasses.replace(u, **{field: arr})
                with _handle(cfg, u2) as h:
                    V, _ = h.adjoint_forward(T, checkpoint_every=4)
                vals.append(V.mean())
            fd = (vals[0] - vals[1]) / (2 * step)
            assert abs(grad[i, k] - fd) <= 1e-5 * abs(fd) + 1e-7 * np.abs(grad).max()


def test_backward_is_deterministic(gpu):
    cfg, u = _small(coul=True)
    T = 12
    out = []
    for _ in range(2):
        with _handle(cfg, u) as h:
            h.adjoint_forward(T, checkpoint_every=5, **GR)
            out.append(h.adjoint_backward(np.linspace(0, 1, T), np.ones(GR["gr_bins"])))
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)


def test_rejects_unsupported_and_bad_arguments(gpu):
    from genesis_b200._lib import GxError
    cfg, u = _small()
    cfg.enable_thermostat = True
    with _handle(cfg, u) as h:
        with pytest.raises(GxError) as e:
            h.adjoint_forward(4)
        assert e.value.status == -8
    cfg, u = _small()
    with _handle(cfg, u) as h:
        with pytest.raises(GxError) as e:
            h.adjoint_backward(np.ones(4))
        assert e.value.status == -9
        with pytest.raises(GxError) as e:
            h.adjoint_forward(4, gr_bins=10, gr_rmax=5.5, gr_width=0.115, gr_support=6.0)
        assert e.value.status == -1


# ---- the full C5 workload -------------------------------------------------

@pytest.fixture(scope="module")
def c5_case(gpu):
    wl, cfg, u = A.c5()
    spec = A.AdjointSpec()
    target = A.gr_target(cfg, u, spec)
    return cfg, u, spec, target


def test_c5_forward_matches_plain_fp64_steps(c5_case):
    from genesis_b200._lib import Handle
    cfg, u, spec, _ = c5_case
    V, _ = A.forward(cfg, u, spec)
    with Handle(cfg, "fp64") as h:
        h.set_universe(u)
        st = h.step(spec.nsteps)
    assert np.max(np.abs(V - st["potential"]) / np.abs(st["potential"])) <= 1e-10


@pytest.fixture(scope="module")
def c5_fd(c5_case):
    cfg, u, spec, target = c5_case
    return A.fd_gradients(cfg, u, spec, target, rel_step=1e-5)


def test_c5_gradients_match_finite_differences(c5_case, c5_fd):
    cfg, u, spec, target = c5_case
    ad = A.gradients(cfg, u, spec, target)
    for key in ("potential", "gr"):
        g = np.r_[ad[key][1], ad[key][2]]
        assert _close(g, c5_fd[key], 1e-4, 1e-6), (key, g, c5_fd[key])


def test_c5_mixed_forward_gradients_match_finite_differences(c5_case, c5_fd):
    """The C5 form: the forward in the mixed method (FP32 pair law,
    fixed-point force sums), the adjoint in FP64 on that trajectory, against
    central differences of the plain FP64 forward, 1e-4 relative."""
    cfg, u, spec, target = c5_case
    ad = A.gradients(cfg, u, spec, target, precision="mixed")
    for key in ("potential", "gr"):
        g = np.r_[ad[key][1], ad[key][2]]
        assert _close(g, c5_fd[key], 1e-4, 1e-6), (key, g, c5_fd[key])


def test_c5_mixed_forward_follows_mixed_steps(c5_case):
    """V_t of the mixed forward against the FP64 forward (the trajectories
    part only by the FP32 pair law's rounding) and against mixed gx_step
    records (whose pair law runs on cell-frame FP32 displacements)."""
    from genesis_b200._lib import Handle
    cfg, u, spec, _ = c5_case
    Vm, gm = A.forward(cfg, u, spec, precision="mixed")
    V64, g64 = A.forward(cfg, u, spec)
    with Handle(cfg, "mixed") as h:
        h.set_universe(u)
        st = h.step(spec.nsteps)
    assert np.max(np.abs(Vm - V64) / np.abs(V64)) <= 1e-5
    assert np.max(np.abs(Vm - st["potential"]) / np.abs(st["potential"])) <= 1e-5
    assert np.max(np.abs(gm - g64)) <= 1e-4 * np.max(np.abs(g64))


def test_mixed_forward_is_deterministic_and_checkpoint_invariant(gpu):
    cfg, u = _small(coul=True)
    T = 24
    out = []
    for K in (1, 5, 24):
        from genesis_b200._lib import Handle
        with Handle(cfg, "mixed") as h:
            h.set_universe(u)
            V, g = h.adjoint_forward(T, checkpoint_every=K, **GR)
            gs, ge = h.adjoint_backward(dl_dpotential=np.full(T, 1.0 / T))
        out.append((V, g, gs, ge))
    for o in out[1:]:
        for x, y in zip(out[0], o):
            assert np.array_equal(x, y)


def test_c5_gradients_match_dual_oracle(c5_case, orc):
    cfg, u, spec, target = c5_case
    ad = A.gradients(cfg, u, spec, target)
    V, g, dV, dg = orc.adjoint_forward(cfg, u.pos, u.vel, np.zeros_like(u.pos), u.elem, u.charge, u.mass,
                                       spec.nsteps, gr_bins=spec.gr_bins, gr_every=spec.gr_every,
                                       gr_rmax=spec.gr_rmax, gr_width=spec.gr_width, gr_support=spec.gr_support,
                                       nthreads=os.cpu_count() or 4, dual=True)
    assert _close(np.r_[ad["potential"][1], ad["potential"][2]], dV.mean(0), 1e-7, 1e-9)
    _, cg = A.gr_loss(g, target)
    assert _close(np.r_[ad["gr"][1], ad["gr"][2]], cg @ dg, 1e-6, 1e-8)
