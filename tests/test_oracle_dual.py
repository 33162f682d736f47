"""The dual-number adjoint reference (oracle/oracle_dual.cpp) on the CPU.

Its T = double instantiation must reproduce orc_ticks (the pinned FP64
restatement) bit for bit, and its dual derivatives must agree with central
finite differences of that double path.
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from genesis_b200 import workloads as W

GR = dict(gr_bins=40, gr_every=2, gr_rmax=4.8, gr_width=0.115, gr_support=6.0)


def _small(n_side=8, coul=False, grav=False, seed=3):
    wl = W.Workload("dual check", n_side=n_side, temperature=60.0, steps=10, seed=seed, electrostatics=coul)
    cfg = wl.config()
    if grav:
        cfg.enable_gravity = True
        cfg.gravity_constant = 0.05
        cfg.gravity_cutoff = 2.5
    return cfg, wl.generate()


@pytest.mark.parametrize("coul,grav,nt", [(False, False, 1), (False, False, 3), (True, False, 2), (True, True, 1)])
def test_double_instantiation_matches_orc_ticks_bitwise(orc, coul, grav, nt):
    cfg, u = _small(coul=coul, grav=grav)
    acc = np.zeros_like(u.pos)
    a = orc.ticks(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 12, nthreads=nt)
    b = orc.adjoint_trajectory(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 12, nthreads=nt)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert np.array_equal(a[3][:, 1], b[3])


def test_dual_values_equal_double_values(orc):
    cfg, u = _small()
    acc = np.zeros_like(u.pos)
    V, g, dV, dg = orc.adjoint_forward(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 8, nthreads=4, dual=True,
                                       **GR)
    V2, g2, _, _ = orc.adjoint_forward(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 8, nthreads=4, **GR)
    assert np.array_equal(V, V2) and np.array_equal(g, g2)
    assert dV.shape == (8, 20) and dg.shape == (40, 20)


def _perturbed(cfg, j, h):
    c = copy.deepcopy(cfg)
    if j < 10:
        s = list(cfg.sigma)
        s[j] += h
        c.sigma = tuple(s)
    else:
        e = list(cfg.epsilon_k)
        e[j - 10] += h
        c.epsilon_k = tuple(e)
    return c


@pytest.mark.parametrize("coul", [False, True])
def test_dual_derivatives_match_central_differences(orc, coul):
    cfg, u = _small(coul=coul)
    acc = np.zeros_like(u.pos)
    T = 10
    w = np.random.default_rng(1).normal(size=GR["gr_bins"])
    V, g, dV, dg = orc.adjoint_forward(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, T, nthreads=4, dual=True,
                                       **GR)
    ad_V, ad_g = dV.mean(0), w @ dg

    def losses(c):
        V, g, _, _ = orc.adjoint_forward(c, u.pos, u.vel, acc, u.elem, u.charge, u.mass, T, nthreads=4, **GR)
        return V.mean(), w @ g

    fd_V, fd_g = np.zeros(20), np.zeros(20)
    for j in range(20):
        base = cfg.sigma[j] if j < 10 else cfg.epsilon_k[j - 10]
        h = 1e-6 * base
        lp, lm = losses(_perturbed(cfg, j, h)), losses(_perturbed(cfg, j, -h))
        fd_V[j] = (lp[0] - lm[0]) / (2 * h)
        fd_g[j] = (lp[1] - lm[1]) / (2 * h)
    assert np.all(np.abs(ad_V - fd_V) <= 1e-6 * np.abs(fd_V) + 1e-7 * np.abs(fd_V).max())
    assert np.all(np.abs(ad_g - fd_g) <= 1e-4 * np.abs(fd_g) + 1e-4 * np.abs(fd_g).max())


def test_dual_rejects_unsupported_configs(orc):
    cfg, u = _small()
    acc = np.zeros_like(u.pos)
    c = copy.deepcopy(cfg)
    c.enable_thermostat = True
    with pytest.raises(ValueError):
        orc.adjoint_forward(c, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 2)
    with pytest.raises(ValueError):  # r_max + support * width beyond the 5.75 cutoff
        orc.adjoint_forward(cfg, u.pos, u.vel, acc, u.elem, u.charge, u.mass, 2, gr_bins=10, gr_rmax=5.5,
                            gr_width=0.115, gr_support=6.0)
