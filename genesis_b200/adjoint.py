"""Gradients of smoothed observables with respect to the element table.

The C5 workload: 20^3 = 8,000 atoms on the lattice, 60 K, NVE, a 200-tick
horizon with a checkpoint every 20 ticks.  Two losses:

* ``potential``: the time-averaged potential energy <V> = mean_t V_t;
* ``gr``: sum_k (gbar_k - target_k)^2 of the Gaussian-kernel pair
  distribution averaged over every tick, kernel width w = 0.05 max sigma
  (0.115 for the built-in table), truncated at 6 w, bin centres
  r_k = (k + 1/2) * 5.0 / 50.  The target is the same observable of a run
  whose sigma are all 2 % larger (a fitting problem with a known answer).

Gradients are taken with respect to the 10 sigma and 10 epsilon_k of the
element table (src/physics/forces.rs:43-54) through gx_adjoint_forward /
gx_adjoint_backward; :func:`fd_gradients` gives the central finite
differences of the same FP64 forward for checking.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np

from . import elements as E
from . import workloads as W
from ._lib import Handle

GR_WIDTH_FACTOR = 0.05      # w = 0.05 * max sigma
GR_SUPPORT = 6.0            # kernel truncated at 6 w
GR_RMAX = 5.0
GR_BINS = 50
TARGET_SIGMA_SCALE = 1.02


@dataclass
class AdjointSpec:
    nsteps: int = 200
    checkpoint_every: int = 20
    gr_bins: int = GR_BINS
    gr_every: int = 1
    gr_rmax: float = GR_RMAX
    gr_width: float = GR_WIDTH_FACTOR * max(E.SIGMA)
    gr_support: float = GR_SUPPORT

    def kwargs(self) -> dict:
        return dict(checkpoint_every=self.checkpoint_every, gr_bins=self.gr_bins, gr_every=self.gr_every,
                    gr_rmax=self.gr_rmax, gr_width=self.gr_width, gr_support=self.gr_support)


def with_params(cfg, sigma=None, epsilon_k=None):
    c = copy.deepcopy(cfg)
    if sigma is not None:
        c.sigma = tuple(float(x) for x in sigma)
    if epsilon_k is not None:
        c.epsilon_k = tuple(float(x) for x in epsilon_k)
    return c


def forward(cfg, universe, spec: AdjointSpec, device: int = 0, precision: str = "fp64"):
    """(V per tick, time-averaged g) of the trajectory: FP64, or the mixed
    method (FP32 pair law, fixed-point force sums) with ``precision="mixed"``."""
    with Handle(cfg, precision, device) as h:
        h.set_universe(universe)
        return h.adjoint_forward(spec.nsteps, **spec.kwargs())


def potential_loss(V: np.ndarray):
    """<V> and its cotangent dL/dV_t."""
    return float(np.mean(V)), np.full(len(V), 1.0 / len(V))


def gr_loss(g: np.ndarray, target: np.ndarray):
    """sum_k (g_k - target_k)^2 and its cotangent dL/dg_k."""
    d = g - target
    return float(d @ d), 2.0 * d


def gr_target(cfg, universe, spec: AdjointSpec, device: int = 0) -> np.ndarray:
    c = with_params(cfg, sigma=np.asarray(cfg.sigma) * TARGET_SIGMA_SCALE)
    return forward(c, universe, spec, device)[1]


def gradients(cfg, universe, spec: AdjointSpec, target=None, device: int = 0, precision: str = "fp64"):
    """Losses and adjoint gradients.  Returns a dict with
    ``potential`` (<V>, dsigma[10], deps[10]) and, with a target, ``gr``.
    ``precision="mixed"`` runs the forward in the mixed method (FP32 pair
    law, fixed-point force sums); the adjoint is FP64 either way."""
    out = {}
    with Handle(cfg, precision, device) as h:
        h.set_universe(universe)
        V, g = h.adjoint_forward(spec.nsteps, **spec.kwargs())
        lv, cv = potential_loss(V)
        gs, ge = h.adjoint_backward(dl_dpotential=cv)
        out["potential"] = (lv, gs, ge)
        if target is not None and g is not None:
            lg, cg = gr_loss(g, target)
            gs, ge = h.adjoint_backward(dl_dgr=cg)
            out["gr"] = (lg, gs, ge)
    return out


def fd_gradients(cfg, universe, spec: AdjointSpec, target=None, rel_step: float = 1e-5, device: int = 0,
                 which=range(20)):
    """Central differences of the losses over the 20 parameters (step
    ``rel_step`` times the parameter).  Returns {"potential": [20], "gr": [20]}."""
    sig0, eps0 = np.asarray(cfg.sigma, dtype=float), np.asarray(cfg.epsilon_k, dtype=float)
    res = {"potential": np.full(20, np.nan), "gr": np.full(20, np.nan)}
    for j in which:
        vals = []
        for sgn in (+1.0, -1.0):
            s, e = sig0.copy(), eps0.copy()
            if j < 10:
                h = rel_step * s[j]
                s[j] += sgn * h
            else:
                h = rel_step * e[j - 10]
                e[j - 10] += sgn * h
            V, g = forward(with_params(cfg, s, e), universe, spec, device)
            vals.append((potential_loss(V)[0], gr_loss(g, target)[0] if target is not None else np.nan))
        res["potential"][j] = (vals[0][0] - vals[1][0]) / (2 * h)
        res["gr"][j] = (vals[0][1] - vals[1][1]) / (2 * h)
    return res


def c5():
    """The C5 workload and its universe."""
    wl = W.C5
    return wl, wl.config(), wl.generate()
