"""Host-side reading of a g(r) histogram from gx_radial_distribution."""
from __future__ import annotations

import math

import numpy as np


def peak_in(bins, dr: float, r_from: float, r_to: float):
    """RadialDistribution::peak_in (src/analysis/mod.rs:67-79): the largest
    g over the bins whose centre r = (i + 1/2) dr lies in [r_from, r_to], as
    (r, g), the first such bin on ties; None when no bin centre is in the
    window.  Below half the box it picks the first coordination shell."""
    best = None
    best_g = -math.inf
    for i, g in enumerate(np.asarray(bins, dtype=np.float64)):
        r = (i + 0.5) * dr
        if r < r_from or r > r_to:
            continue
        if g > best_g:
            best, best_g = (r, float(g)), float(g)
    return best
