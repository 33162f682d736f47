"""The allocation-free g(r) entry point, checked against the allocating one.

gx_radial_distribution_noalloc exists for callers that cannot allocate
device memory (a fixed device-memory budget, or code that must not call
cudaMalloc/cudaFree because they can synchronise the device).  It keeps its
scratch in one fixed device array, so two calls in a row must each give the
counts gx_radial_distribution gives (integer bins: exact equality).  The
file sorts last so a run that stops at the first failure has run the rest.
"""
import numpy as np
import pytest

from genesis_b200 import elements as E
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _state(n_side, ticks):
    from genesis_b200._lib import Handle
    wl = W.C1.scaled(n_side)
    cfg = wl.config()
    u = wl.generate()
    h = Handle(cfg, "fp64")
    h.set_universe(u)
    if ticks:
        h.step(ticks, stats=False)
    return cfg, h


def test_noalloc_gr_matches_allocating_entry_point_twice(gpu):
    from genesis_b200._lib import radial_distribution_noalloc
    # call 1: 4096 atoms (no subsample), r_max = 3 r_c -> 2 cells per axis
    # call 2: 10648 atoms (reference subsample), different r_max and bins
    for n_side, ticks, r_max, nbins in [(16, 5, 17.25, 256), (22, 0, 9.0, 300)]:
        cfg, h = _state(n_side, ticks)
        pos, _, _ = h.get_state()
        c_ref, b_ref, rm_ref, dr_ref = h.radial_distribution(r_max, nbins, E.G_SAMPLE_CAP)
        counts, bins, rm, dr = radial_distribution_noalloc(pos, cfg.size, r_max, nbins)
        assert c_ref.sum() > 0
        assert np.array_equal(counts, c_ref)
        assert np.array_equal(bins, b_ref)
        assert rm == rm_ref and dr == dr_ref
        h.close()


def test_noalloc_gr_clustered_sample_matches_allocating_entry_point(gpu):
    """A droplet: 6,000 of 8,000 atoms inside one cell of the g(r) grid.

    Each cell lists its samples in ascending order, ranked in parallel, so a
    cell that holds most of the sample stays fast; the counts still equal the
    allocating entry point's on two calls in a row."""
    from genesis_b200._lib import Handle, radial_distribution_noalloc
    from genesis_b200 import synth
    wl = W.C1.scaled(20)
    cfg = wl.config()
    u = wl.generate()
    L = cfg.size[0]
    rng = np.random.default_rng(5)
    k = 6000
    d = rng.normal(size=(k, 3))
    d *= (rng.random(k) ** (1.0 / 3.0) * 4.0 / np.linalg.norm(d, axis=1))[:, None]
    pos = u.pos.copy()
    pos[:k] = 0.25 * L + d  # radius 4 around one point, inside a cell of edge L/2
    u2 = synth.Universe(box=u.box, pos=pos, vel=u.vel, elem=u.elem, charge=u.charge, mass=u.mass,
                        entity=u.entity)
    with Handle(cfg, "fp64") as h:
        h.set_universe(u2)
        p_dev, _, _ = h.get_state()
        c_ref, b_ref, _, _ = h.radial_distribution(0.5 * L, 128, E.G_SAMPLE_CAP)
    for _ in range(2):
        counts, bins, _, _ = radial_distribution_noalloc(p_dev, cfg.size, 0.5 * L, 128)
        assert np.array_equal(counts, c_ref)
        assert np.array_equal(bins, b_ref)


def test_noalloc_gr_rejects_a_grid_beyond_its_limit(gpu):
    from genesis_b200._lib import GxError, radial_distribution_noalloc
    pos = np.zeros((10, 3))
    with pytest.raises(GxError) as e:
        radial_distribution_noalloc(pos, (200.0, 200.0, 200.0), 1.0, 64)  # 200^3 cells > 65536
    assert e.value.status == -4
