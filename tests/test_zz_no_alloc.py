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


def test_noalloc_gr_rejects_a_grid_beyond_its_limit(gpu):
    from genesis_b200._lib import GxError, radial_distribution_noalloc
    pos = np.zeros((10, 3))
    with pytest.raises(GxError) as e:
        radial_distribution_noalloc(pos, (200.0, 200.0, 200.0), 1.0, 64)  # 200^3 cells > 65536
    assert e.value.status == -4
