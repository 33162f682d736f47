"""RadialDistribution::peak_in (src/analysis/mod.rs:67-79) on host bins."""
from __future__ import annotations

from genesis_b200.rdf import peak_in


def test_peak_in_window_and_ties():
    bins = [0.0, 3.0, 1.0, 3.0, 5.0]
    assert peak_in(bins, 1.0, 0.0, 4.0) == (1.5, 3.0)  # the first of the tied maxima
    assert peak_in(bins, 1.0, 2.0, 10.0) == (4.5, 5.0)
    assert peak_in(bins, 1.0, 1.5, 1.5) == (1.5, 3.0)  # bounds are inclusive
    assert peak_in(bins, 1.0, 5.0, 9.0) is None
