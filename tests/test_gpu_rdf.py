"""g(r) on the device read through peak_in, against the reference's own
known answer (src/analysis/mod.rs:455-468: one pair at d = 1.7)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from genesis_b200.rdf import peak_in

pytestmark = pytest.mark.gpu

CASES = {c["id"]: c for c in json.loads(
    (Path(__file__).resolve().parent / "golden" / "reference_known_answers.json").read_text())["cases"]}


def test_pair_peak_at_the_pair_distance(gpu):
    from genesis_b200._lib import Handle
    from genesis_b200.config import default_config
    c = CASES["gr_pair_peak"]
    cfg = default_config()
    cfg.size = tuple(c["world"])
    h = Handle(cfg, "fp64")
    h.set_state(np.array([[0.0, 0.0, 0.0], [c["d"], 0.0, 0.0]]), np.zeros((2, 3)), np.zeros(2, dtype=np.uint8))
    counts, bins, r_max, dr = h.radial_distribution(c["r_max"], c["nbins"])
    assert abs(dr - c["dr"]) < 1e-12 and int(counts.sum()) == 1
    r, g = peak_in(bins, dr, *c["window"])
    assert abs(r - c["d"]) < c["peak_tol"] and g > c["g_min"]
