"""XYZ frames formatted on the device (gx_xyz_frame) against the oracle's
text of export::write_frame (src/export/mod.rs:152-172): the reference's own
known answer, rounding edge cases, slot order after the atoms were re-sorted
by cell, and the full 2,097,152-atom lattice byte for byte."""
from __future__ import annotations

import math

import numpy as np
import pytest

from genesis_b200 import export as X
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _handle(cfg, precision="mixed"):
    from genesis_b200._lib import Handle
    return Handle(cfg, precision)


def _small(pos, elem):
    from genesis_b200.config import default_config
    cfg = default_config()
    cfg.size = (400.0, 400.0, 400.0)
    h = _handle(cfg, "fp64")
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    h.set_state(pos, np.zeros_like(pos), np.asarray(elem, dtype=np.uint8))
    return h


def test_reference_known_answer(gpu):
    h = _small([[1.0, 2.0, 3.0], [-1.0, 0.0, 0.5]], [0, 2])
    assert h.xyz_frame(0) == b"2\nframe 0\nH 1.000000 2.000000 3.000000\nC -1.000000 0.000000 0.500000\n"


def test_rounding_edge_cases_match_the_oracle(gpu, orc):
    # ties at 6 decimals (k/128), signed zeros, values rounding across the
    # integer part, subnormals, large magnitudes, non-finite values; the
    # state is only uploaded and formatted, never stepped
    v = [0.0, -0.0, 1e-9, -1e-9, 5e-7, -5e-7, 4.9999999999999996e-07, 0.9999995, 999999.9999995, 1e15, 1e20,
         1e23, -1e23, 2.0 ** 99, -(2.0 ** 99.9), 2.0 ** -1074, -(2.0 ** -1022), 123.456789, -176.64, 0.1,
         math.nan, math.inf, -math.inf]
    v += [k / 128.0 for k in range(-300, 300, 3)]
    rng = np.random.default_rng(5)
    mags = 10.0 ** rng.uniform(-9, 29, 3000)
    v += list(np.where(rng.random(3000) < 0.5, -mags, mags))
    v += [0.0] * ((-len(v)) % 3)
    pos = np.array(v).reshape(-1, 3)
    elem = np.arange(len(pos)) % 10
    h = _small(pos, elem)
    got = h.xyz_frame(123456789012)
    assert got == orc.xyz_frame_py(123456789012, pos, elem) == orc.xyz_frame(123456789012, pos, elem)


def test_out_of_range_and_size_query(gpu):
    from genesis_b200._lib import GxError
    h = _small([[2.0 ** 100, 0.0, 0.0]], [0])
    with pytest.raises(GxError) as e:
        h.xyz_frame(0)
    assert e.value.status == -8
    h = _small([[1.0, 2.0, 3.0]], [9])
    assert h.xyz_frame(3) == b"1\nframe 3\nFe 1.000000 2.000000 3.000000\n"


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_slot_order_after_steps(gpu, orc, tmp_path, precision):
    wl = W.C2
    cfg, u = wl.config(), wl.generate()
    h = _handle(cfg, precision)
    h.set_universe(u)
    h.step(20)
    pos, _, _ = h.get_state()
    want = orc.xyz_frame(20, pos, u.elem)
    assert h.xyz_frame(20) == want
    path = X.write_frame(tmp_path / "frame", 20, h)
    assert path.endswith("frame_00000020.xyz")
    assert open(path, "rb").read() == want


def test_full_lattice_byte_for_byte(gpu, orc):
    wl = W.C3
    cfg, u = wl.config(), wl.generate()
    h = _handle(cfg)
    h.set_universe(u)
    h.step(2)
    pos, _, _ = h.get_state()
    got = h.xyz_frame(2)
    assert got.count(b"\n") == len(u.elem) + 2
    assert got == orc.xyz_frame(2, pos, u.elem)
