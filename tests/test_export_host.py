"""The export formats of src/export/mod.rs on the host: the metrics CSV row
(the reference's own test, mod.rs:181-248), the XYZ frame oracle (the
reference's own test, mod.rs:250-280) and the exact fixed-point algorithm
the device formatter uses, checked here in Python integers against
Python's own correctly rounded formatting."""
from __future__ import annotations

import math
import struct

import numpy as np

from genesis_b200 import export as X
from oracle import oracle as orc


def _snapshot():
    matrix = [0.0] * 100
    matrix[5 * 10 + 4] = 3.0  # Na-O
    return {
        "tick": 7, "time": 0.42, "entities": 3, "energy_total": 5.0, "energy_avg": 1.5, "energy_potential": 2.0,
        "temperature_avg": 300.0, "mean_speed": 1.1, "density": 0.02, "collisions": 1, "systems_run": 6,
        "fps": 10.0, "memory_bytes": 2048,
        "structure": {"aggregates": 1, "monomers": 1, "largest": 2, "bound_pairs": 1},
        "bonded_pairs": 3, "bonds_formed": 4, "bond_lifetime_ticks": 25.0, "bond_energy": 0.5,
        "bond_matrix": matrix,
        "chemical": {"aggregates": 2, "appeared": 2, "disappeared": 0, "fusions": 1, "scissions": 1,
                     "compositions": [("Na-O", 2, -0.53), ("Na2-O", 1, -0.71)],
                     "reactions": [(["Na-O", "Na-O"], ["Na2-O2"], 2), (["Na2-O2"], ["Na-O", "Na-O"], 1)]},
    }


def test_csv_row_matches_the_reference_known_answer():
    row = X.csv_row(_snapshot())
    assert len(X.CSV_HEADER.split(",")) == len(row.split(",")) == 30
    assert row.startswith("7,0.420000,3,")
    assert row.endswith("Na-O:3,2,2,0,1,1,Na-O:2@-0.53;Na2-O:1@-0.71,Na-O+Na-O->Na2-O2x2;Na2-O2->Na-O+Na-O")


def test_csv_row_without_lenses_and_the_header_once(tmp_path):
    s = _snapshot()
    s["structure"] = None
    s["chemical"] = None
    s["bond_matrix"] = [0.0] * 100
    row = X.csv_row(s)
    assert len(row.split(",")) == 30
    assert row.endswith(",2.0,0,0,0,0,3,4,25.0,0.500000,,0,0,0,0,0,,")
    p = tmp_path / "m.csv"
    X.append_csv(p, s)
    X.append_csv(p, s)
    lines = p.read_text().splitlines()
    assert lines[0] == X.CSV_HEADER and lines[1] == lines[2] == row


def test_bond_species_orders_by_count_then_name():
    m = [0.0] * 100
    m[6 * 10 + 4] = 12.0  # Si-O
    m[5 * 10 + 4] = 3.0   # Na-O
    m[0] = 3.0            # H-H
    m[4 * 10 + 5] = 99.0  # upper triangle: ignored
    assert X.bond_species(m) == "Si-O:12;H-H:3;Na-O:3"
    assert X.bond_species([0.0] * 100) == ""


def test_fixed_uses_rust_spellings_and_ties_to_even():
    assert X.fixed(float("nan"), 6) == "NaN" and X.fixed(float("inf"), 2) == "inf"
    assert X.fixed(float("-inf"), 1) == "-inf" and X.fixed(-0.0, 6) == "-0.000000"
    assert X.fixed(0.125, 2) == "0.12" and X.fixed(0.375, 2) == "0.38"
    assert X.frame_path("out/frame", 42) == "out/frame_00000042.xyz"


def test_xyz_oracle_matches_the_reference_known_answer():
    pos = np.array([[1.0, 2.0, 3.0], [-1.0, 0.0, 0.5]])
    text = orc.xyz_frame(0, pos, np.array([0, 2])).decode()
    lines = text.splitlines()
    assert lines[:2] == ["2", "frame 0"]
    assert sorted(lines[2:]) == ["C -1.000000 0.000000 0.500000", "H 1.000000 2.000000 3.000000"]
    assert text.endswith("\n")


def _edge_values():
    v = [0.0, -0.0, 1e-9, -1e-9, 5e-7, -5e-7, 4.9999999999999996e-07, 5.000000000000001e-07, 1.5e-6, 2.5e-6,
         0.9999995, 0.99999949999999994, 999999.9999995, 999999.99999949, 1e15, 1e20, 1e23, -1e23,
         2.0 ** 99, -(2.0 ** 99.9), 2.0 ** -1074, -(2.0 ** -1022), 123.456789, -176.64, 176.64, 0.1, 0.3]
    v += [k / 128.0 for k in range(-300, 300, 3)] + [k / 2 ** 20 for k in range(1, 400, 7)]
    return v


def _rand_values(n=40000, seed=3):
    rng = np.random.default_rng(seed)
    mags = 10.0 ** rng.uniform(-9, 29, n)
    return list(np.where(rng.random(n) < 0.5, -mags, mags)) + list(rng.uniform(-200, 200, n))


def _ndig64(v: int) -> int:
    t = (max(v, 1).bit_length() * 1233) >> 12
    return max(t + 1 - (1 if v < 10 ** t else 0), 1)


def _fixed6_int(x: float) -> str:
    """The device formatter's algorithm (gx_export.cu to_fixed6 and
    fixed6_put) in Python integers."""
    bits = struct.unpack("<Q", struct.pack("<d", x))[0]
    neg, ex, fr = bits >> 63, (bits >> 52) & 0x7FF, bits & ((1 << 52) - 1)
    assert ex != 0x7FF and ex < 1023 + 100
    m = (fr | (1 << 52)) if ex else fr
    e = (ex if ex else 1) - 1075
    if e >= 0:
        ip, frac = m << e, 0
        assert ip < 2 ** 100
    elif -e > 74:
        ip, frac = 0, 0
    else:
        s = -e
        p = m * 10 ** 6
        assert p < 2 ** 73
        q, rem, half = p >> s, p & ((1 << s) - 1), 1 << (s - 1)
        n = q + (1 if rem > half or (rem == half and q & 1) else 0)
        ip = m >> s
        frac = n - ip * 10 ** 6
        assert 0 <= frac <= 10 ** 6
        if frac == 10 ** 6:
            ip, frac = ip + 1, 0
    nd = _ndig64(ip) if ip < 2 ** 64 else _ndig64(ip // 10 ** 19) + 19
    assert nd == len(str(ip)) <= 31
    return ("-" if neg else "") + f"{ip}.{frac:06d}"


def test_digit_count_formula():
    for d in range(1, 21):
        for v in (10 ** (d - 1), 10 ** (d - 1) + 1, 2 * 10 ** (d - 1), 10 ** d - 1):
            if v < 2 ** 64:
                assert _ndig64(v) == d, v
    for b in range(64):
        for v in (2 ** b - 1, 2 ** b, 2 ** b + 1):
            if v < 2 ** 64:
                assert _ndig64(v) == len(str(v)), v


def test_device_algorithm_matches_correct_rounding():
    for x in _edge_values() + _rand_values():
        x = float(x)
        assert _fixed6_int(x) == f"{x:.6f}", x


def test_c_oracle_matches_python_formatting():
    vals = np.array(_edge_values() + _rand_values(3000) + [math.nan, math.inf, -math.inf])
    vals = np.concatenate([vals, np.zeros((-len(vals)) % 3)]).reshape(-1, 3)
    elem = np.arange(len(vals)) % 10
    assert orc.xyz_frame(17, vals, elem) == orc.xyz_frame_py(17, vals, elem)
