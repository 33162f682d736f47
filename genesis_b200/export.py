"""Observability exports of the device state: the metrics CSV and XYZ
position frames of src/export/mod.rs, with the same bytes.

* ``write_frame`` replaces export::write_frame (mod.rs:152-172): the frame
  text is formatted on the GPU (gx_xyz_frame) from the resident positions
  and written to ``{prefix}_{tick:08}.xyz``.
* ``csv_row`` / ``append_csv`` restate export::csv_row / append_csv
  (mod.rs:99-150) with bond_species, chemical_compositions and
  chemical_reactions (mod.rs:23-97): one row per sampled tick, formatted on
  the host like the reference's own (a few hundred bytes a sample).

Numbers follow Rust's ``{:.N}``: the exact binary value rounded to N
decimals, ties to even (Python's own fixed-point formatting does the same),
with Rust's spellings of the non-finite values.
"""
from __future__ import annotations

import math
from pathlib import Path

from . import elements as E

CSV_HEADER = ("tick,time_s,entities,energy_total,energy_kinetic,energy_potential,energy_avg,temperature_avg,"
              "mean_speed,density,collisions,systems_run,fps,memory_kb,aggregates,largest,monomers,bound_pairs,"
              "bonded_pairs,bonds_formed,bond_lifetime_ticks,bond_energy,bond_species,chemical_aggregates,"
              "chemical_appeared,chemical_disappeared,chemical_fusions,chemical_scissions,chemical_compositions,"
              "chemical_reactions")  # mod.rs:14


def fixed(x: float, digits: int) -> str:
    """Rust's ``{:.digits}`` of an f64."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return f"{x:.{digits}f}"


def bond_species(matrix) -> str:
    """Non-zero entries of the symmetric species matrix (lower triangle with
    the diagonal), 'A-B:count' sorted by count then name, ';' joined
    (mod.rs:23-47)."""
    n = len(E.SYMBOLS)
    pairs = []
    for ia in range(n):
        for ib in range(ia + 1):
            k = ia * n + ib
            c = float(matrix[k]) if k < len(matrix) else 0.0
            if c > 0.0:
                pairs.append((f"{E.SYMBOLS[ia]}-{E.SYMBOLS[ib]}", int(c)))
    pairs.sort(key=lambda p: (-p[1], p[0]))
    return ";".join(f"{s}:{c}" for s, c in pairs)


def chemical_compositions(chemical) -> str:
    """'formula:count@mean' per composition, ';' joined (mod.rs:52-64)."""
    if not chemical:
        return ""
    return ";".join(f"{f}:{int(c)}@{fixed(m, 2)}" for f, c, m in chemical["compositions"])


def chemical_reactions(chemical) -> str:
    """'A+B->C' per transition with 'xN' when seen N > 1 times, ';' joined
    (mod.rs:71-96)."""
    if not chemical:
        return ""
    out = []
    for reactants, products, count in chemical["reactions"]:
        s = "+".join(reactants) + "->" + "+".join(products)
        if count > 1:
            s += f"x{int(count)}"
        out.append(s)
    return ";".join(out)


def csv_row(s: dict) -> str:
    """One metrics row (mod.rs:99-137).  ``s`` carries StatsSnapshot's
    fields (src/stats/mod.rs): tick, time, entities, energy_total,
    energy_potential, energy_avg, temperature_avg, mean_speed, density,
    collisions, systems_run, fps, memory_bytes, structure (dict with
    aggregates, monomers, largest, bound_pairs, or None), bonded_pairs,
    bonds_formed, bond_lifetime_ticks, bond_energy, bond_matrix (10 x 10)
    and chemical (the chemistry lens's sample, or None)."""
    st = s.get("structure")
    aggregates, monomers, largest, bound = ((st["aggregates"], st["monomers"], st["largest"], st["bound_pairs"])
                                            if st else (0, 0, 0, 0))
    ch = s.get("chemical")
    g = (lambda k: ch[k]) if ch else (lambda k: 0)
    cols = [
        str(int(s["tick"])), fixed(s["time"], 6), str(int(s["entities"])), fixed(s["energy_total"], 6),
        fixed(s["energy_total"] - s["energy_potential"], 6), fixed(s["energy_potential"], 6),
        fixed(s["energy_avg"], 6), fixed(s["temperature_avg"], 6), fixed(s["mean_speed"], 6),
        fixed(s["density"], 6), str(int(s["collisions"])), str(int(s["systems_run"])), fixed(s["fps"], 3),
        fixed(s["memory_bytes"] / 1024.0, 1), str(int(aggregates)), str(int(largest)), str(int(monomers)),
        str(int(bound)), str(int(s["bonded_pairs"])), str(int(s["bonds_formed"])),
        fixed(s["bond_lifetime_ticks"], 1), fixed(s["bond_energy"], 6), bond_species(s["bond_matrix"]),
        str(int(g("aggregates"))), str(int(g("appeared"))), str(int(g("disappeared"))), str(int(g("fusions"))),
        str(int(g("scissions"))), chemical_compositions(ch), chemical_reactions(ch),
    ]
    return ",".join(cols)


def append_csv(path, s: dict) -> None:
    """Appends one row, writing the header first when the file is new
    (mod.rs:139-150)."""
    path = Path(path)
    fresh = not path.exists()
    with open(path, "a", encoding="utf-8") as f:
        if fresh:
            f.write(CSV_HEADER + "\n")
        f.write(csv_row(s) + "\n")


def frame_path(prefix, tick: int) -> str:
    """``{prefix}_{tick:08}.xyz`` (mod.rs:170)."""
    return f"{prefix}_{int(tick):08d}.xyz"


def write_frame(prefix, tick: int, handle) -> str:
    """The handle's current positions as one XYZ frame file, formatted on
    the device; returns the path."""
    path = frame_path(prefix, tick)
    Path(path).write_bytes(handle.xyz_frame(tick))
    return path
