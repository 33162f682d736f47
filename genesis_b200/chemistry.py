"""The bond-graph chemistry lens: BondStructureSystem::run
(src/systems/bond_structure.rs:55-246) over the device's bond components.

The device (gx_bond_components) labels every atom with the smallest slot of
its component of the persistent-bond graph and gives the raw pair energy of
every bond; this module turns them into the reference's ChemicalStructure
resource (src/stats/mod.rs:93-147): the components with their stoichiometry
(bond_components / formula, src/analysis/mod.rs:331-434), the composition
histogram with each formula's mean binding energy, and the lifecycle
between samples (aggregates that appeared, disappeared, fused or split,
and the reactions those transitions imply).  Runs every structure interval,
on the host like the reference's own system.
"""
from __future__ import annotations

import numpy as np

from . import elements as E

NO_COMPONENT = 0xFFFFFFFF


def formula(counts) -> str:
    """Element symbols by descending multiplicity, then symbol, joined by
    '-', the multiplicity written when above 1 (analysis/mod.rs:417-434)."""
    parts = sorted(((int(c), E.SYMBOLS[i]) for i, c in enumerate(counts) if c > 0), key=lambda p: (-p[0], p[1]))
    return "-".join(f"{s}{c}" if c > 1 else s for c, s in parts)


def components(labels: np.ndarray, elem: np.ndarray):
    """(members, composition) of each component: members is a list of
    sorted slot arrays, composition an (n_components, 10) count matrix."""
    labels = np.asarray(labels, dtype=np.uint64)
    slots = np.nonzero(labels != NO_COMPONENT)[0]
    if len(slots) == 0:
        return [], np.zeros((0, len(E.SYMBOLS)), dtype=np.int64)
    lab = labels[slots]
    order = np.lexsort((slots, lab))
    slots, lab = slots[order], lab[order]
    starts = np.flatnonzero(np.r_[True, lab[1:] != lab[:-1]])
    group = np.cumsum(np.r_[True, lab[1:] != lab[:-1]]) - 1
    comp = np.zeros((len(starts), len(E.SYMBOLS)), dtype=np.int64)
    np.add.at(comp, (group, np.asarray(elem)[slots].astype(np.int64)), 1)
    members = np.split(slots, starts[1:])
    return members, comp


class BondStructureLens:
    """One sample per call; keeps the previous sample's aggregates."""

    def __init__(self):
        self.prev: list[tuple[tuple, str]] = []

    def sample(self, labels, elem, bonds, energy, n_entities: int) -> dict:
        labels = np.asarray(labels)
        members, comp = components(labels, elem)
        forms = [formula(c) for c in comp]
        # binding: the raw energies of each component's distinct bonds
        # (bond_structure.rs:98-117), summed in increasing (a, b) order
        bonds = np.asarray(bonds, dtype=np.int64).reshape(-1, 2)
        energy = np.asarray(energy, dtype=np.float64)
        binding = np.zeros(len(members))
        if len(bonds):
            lo, hi = bonds.min(axis=1), bonds.max(axis=1)
            keep = lo != hi
            key = (lo[keep] << 32) | hi[keep]
            ukey, first = np.unique(key, return_index=True)
            e = energy[np.flatnonzero(keep)[first]]
            root = labels[(ukey >> 32).astype(np.int64)].astype(np.uint64)
            roots = np.array([m[0] for m in members], dtype=np.uint64)  # a component's label is its smallest slot
            np.add.at(binding, np.searchsorted(roots, root), e)
        sizes = np.array([len(m) for m in members], dtype=np.int64)
        # composition histogram, formulas in the reference's component order
        comp_order = sorted(range(len(members)), key=lambda i: (-sizes[i], forms[i]))
        by_formula: dict[str, list] = {}
        for i in comp_order:
            acc = by_formula.setdefault(forms[i], [0.0, 0])
            acc[0] += binding[i]
            acc[1] += 1
        compositions = sorted(((f, c, s / c) for f, (s, c) in by_formula.items()), key=lambda x: (-x[1], x[0]))
        # lifecycle against the previous sample (bond_structure.rs:139-224)
        current = [(tuple(int(x) for x in members[i]), forms[i]) for i in comp_order]
        cur = dict(current)
        prev = dict(self.prev)
        new_keys = [k for k in cur if k not in prev]
        gone_keys = [k for k in prev if k not in cur]
        # an aggregate of one sample lies inside one of the other only if
        # they share a member: index the members by aggregate
        owner_prev = {m: p for p in prev for m in p}
        owner_cur = {m: c for c in cur for m in c}

        def inside(key, owner, other_owner):
            # the aggregates of the other sample wholly inside `key`, and
            # whether they cover it
            cand = {owner[m] for m in key if m in owner}
            parts = [c for c in cand if all(other_owner.get(m) == key for m in c)]
            return parts, sum(len(c) for c in parts) == len(key)

        reactions: dict[tuple, int] = {}
        fusions = scissions = 0
        for k in new_keys:
            parts, covered = inside(k, owner_prev, owner_cur)
            if len(parts) >= 2 and covered:
                fusions += 1
                r = (tuple(sorted(prev[p] for p in parts)), (cur[k],))
                reactions[r] = reactions.get(r, 0) + 1
        for k in gone_keys:
            parts, covered = inside(k, owner_cur, owner_prev)
            if len(parts) >= 2 and covered:
                scissions += 1
                r = ((prev[k],), tuple(sorted(cur[c] for c in parts)))
                reactions[r] = reactions.get(r, 0) + 1
        rx = sorted(([list(a), list(b), c] for (a, b), c in reactions.items()), key=lambda x: (-x[2], "+".join(x[0])))
        bound = int(sizes.sum())
        self.prev = current
        return {"aggregates": len(members), "bound_entities": bound, "monomers": max(int(n_entities) - bound, 0),
                "largest": int(sizes.max()) if len(sizes) else 0,
                "compositions": [(f, int(c), float(m)) for f, c, m in compositions],
                "appeared": len(new_keys), "disappeared": len(gone_keys), "fusions": fusions,
                "scissions": scissions, "reactions": [(r[0], r[1], int(r[2])) for r in rx]}
