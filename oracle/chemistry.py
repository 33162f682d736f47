"""Test infrastructure only: a plain-Python restatement of the bond-graph
chemistry lens, the checker for genesis_b200.chemistry and for
gx_bond_components.  Nothing in the product imports it.

Follows, step by step:
  bond_components      src/analysis/mod.rs:331-411 (union-find with rank,
                       duplicate and dangling edges ignored, components
                       sorted by size then formula)
  formula              src/analysis/mod.rs:413-434
  pair_potential_raw   src/physics/forces.rs:355-384 with lj_raw
                       (forces.rs:346-353), well_curvature (forces.rs:193-195)
                       and equilibrium_distance (forces.rs:281-283)
  BondStructure.sample BondStructureSystem::run,
                       src/systems/bond_structure.rs:55-246 (binding energy
                       per component, composition histogram, lifecycle:
                       appeared, disappeared, fusions, scissions, reactions)

Pure-Python loops over small cases; the per-pair energies are IEEE double
arithmetic in the reference's operation order.  The reference sums a
component's binding over a hash set (an unspecified order); this
restatement sums in increasing (a, b) order.
"""
from __future__ import annotations

import math

SYMBOLS = ("H", "He", "C", "N", "O", "Na", "Si", "P", "S", "Fe")  # src/components/atom_type.rs:64-77
NELEM = len(SYMBOLS)


def formula(composition) -> str:
    """Element symbols by descending multiplicity, then symbol; '-' joined;
    the multiplicity written only when above 1 (analysis/mod.rs:417-434)."""
    parts = [(c, SYMBOLS[i]) for i, c in enumerate(composition) if c > 0]
    parts.sort(key=lambda p: (-p[0], p[1]))
    return "-".join(f"{s}{c}" if c > 1 else s for c, s in parts)


def _find(parent, x):
    while parent[x] != x:
        parent[x] = parent[parent[x]]
        x = parent[x]
    return x


def _union(parent, rank, a, b):
    ra, rb = _find(parent, a), _find(parent, b)
    if ra == rb:
        return
    if rank[ra] < rank[rb]:
        ra, rb = rb, ra
    parent[rb] = ra
    if rank[ra] == rank[rb]:
        rank[ra] += 1


def bond_components(entities, edges):
    """entities: [(entity id, element index)], edges: [(a, b)].  Returns
    [{size, composition, formula, members, edges}] largest first."""
    n = len(entities)
    if n == 0:
        return []
    index = {e: i for i, (e, _) in enumerate(entities)}
    parent = list(range(n))
    rank = [0] * n
    seen = set()
    for a, b in edges:
        if a not in index or b not in index:
            continue
        ia, ib = index[a], index[b]
        if ia == ib:
            continue
        edge = (min(a, b), max(a, b))
        if edge in seen:
            continue
        seen.add(edge)
        _union(parent, rank, ia, ib)
    comps = {}
    for i, (e, el) in enumerate(entities):
        d = comps.setdefault(_find(parent, i), {"composition": [0] * NELEM, "members": [], "edges": []})
        d["members"].append(e)
        d["composition"][el] += 1
    for a, b in sorted(seen):
        comps[_find(parent, index[a])]["edges"].append((a, b))
    out = []
    for d in comps.values():
        members = sorted(d["members"])
        out.append({"size": len(members), "composition": d["composition"], "formula": formula(d["composition"]),
                    "members": members, "edges": d["edges"]})
    out.sort(key=lambda c: (-c["size"], c["formula"]))
    return out


def pair_potential_raw(sigma, epsilon_k, charge, thermal_constant, ta, tb, r, k_e, with_coulomb, with_bond):
    sig = 0.5 * (sigma[ta] + sigma[tb])                                # mix_sigma, forces.rs:127-129
    eps = thermal_constant * math.sqrt(epsilon_k[ta] * epsilon_k[tb])  # mix_epsilon, forces.rs:132-134
    s = sig / r
    s6 = s * s * s * s * s * s
    s12 = s6 * s6
    total = 4.0 * eps * (s12 - s6)
    if with_coulomb:
        q = k_e * charge[ta] * charge[tb]
        total += q / r
    if with_bond:
        k = 72.0 * 2.0 ** (-1.0 / 3.0) * eps / (sig * sig)
        r_eq = sig * 2.0 ** (1.0 / 6.0)
        total += 0.5 * k * (r - r_eq) * (r - r_eq)
    return total


def _min_image(d, size):
    return d - size * _round_half_away(d / size)


def _round_half_away(x):
    # f64::round: half away from zero (ax - floor(ax) is exact)
    ax = abs(x)
    f = math.floor(ax)
    if ax - f >= 0.5:
        f += 1.0
    return math.copysign(f, x)


def pair_distance(pa, pb, size):
    dx, dy, dz = (_min_image(pa[k] - pb[k], size[k]) for k in range(3))
    return max(math.sqrt(dx * dx + dy * dy + dz * dz), 1e-9)


class BondStructure:
    """BondStructureSystem::run on explicit inputs: the previous sample's
    aggregates are kept between calls."""

    def __init__(self):
        self.prev = []  # [(members tuple, formula)]

    def sample(self, n_entities, elem, bonds, pos, cfg, k_e=None):
        """n_entities: world size; elem[e], pos[e]: element and position of
        entity e; bonds: [(a, b)] persistent bonds."""
        bonded = sorted({a for a, b in bonds} | {b for a, b in bonds})
        entities = [(e, int(elem[e])) for e in bonded]
        comps = bond_components(entities, bonds)
        k_e = cfg.coulomb_constant if k_e is None else k_e
        by_formula = {}
        largest = 0
        for c in comps:
            largest = max(largest, c["size"])
            binding = 0.0
            for a, b in c["edges"]:
                r = pair_distance(pos[a], pos[b], cfg.size)
                binding += pair_potential_raw(cfg.sigma, cfg.epsilon_k, cfg.charge, cfg.thermal_constant,
                                              int(elem[a]), int(elem[b]), r, k_e, cfg.enable_electrostatics,
                                              cfg.enable_bond_interaction)
            sm, cnt = by_formula.get(c["formula"], (0.0, 0))
            by_formula[c["formula"]] = (sm + binding, cnt + 1)
        compositions = [(f, cnt, sm / cnt if cnt else 0.0) for f, (sm, cnt) in by_formula.items()]
        compositions.sort(key=lambda x: (-x[1], x[0]))

        current = [(tuple(c["members"]), c["formula"]) for c in comps]
        cur_keys = {m for m, _ in current}
        prev_keys = {m for m, _ in self.prev}
        cur_f = dict(current)
        prev_f = dict(self.prev)
        reactions = {}
        fusions = scissions = 0
        for new in cur_keys - prev_keys:
            inside = [pk for pk in prev_keys if set(pk) <= set(new)]
            if len(inside) >= 2 and set().union(*map(set, inside)) == set(new):
                fusions += 1
                key = (tuple(sorted(prev_f[k] for k in inside)), (cur_f[new],))
                reactions[key] = reactions.get(key, 0) + 1
        for old in prev_keys - cur_keys:
            inside = [ck for ck in cur_keys if set(ck) <= set(old)]
            if len(inside) >= 2 and set().union(*map(set, inside)) == set(old):
                scissions += 1
                key = ((prev_f[old],), tuple(sorted(cur_f[k] for k in inside)))
                reactions[key] = reactions.get(key, 0) + 1
        rx = [(list(r), list(p), c) for (r, p), c in reactions.items()]
        rx.sort(key=lambda x: (-x[2], "+".join(x[0])))
        out = {"aggregates": len(comps), "bound_entities": len(bonded), "monomers": max(n_entities - len(bonded), 0),
               "largest": largest, "compositions": compositions, "appeared": len(cur_keys - prev_keys),
               "disappeared": len(prev_keys - cur_keys), "fusions": fusions, "scissions": scissions,
               "reactions": rx}
        self.prev = current
        return out
