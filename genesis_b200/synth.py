"""Seeded synthetic universes: cubic lattices with Gaussian jitter, species
draws and Maxwell-Boltzmann velocities.

The reference seeds with rand 0.8 + rand_xoshiro 0.6 (src/rng/mod.rs:24-63,
src/universe/mod.rs:221-273), crates that are not vendored, so its particle
sets cannot be reproduced here.  This generator restates the same recipe with
published generators: each atom has its own xoshiro256++ stream (Blackman &
Vigna) whose 256-bit state comes from SplitMix64 (Steele, Lea & Flood) applied
to (seed, atom index), so every atom's draws are independent of the others
and the whole lattice is generated with vectorised numpy.  Normals use the
Box-Muller cosine branch, as Rng::gaussian does (src/rng/mod.rs:50-54).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import elements as E

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)
_ATOM = np.uint64(0xD1B54A32D192ED03)


def _splitmix_next(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One SplitMix64 step on an array of states: (new_state, output)."""
    with np.errstate(over="ignore"):
        x = x + _GOLD
        z = x.copy()
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
        z = z ^ (z >> np.uint64(31))
    return x, z


def _rotl(x: np.ndarray, k: int) -> np.ndarray:
    return (x << np.uint64(k)) | (x >> np.uint64(64 - k))


class AtomStreams:
    """Per-atom xoshiro256++ streams advanced in lock step."""

    def __init__(self, seed: int, n: int, salt: int = 0):
        base = np.full(1, np.uint64(seed & 0xFFFFFFFFFFFFFFFF))
        base, k0 = _splitmix_next(base ^ np.uint64(salt & 0xFFFFFFFFFFFFFFFF))
        with np.errstate(over="ignore"):
            x = k0[0] + np.arange(n, dtype=np.uint64) * _ATOM
        s = []
        for _ in range(4):
            x, z = _splitmix_next(x)
            s.append(z)
        self.s = s

    def next_u64(self) -> np.ndarray:
        s0, s1, s2, s3 = self.s
        with np.errstate(over="ignore"):
            result = _rotl(s0 + s3, 23) + s0
        t = s1 << np.uint64(17)
        s2 = s2 ^ s0
        s3 = s3 ^ s1
        s1 = s1 ^ s2
        s0 = s0 ^ s3
        s2 = s2 ^ t
        s3 = _rotl(s3, 45)
        self.s = [s0, s1, s2, s3]
        return result

    def unit(self) -> np.ndarray:
        """Uniform doubles in [0, 1) from the top 53 bits."""
        return (self.next_u64() >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def normal(self) -> np.ndarray:
        u1 = np.maximum(self.unit(), np.finfo(np.float64).tiny)
        u2 = self.unit()
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


@dataclass
class Universe:
    """Host columns of one universe, in ECS slot order."""

    box: np.ndarray      # (3,)
    pos: np.ndarray      # (n, 3) f64
    vel: np.ndarray      # (n, 3) f64
    elem: np.ndarray     # (n,) u8 element index
    charge: np.ndarray   # (n,) f64
    mass: np.ndarray     # (n,) f64
    entity: np.ndarray   # (n,) u32 EntityId::index

    @property
    def n(self) -> int:
        return len(self.elem)


def lattice(n_side: int, spacing: float, jitter_frac: float, temperature: float,
            thermal_constant: float, seed: int, species: tuple[int, ...] | None = None,
            fixed_fractions: dict[int, float] | None = None,
            charges: tuple[float, ...] = E.CHARGE, salt: int = 0) -> Universe:
    """n_side^3 atoms on a cubic lattice of the given spacing (box n*spacing),
    site centres (i+1/2)s - L/2 as in seed_lattice (src/universe/mod.rs:221-243),
    Gaussian jitter jitter_frac*s per axis, species uniform over `species`
    (or exact fractions, shuffled), velocities N(0, sqrt(k T / m)) per
    component (src/universe/mod.rs:265-270) with net momentum removed."""
    n = n_side ** 3
    L = n_side * spacing
    box = np.array([L, L, L], dtype=np.float64)
    st = AtomStreams(seed, n, salt)
    g = np.arange(n_side, dtype=np.float64)
    ix, iy, iz = np.meshgrid(g, g, g, indexing="ij")  # ix outer, iz inner
    base = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1)
    base = (base + 0.5) * spacing - 0.5 * L
    jit = jitter_frac * spacing
    pos = base + np.stack([st.normal(), st.normal(), st.normal()], axis=1) * jit
    species = tuple(range(E.COUNT)) if species is None else tuple(species)
    u = st.unit()
    if fixed_fractions:
        keys = st.next_u64()
        order = np.argsort(keys, kind="stable")
        elem = np.empty(n, dtype=np.uint8)
        start = 0
        items = list(fixed_fractions.items())
        for k, (e, frac) in enumerate(items):
            cnt = n - start if k == len(items) - 1 else int(round(frac * n))
            elem[order[start:start + cnt]] = e
            start += cnt
    else:
        idx = np.minimum((u * len(species)).astype(np.int64), len(species) - 1)
        elem = np.asarray(species, dtype=np.uint8)[idx]
    mass = np.asarray(E.MASS, dtype=np.float64)[elem]
    charge = np.asarray(charges, dtype=np.float64)[elem]
    sig_v = np.sqrt(thermal_constant * temperature / mass)
    vel = np.stack([st.normal(), st.normal(), st.normal()], axis=1) * sig_v[:, None]
    p = (vel * mass[:, None]).sum(axis=0) / mass.sum()
    vel = vel - p[None, :]
    return Universe(box=box, pos=np.ascontiguousarray(pos), vel=np.ascontiguousarray(vel),
                    elem=elem, charge=charge, mass=mass,
                    entity=np.arange(n, dtype=np.uint32))


def uniform_box(n: int, box: tuple[float, float, float], seed: int,
                species: tuple[int, ...] | None = None, salt: int = 0) -> Universe:
    """n atoms uniform in the box (Rng::in_box, src/rng/mod.rs:57-63), zero velocity."""
    st = AtomStreams(seed, n, salt)
    b = np.asarray(box, dtype=np.float64)
    pos = np.stack([(st.unit() - 0.5) * b[0], (st.unit() - 0.5) * b[1], (st.unit() - 0.5) * b[2]], axis=1)
    species = tuple(range(E.COUNT)) if species is None else tuple(species)
    idx = np.minimum((st.unit() * len(species)).astype(np.int64), len(species) - 1)
    elem = np.asarray(species, dtype=np.uint8)[idx]
    mass = np.asarray(E.MASS, dtype=np.float64)[elem]
    return Universe(box=b, pos=np.ascontiguousarray(pos), vel=np.zeros((n, 3)), elem=elem,
                    charge=np.asarray(E.CHARGE, dtype=np.float64)[elem], mass=mass,
                    entity=np.arange(n, dtype=np.uint32))
