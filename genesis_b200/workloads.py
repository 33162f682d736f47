"""The benchmark workloads: synthetic lattices of the named shapes.

Geometry: spacing s = 1.2 x max sigma = 2.76 (Si, src/physics/forces.rs:50),
box L = n*s, r_c = 2.5 x max sigma = 5.75, dt from config/universe.toml:12.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

from . import elements as E
from . import synth
from .config import Config

DT = 0.016666666666666666  # config/universe.toml:12
SPACING_FACTOR = 1.2
JITTER_FRAC = 0.02


@dataclass
class Workload:
    name: str
    n_side: int
    temperature: float
    steps: int
    seed: int = 0
    electrostatics: bool = False
    thermostat: bool = False
    thermostat_temperature: float = 300.0
    thermostat_tau: float = 20.0
    bond_observation: bool = False
    bond_interaction: bool = False
    species: tuple[int, ...] | None = None
    fixed_fractions: dict | None = None
    gr_every: int = 0
    gr_bins: int = 256
    gr_rmax_factor: float = 3.0

    @property
    def n_atoms(self) -> int:
        return self.n_side ** 3

    def config(self) -> Config:
        c = Config()
        s = SPACING_FACTOR * max(E.SIGMA)
        L = self.n_side * s
        c.name = self.name
        c.size = (L, L, L)
        c.dt = DT
        c.initial_atoms = self.n_atoms
        c.seed = self.seed
        c.initial_temperature = self.temperature
        c.thermal_constant = 0.01
        c.enable_forces = True
        c.enable_boundaries = True
        c.enable_electrostatics = self.electrostatics
        c.enable_thermostat = self.thermostat
        c.thermostat_temperature = self.thermostat_temperature
        c.thermostat_tau = self.thermostat_tau
        c.enable_bond_observation = self.bond_observation
        c.enable_bond_interaction = self.bond_interaction
        return c

    def generate(self, salt: int = 0) -> synth.Universe:
        s = SPACING_FACTOR * max(E.SIGMA)
        return synth.lattice(self.n_side, s, JITTER_FRAC, self.temperature, 0.01, self.seed,
                             species=self.species, fixed_fractions=self.fixed_fractions, salt=salt)

    def scaled(self, n_side: int) -> "Workload":
        return replace(self, n_side=n_side)


NA, O = E.by_name("Na"), E.by_name("O")

C1 = Workload("plain LJ NVE 16^3", n_side=16, temperature=60.0, steps=1000)
C2 = Workload("ionic NVT Na/O 32^3", n_side=32, temperature=300.0, steps=5000,
              electrostatics=True, thermostat=True, thermostat_temperature=300.0,
              bond_observation=True, bond_interaction=True, species=(NA, O),
              fixed_fractions={NA: 0.5, O: 0.5})
C3 = Workload("condensation quench 128^3", n_side=128, temperature=300.0, steps=10000,
              electrostatics=True, thermostat=True, thermostat_temperature=20.0,
              gr_every=100, gr_bins=256, gr_rmax_factor=3.0)
C5 = Workload("adjoint LJ NVE 20^3", n_side=20, temperature=60.0, steps=200)

WORKLOADS = {"c1": C1, "c2": C2, "c3": C3, "c5": C5}


@dataclass
class Replica:
    n_side: int
    temperature: float
    seed: int


def sweep_replicas(count: int = 256, seed: int = 0, lo: int = 512, hi: int = 16384,
                   t_lo: float = 20.0, t_hi: float = 120.0) -> list[Replica]:
    """C4: sizes log-uniform in [lo, hi] rounded to cubes (n in [8, 25]),
    temperatures uniform in [t_lo, t_hi] (initial = Berendsen target)."""
    st = synth.AtomStreams(seed, count, salt=0x5EE9)
    u_size = st.unit()
    u_temp = st.unit()
    sizes = np.exp(np.log(lo) + u_size * (np.log(hi) - np.log(lo)))
    reps = []
    for k in range(count):
        n = int(round(sizes[k] ** (1.0 / 3.0)))
        n = min(max(n, 8), 25)
        t = t_lo + u_temp[k] * (t_hi - t_lo)
        reps.append(Replica(n_side=n, temperature=float(t), seed=seed * 1000003 + k))
    return reps


def replica_workload(r: Replica, steps: int = 2000) -> Workload:
    return Workload(f"sweep replica {r.n_side}^3 @ {r.temperature:.1f} K", n_side=r.n_side,
                    temperature=r.temperature, steps=steps, seed=r.seed, thermostat=True,
                    thermostat_temperature=r.temperature, thermostat_tau=20.0)


def lattice_rc() -> float:
    return E.LJ_CUTOFF_FACTOR * max(E.SIGMA)


def lattice_pairs_per_atom() -> float:
    s = SPACING_FACTOR * max(E.SIGMA)
    return (4.0 / 3.0) * math.pi * lattice_rc() ** 3 / s ** 3 / 2.0
