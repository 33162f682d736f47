"""Universe configuration: the reference's TOML files, read with the same
defaults and fail-fast validation (src/config/mod.rs:15-286).

Only the fields the hot path and its observers read are kept typed; the rest
of the file is accepted and preserved in ``raw``.
"""
from __future__ import annotations

import math
import tomllib
from dataclasses import dataclass, field
from pathlib import Path

from . import elements as E


class ConfigError(ValueError):
    """Invalid configuration (ConfigError, src/config/mod.rs:318-345)."""


@dataclass
class Config:
    name: str = "Genesis"
    size: tuple[float, float, float] = (128.0, 128.0, 128.0)
    dt: float = 1.0 / 60.0
    initial_atoms: int = 10_000
    seed_elements: tuple[int, ...] = tuple(range(E.COUNT))
    stats_history: int = 1024
    seed: int = 42
    initial_temperature: float = 300.0
    speed_limit: float = 1000.0
    thermal_constant: float = 0.01
    gravity_constant: float = 6.674e-11
    coulomb_constant: float = 1.0
    coulomb_cutoff: float = 2.5
    gravity_cutoff: float = 3.0
    thermostat_temperature: float = 300.0
    thermostat_tau: float = 20.0
    sigma: list[float] = field(default_factory=lambda: list(E.SIGMA))
    epsilon_k: list[float] = field(default_factory=lambda: list(E.EPSILON_K))
    charge: list[float] = field(default_factory=lambda: list(E.CHARGE))
    enable_movement: bool = True
    enable_boundaries: bool = True
    enable_collisions: bool = False
    particle_radius: float = 0.4  # physics.particle_radius (config/mod.rs:98-100)
    enable_forces: bool = True
    enable_electrostatics: bool = False
    enable_gravity: bool = False
    enable_thermostat: bool = False
    enable_bond_observation: bool = False
    enable_bond_interaction: bool = False
    structure_interval: int = 100
    bond_min_periods: float = 10.0
    bond_k_bind: float = 1.5
    raw: dict = field(default_factory=dict)

    @property
    def max_sigma(self) -> float:
        return max(self.sigma)


_UNIVERSE_REQUIRED = ("name", "size", "dt", "initial_atoms", "stats_history")
_PHYSICS_REQUIRED = ("initial_temperature", "speed_limit", "gravity_constant")


def _req(tbl: dict, key: str, where: str):
    if key not in tbl:
        raise ConfigError(f"missing field `{key}` in [{where}]")
    return tbl[key]


def _num(v, what: str) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise ConfigError(f"`{what}` must be a number")
    return float(v)


def from_toml(text: str) -> Config:
    """Config::from_toml (src/config/mod.rs:269-273): parse, then validate."""
    try:
        d = tomllib.loads(text)
    except tomllib.TOMLDecodeError as e:
        raise ConfigError(f"invalid TOML: {e}") from e
    for sec in ("universe", "rng", "physics", "systems"):
        if sec not in d:
            raise ConfigError(f"missing table [{sec}]")
    u, r, p = d["universe"], d["rng"], d["physics"]
    s, st = d.get("systems", {}), d.get("stats", {})
    c = Config(raw=d)
    for k in _UNIVERSE_REQUIRED:
        _req(u, k, "universe")
    for k in _PHYSICS_REQUIRED:
        _req(p, k, "physics")
    c.name = str(u["name"])
    size = u["size"]
    if not isinstance(size, dict) or not all(k in size for k in "xyz"):
        raise ConfigError("`universe.size` must be { x, y, z }")
    c.size = (_num(size["x"], "size.x"), _num(size["y"], "size.y"), _num(size["z"], "size.z"))
    c.dt = _num(u["dt"], "dt")
    c.initial_atoms = int(u["initial_atoms"])
    c.stats_history = int(u["stats_history"])
    if "elements" in u:
        idx = []
        for nm in u["elements"]:
            i = E.by_name(str(nm))
            if i is None:
                raise ConfigError(f"unknown element `{nm}` in universe.elements")
            idx.append(i)
        c.seed_elements = tuple(idx)
    c.seed = int(_req(r, "seed", "rng"))
    c.initial_temperature = _num(p["initial_temperature"], "initial_temperature")
    c.speed_limit = _num(p["speed_limit"], "speed_limit")
    c.gravity_constant = _num(p["gravity_constant"], "gravity_constant")
    for k in ("thermal_constant", "coulomb_constant", "coulomb_cutoff", "gravity_cutoff",
              "thermostat_temperature", "thermostat_tau", "particle_radius"):
        if k in p:
            setattr(c, k, _num(p[k], k))
    # Affinity table overrides (ElementTable::apply_overrides, physics/forces.rs:90-109;
    # Config::validate, config/mod.rs:277-286).
    for sym, o in (p.get("elements") or {}).items():
        i = E.by_name(sym)
        if i is None:
            raise ConfigError(f"affinity table references unknown element symbol `{sym}`")
        if "sigma" in o:
            c.sigma[i] = _num(o["sigma"], f"{sym}.sigma")
        if "epsilon_k" in o:
            c.epsilon_k[i] = _num(o["epsilon_k"], f"{sym}.epsilon_k")
        if "charge" in o:
            c.charge[i] = _num(o["charge"], f"{sym}.charge")
    for k in ("enable_movement", "enable_boundaries", "enable_collisions", "enable_forces",
              "enable_electrostatics", "enable_gravity", "enable_thermostat",
              "enable_bond_observation", "enable_bond_interaction"):
        if k in s:
            setattr(c, k, bool(s[k]))
    if "structure_interval" in st:
        c.structure_interval = int(st["structure_interval"])
    if "bond_min_periods" in st:
        c.bond_min_periods = _num(st["bond_min_periods"], "bond_min_periods")
    if "bond_k_bind" in st:
        c.bond_k_bind = _num(st["bond_k_bind"], "bond_k_bind")
    if not all(math.isfinite(x) and x > 0 for x in c.size):
        raise ConfigError("universe.size must be positive")
    return c


def from_file(path: str | Path) -> Config:
    return from_toml(Path(path).read_text())


def default_config() -> Config:
    """Config::default_config (src/config/mod.rs:233-260)."""
    return Config()
