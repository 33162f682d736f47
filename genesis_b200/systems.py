"""Host-side mirror of the reference's plugin interface, driving the GPU path.

The reference composes a tick from systems: ``trait System { name, access,
run(&mut SystemContext) }`` (src/scheduler/system.rs:86-97), registered in
order by ``build_schedule`` (src/universe/mod.rs:355-392) and run
sequentially by ``Scheduler::run`` (src/scheduler/mod.rs:83-89).  This
module restates that interface in Python over the C ABI: the same system
names, the same Access declarations and the same order.  The ECS columns
live in a :class:`World` on the host; the GPU systems share one
:class:`GpuWorld` (one device handle) and sync columns lazily, so a tick of
GPU systems never crosses PCIe unless a host system touches the columns.

The bond observation's pair tracker and persistence threshold
(src/analysis/pairs.rs:43-109, src/systems/bonds.rs:73-185) run on the device
(gx_bond_observe); :class:`GpuBondObservation` only reads their summary.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import elements as E
from ._lib import Handle
from .chemistry import BondStructureLens


# ---------------------------------------------------------------- scheduler


@dataclass
class Access:
    """Declared reads/writes (src/scheduler/system.rs:16-69)."""

    reads: list = field(default_factory=list)
    writes: list = field(default_factory=list)
    resources_read: list = field(default_factory=list)
    resources_write: list = field(default_factory=list)

    def conflicts_with(self, o: "Access") -> bool:  # system.rs:47-69
        comp = any(c in o.reads or c in o.writes for c in self.writes) or \
            any(c in self.reads or c in self.writes for c in o.writes)
        res = any(c in o.resources_read or c in o.resources_write for c in self.resources_write) or \
            any(c in self.resources_read or c in self.resources_write for c in o.resources_write)
        return comp or res


@dataclass
class Time:
    dt: float
    t: float = 0.0
    tick: int = 0

    def advance(self):  # src/universe/time.rs:25-28
        self.t += self.dt
        self.tick += 1


@dataclass
class World:
    """ECS columns in slot order (Position, Velocity, Acceleration, AtomType,
    Mass, Charge, EntityId::index, Bonds)."""

    pos: np.ndarray
    vel: np.ndarray
    acc: np.ndarray
    elem: np.ndarray
    mass: np.ndarray
    charge: np.ndarray
    entity: np.ndarray
    bonds: dict = field(default_factory=dict)  # entity -> list of bonded entities

    @classmethod
    def from_universe(cls, u) -> "World":
        return cls(pos=u.pos.copy(), vel=u.vel.copy(), acc=np.zeros_like(u.pos), elem=u.elem.copy(),
                   mass=u.mass.copy(), charge=u.charge.copy(), entity=u.entity.copy())

    def __len__(self):
        return len(self.elem)


class StatsCollector:
    """StatsCollector (src/stats/mod.rs:151-212): the latest snapshot, a
    bounded history, and the scheduler's execution count and the main loop's
    FPS that StatsSystem copies into each snapshot."""

    def __init__(self, history_cap: int = 1024):
        self.snapshot: dict = {}
        self.systems_run = 0
        self.fps = 0.0
        self.history: list[dict] = []
        self.history_cap = max(int(history_cap), 1)

    def record(self, snap: dict) -> None:
        if len(self.history) == self.history_cap:
            self.history.pop(0)
        self.snapshot = snap
        self.history.append(snap)


@dataclass
class SystemContext:
    world: World
    resources: dict
    time: Time
    dt: float
    stats: StatsCollector = field(default_factory=StatsCollector)


class System:
    def name(self) -> str:
        raise NotImplementedError

    def access(self) -> Access:
        return Access()

    def run(self, ctx: SystemContext) -> None:
        raise NotImplementedError


class Scheduler:
    """Sequential run in registration order (src/scheduler/mod.rs:59-89)."""

    def __init__(self):
        self.systems: list[System] = []
        self.executions = 0

    def add_system(self, s: System):
        self.systems.append(s)

    def run(self, ctx: SystemContext):
        for s in self.systems:
            s.run(ctx)
            self.executions += 1
        ctx.stats.systems_run = self.executions  # mod.rs:88: after the whole schedule

    def names(self) -> list[str]:
        return [s.name() for s in self.systems]


# ---------------------------------------------------------------- device world


class GpuWorld:
    """One device handle shared by every GPU system, with lazy column sync.

    ``host_dirty``: a host system wrote the columns, upload before the next
    GPU system.  ``device_dirty``: the device copy is newer, download before a
    host system reads.
    """

    def __init__(self, cfg, world: World, precision: str = "mixed", device: int = 0):
        self.h = Handle(cfg, precision, device)
        self.world = world
        self.h.set_state(world.pos, world.vel, world.elem, acc=world.acc, charge=world.charge, mass=world.mass,
                         entity=world.entity)
        self.host_dirty = False
        self.device_dirty = False
        self.bonds_on_device = False  # the device bond list came from gx_bond_observe
        self.slot_of_entity = {int(e): i for i, e in enumerate(world.entity)}

    def to_device(self):
        if self.host_dirty:
            self.h.set_dynamic(self.world.pos, self.world.vel, self.world.acc)
            self.host_dirty = False

    def to_host(self):
        if self.device_dirty:
            self.world.pos, self.world.vel, self.world.acc = self.h.get_state()
            self.device_dirty = False

    def set_bonds_from_world(self):
        """Bonds component -> slot pairs, once per bond (systems/forces.rs:208-226):
        from entity e's list, only neighbours with a larger index are taken."""
        pairs = []
        for e, lst in self.world.bonds.items():
            si = self.slot_of_entity.get(int(e))
            if si is None:
                continue
            for nb in lst:
                if int(e) >= int(nb):
                    continue
                sj = self.slot_of_entity.get(int(nb))
                if sj is not None:
                    pairs.append((si, sj))
        self.h.set_bonds(np.asarray(pairs, dtype=np.uint32).reshape(-1, 2))


class _GpuSystem(System):
    def __init__(self, gpu: GpuWorld):
        self.gpu = gpu

    def _enter(self):
        self.gpu.to_device()

    def _leave(self):
        self.gpu.device_dirty = True


class GpuVelocityHalfKick(_GpuSystem):
    """VelocityHalfKick (src/systems/integrate.rs:25-45)."""

    def name(self):
        return "velocity_half_kick"

    def access(self):
        return Access(reads=["Acceleration"], writes=["Velocity"])

    def run(self, ctx):
        self._enter()
        self.gpu.h.half_kick()
        self._leave()


class GpuPositionDrift(_GpuSystem):
    """PositionDrift (src/systems/integrate.rs:48-68)."""

    def name(self):
        return "position_drift"

    def access(self):
        return Access(reads=["Velocity"], writes=["Position"])

    def run(self, ctx):
        self._enter()
        self.gpu.h.drift()
        self._leave()


class GpuBoundary(_GpuSystem):
    """BoundarySystem (src/systems/boundary.rs:22-35)."""

    def name(self):
        return "boundary"

    def access(self):
        return Access(writes=["Position"], resources_read=["Config"])

    def run(self, ctx):
        self._enter()
        self.gpu.h.wrap()
        self._leave()


class GpuForceSystem(_GpuSystem):
    """ForceSystem (src/systems/forces.rs:145-353)."""

    def __init__(self, gpu: GpuWorld, bonds_on: bool):
        super().__init__(gpu)
        self.bonds_on = bonds_on

    def name(self):
        return "forces"

    def access(self):
        return Access(reads=["Position", "Mass", "AtomType", "Charge", "Bonds"], writes=["Acceleration"],
                      resources_read=["Config"], resources_write=["PotentialEnergy", "BondEnergy"])

    def run(self, ctx):
        self._enter()
        if self.bonds_on and not self.gpu.bonds_on_device:
            self.gpu.set_bonds_from_world()
        V, Vb, _ = self.gpu.h.forces()
        ctx.resources["PotentialEnergy"] = V
        ctx.resources["BondEnergy"] = Vb
        self._leave()


class GpuThermostat(_GpuSystem):
    """ThermostatSystem (src/systems/thermostat.rs:19-71)."""

    def name(self):
        return "thermostat"

    def access(self):
        return Access(reads=["Mass"], writes=["Velocity"])

    def run(self, ctx):
        self._enter()
        self.gpu.h.thermostat()
        self._leave()


class GpuStructure(_GpuSystem):
    """StructureSystem (src/systems/structure.rs:44-84): FoF every interval ticks."""

    def __init__(self, gpu: GpuWorld, interval: int):
        super().__init__(gpu)
        self.interval = max(int(interval), 1)

    def name(self):
        return "structure"

    def access(self):
        return Access(reads=["Position", "AtomType"], resources_read=["Config"],
                      resources_write=["StructureStats"])

    def run(self, ctx):
        if ctx.time.tick % self.interval != 0:
            return
        self._enter()
        _, st = self.gpu.h.clusters(E.BOND_FACTOR)
        st["tick"] = ctx.time.tick
        ctx.resources["StructureStats"] = st


class GpuBondObservation(_GpuSystem):
    """BondObservationSystem (src/systems/bonds.rs:58-185) on the device
    (gx_bond_observe): bound pairs, episodes, persistence and the summary all
    stay on the GPU; the persistent pairs become the device bond list the next
    force pass reads, and are mirrored into the host Bonds column."""

    def __init__(self, gpu: GpuWorld, cfg):
        super().__init__(gpu)
        self.cfg = cfg

    def name(self):
        return "bond-observation"

    def access(self):
        return Access(reads=["Position", "AtomType"], writes=["Bonds"], resources_read=["Config"],
                      resources_write=["BondObservation"])

    def run(self, ctx):
        self._enter()
        st = self.gpu.h.bond_observe(self.cfg.bond_k_bind, self.cfg.bond_min_periods, ctx.time.tick,
                                     debounce=E.DEBOUNCE, apply_bonds=True)
        self.gpu.bonds_on_device = True
        ent = self.gpu.world.entity
        bonds: dict = {}
        for a, b in self.gpu.h.get_bonds():
            ea, eb = int(ent[a]), int(ent[b])
            bonds.setdefault(ea, []).append(eb)
            bonds.setdefault(eb, []).append(ea)
        ctx.world.bonds = bonds
        bo = ctx.resources.setdefault("BondObservation", {})
        bo.update(tick=st["tick"], bonded_pairs=st["bonded_pairs"], bonded_entities=st["bonded_entities"],
                  mean_coordination=st["mean_coordination"], bonds_formed=st["bonds_formed"],
                  lifetime_sum_ticks=st["lifetime_sum_ticks"], species_matrix=st["species_matrix"])


class GpuCollisions(_GpuSystem):
    """CollisionSystem (src/systems/collisions.rs:23-88): elastic impulses
    between the pairs within 2 * particle_radius (gx_collisions)."""

    def name(self):
        return "collisions"

    def access(self):
        return Access(reads=["Position", "Velocity", "Mass"], writes=["Velocity"], resources_read=["Config"],
                      resources_write=["CollisionCounter"])

    def run(self, ctx):
        self._enter()
        c = self.gpu.h.collisions()
        self._leave()
        ctx.resources["CollisionCounter"] = ctx.resources.get("CollisionCounter", 0) + c


class GpuBondStructure(_GpuSystem):
    """BondStructureSystem (src/systems/bond_structure.rs:25-246) every
    interval ticks: the components of the persistent-bond graph and each
    bond's raw energy from the device (gx_bond_components), the composition
    histogram and the lifecycle events on the host (genesis_b200.chemistry)."""

    def __init__(self, gpu: GpuWorld, interval: int):
        super().__init__(gpu)
        self.interval = max(int(interval), 1)
        self.lens = BondStructureLens()

    def name(self):
        return "bond-structure"

    def access(self):
        return Access(reads=["Bonds", "AtomType", "Position"], resources_read=["Config"],
                      resources_write=["ChemicalStructure"])

    def run(self, ctx):
        if ctx.time.tick % self.interval != 0:
            return
        self._enter()
        labels, energy = self.gpu.h.bond_components()
        cs = self.lens.sample(labels, self.gpu.world.elem, self.gpu.h.get_bonds(), energy, len(ctx.world))
        cs["tick"] = ctx.time.tick
        ctx.resources["ChemicalStructure"] = cs


class GpuStats(_GpuSystem):
    """StatsSystem (src/systems/aggregate.rs:36-144): K and the speed sum
    from the device, the resources the other systems wrote, one
    StatsSnapshot (src/stats/mod.rs:27-91) recorded per tick.  memory_bytes
    counts the host column mirror's arrays (the reference counts its ECS
    storage, World::memory_bytes)."""

    def __init__(self, gpu: GpuWorld, cfg):
        super().__init__(gpu)
        self.cfg = cfg

    def name(self):
        return "stats"

    def access(self):
        return Access(reads=["Velocity", "Mass"],
                      resources_read=["Config", "CollisionCounter", "PotentialEnergy", "StructureStats",
                                      "BondObservation", "BondEnergy", "ChemicalStructure"])

    def run(self, ctx):
        self._enter()
        K, speed = self.gpu.h.stats()
        n = len(ctx.world)
        r = ctx.resources
        V = r.get("PotentialEnergy", 0.0)
        Vb = r.get("BondEnergy", 0.0)
        st = r.get("StructureStats")
        st = st if st and st.get("tick", 0) > 0 else None
        bo = r.get("BondObservation") or {}
        formed = int(bo.get("bonds_formed", 0))
        ch = r.get("ChemicalStructure")
        ch = ch if ch and ch.get("tick", 0) > 0 else None
        e_avg = K / n if n else 0.0
        k = self.cfg.thermal_constant
        vol = float(np.prod(self.cfg.size))
        w = ctx.world
        mem = sum(a.nbytes for a in (w.pos, w.vel, w.acc, w.elem, w.mass, w.charge, w.entity))
        snap = {"tick": ctx.time.tick, "time": ctx.time.t, "entities": n, "energy_total": K + V + Vb,
                "energy_avg": e_avg, "energy_potential": V, "temperature_avg": (2.0 / 3.0) * e_avg / k if k > 0 else 0.0,
                "mean_speed": speed / n if n else 0.0, "density": n / vol if vol > 0 else 0.0,
                "collisions": int(r.get("CollisionCounter", 0)), "systems_run": ctx.stats.systems_run,
                "fps": ctx.stats.fps, "memory_bytes": mem,
                "structure": st, "bonded_pairs": int(bo.get("bonded_pairs", 0)), "bonds_formed": formed,
                "bond_lifetime_ticks": bo.get("lifetime_sum_ticks", 0.0) / formed if formed > 0 else 0.0,
                "bond_energy": Vb, "bond_matrix": [float(c) for c in np.ravel(bo.get("species_matrix", []))],
                "chemical": ch, "kinetic": K}
        ctx.resources["StatsSnapshot"] = snap
        ctx.stats.record(snap)


def build_schedule(cfg, gpu: GpuWorld) -> Scheduler:
    """The force schedule of build_schedule (src/universe/mod.rs:355-392)."""
    s = Scheduler()
    s.add_system(GpuVelocityHalfKick(gpu))
    s.add_system(GpuPositionDrift(gpu))
    if cfg.enable_boundaries:
        s.add_system(GpuBoundary(gpu))
    s.add_system(GpuForceSystem(gpu, cfg.enable_bond_interaction))
    if cfg.enable_collisions:
        s.add_system(GpuCollisions(gpu))
    s.add_system(GpuVelocityHalfKick(gpu))
    if cfg.enable_thermostat:
        s.add_system(GpuThermostat(gpu))
    if cfg.enable_bond_observation:
        s.add_system(GpuBondObservation(gpu, cfg))
        s.add_system(GpuBondStructure(gpu, cfg.structure_interval))
    s.add_system(GpuStructure(gpu, cfg.structure_interval))
    s.add_system(GpuStats(gpu, cfg))
    return s


class GpuUniverse:
    """Universe::tick over the GPU schedule (src/universe/mod.rs:141-159)."""

    def __init__(self, cfg, u, precision: str = "mixed", device: int = 0):
        self.cfg = cfg
        self.world = World.from_universe(u)
        self.gpu = GpuWorld(cfg, self.world, precision, device)
        self.time = Time(cfg.dt)
        self.resources: dict = {"Config": cfg}
        self.scheduler = build_schedule(cfg, self.gpu)
        self.stats = StatsCollector()

    def tick(self):
        self.time.advance()
        t0 = time.perf_counter()
        ctx = SystemContext(self.world, self.resources, self.time, self.time.dt, self.stats)
        self.scheduler.run(ctx)
        elapsed = time.perf_counter() - t0
        self.stats.fps = 1.0 / elapsed if elapsed > 0 else 0.0  # universe/mod.rs:156-157

    def append_csv(self, path) -> None:
        """One metrics row of the latest snapshot (export::append_csv)."""
        from . import export
        export.append_csv(path, self.stats.snapshot)

    def write_frame(self, prefix) -> str:
        """The current positions as an XYZ frame (export::write_frame),
        formatted on the device."""
        from . import export
        self.gpu.to_device()
        return export.write_frame(prefix, self.time.tick, self.gpu.h)

    def run_ticks(self, n: int):
        for _ in range(n):
            self.tick()

    def sync(self) -> World:
        self.gpu.to_host()
        return self.world
