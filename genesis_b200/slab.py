"""One universe over several ranks: a z-slab decomposition with a per-tick
halo exchange.

The reference advances one universe on one process (ForceSystem::run,
src/systems/forces.rs:163-353, over the whole World).  Spread over R ranks,
the box is cut into R slabs along z of width W = L_z / R; rank r owns the
atoms whose wrapped z lies in [-L/2 + r W, -L/2 + (r + 1) W).  One tick, in
the reference's order (src/universe/mod.rs:356-369):

  1. kick (v += a dt/2), drift, wrap on the owned atoms;
  2. migrate: atoms that left the slab go to the rank that owns them now
     (a neighbour: an atom moves far less than W in a tick);
  3. halo: every rank sends the neighbouring ranks its owned atoms within
     r_c of the boundary they share;
  4. forces on the owned atoms from owned + halo atoms (every neighbour of an
     owned atom within r_c is present; a pair across a boundary is evaluated
     on both ranks, each keeping its own atom's force, so no force travels
     back);
  5. kick; 6. Berendsen: the kinetic energy is one all-reduce of the owned
     sums, so every rank computes the same scale (thermostat.rs:47-71).

Communication uses torch.distributed point-to-point messages (gloo on the
CPU, NCCL between GPUs): a count, then the rows.  The force engine is a
callable (positions, elements, charges, masses) -> accelerations for every
given atom; the caller keeps the rows of its owned atoms.  A slab must be at
least 2 r_c wide so that an atom is within r_c of one boundary at most.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# per-atom columns carried by a migration: x y z vx vy vz ax ay az charge mass id elem
_MIG = 13
# per-atom columns of a halo row: x y z charge mass elem
_HALO = 6


@dataclass
class Owned:
    """The owned atoms of one rank (rows in any order; `ids` are global)."""

    pos: np.ndarray
    vel: np.ndarray
    acc: np.ndarray
    elem: np.ndarray
    charge: np.ndarray
    mass: np.ndarray
    ids: np.ndarray

    @property
    def n(self) -> int:
        return len(self.ids)

    def rows(self, sel) -> np.ndarray:
        return np.column_stack([self.pos[sel], self.vel[sel], self.acc[sel], self.charge[sel], self.mass[sel],
                                self.ids[sel].astype(np.float64), self.elem[sel].astype(np.float64)])

    @staticmethod
    def from_rows(r: np.ndarray) -> "Owned":
        r = r.reshape(-1, _MIG)
        return Owned(r[:, 0:3].copy(), r[:, 3:6].copy(), r[:, 6:9].copy(), r[:, 12].astype(np.uint8),
                     r[:, 9].copy(), r[:, 10].copy(), r[:, 11].astype(np.int64))

    def concat(self, o: "Owned") -> "Owned":
        return Owned(np.vstack([self.pos, o.pos]), np.vstack([self.vel, o.vel]), np.vstack([self.acc, o.acc]),
                     np.concatenate([self.elem, o.elem]), np.concatenate([self.charge, o.charge]),
                     np.concatenate([self.mass, o.mass]), np.concatenate([self.ids, o.ids]))

    def take(self, sel) -> "Owned":
        return Owned(self.pos[sel], self.vel[sel], self.acc[sel], self.elem[sel], self.charge[sel], self.mass[sel],
                     self.ids[sel])


class Slabs:
    """z-slab geometry and the per-tick exchanges of one rank."""

    def __init__(self, box, rc: float, rank: int, world: int, dist=None, device: str = "cpu"):
        self.box = np.asarray(box, dtype=np.float64)
        self.rc = float(rc)
        self.rank, self.world = int(rank), int(world)
        self.dist = dist
        self.device = device
        self.width = self.box[2] / self.world
        if self.world > 1 and self.width < 2.0 * self.rc:
            raise ValueError(f"slab width {self.width:.3f} is below 2 r_c = {2 * self.rc:.3f}")
        self.lo = -0.5 * self.box[2] + self.rank * self.width
        self.hi = self.lo + self.width

    def owner(self, z: np.ndarray) -> np.ndarray:
        """Rank owning each wrapped z (the same floor as a grid cell index)."""
        k = np.floor((np.asarray(z) + 0.5 * self.box[2]) / self.width).astype(np.int64)
        return np.clip(k, 0, self.world - 1)

    def peers(self) -> list[int]:
        return sorted({(self.rank - 1) % self.world, (self.rank + 1) % self.world} - {self.rank})

    def _exchange(self, outgoing: dict[int, np.ndarray], cols: int) -> np.ndarray:
        """Sends outgoing[peer] (rows of `cols` floats) to every peer and
        returns what the peers sent, stacked.  Counts first, then rows;
        non-blocking sends and receives, so no ordering can deadlock."""
        import torch

        dist = self.dist
        peers = self.peers()
        if not peers:
            return np.zeros((0, cols))
        cnt_out = {p: torch.tensor([len(outgoing.get(p, ()))], dtype=torch.int64, device=self.device) for p in peers}
        cnt_in = {p: torch.zeros(1, dtype=torch.int64, device=self.device) for p in peers}
        reqs = [dist.isend(cnt_out[p], p) for p in peers] + [dist.irecv(cnt_in[p], p) for p in peers]
        for r in reqs:
            r.wait()
        data_out = {p: torch.as_tensor(np.ascontiguousarray(outgoing.get(p, np.zeros((0, cols))), dtype=np.float64)
                                       .reshape(-1, cols), device=self.device) for p in peers}
        data_in = {p: torch.zeros((int(cnt_in[p].item()), cols), dtype=torch.float64, device=self.device)
                   for p in peers}
        reqs = [dist.isend(data_out[p], p) for p in peers if len(data_out[p])]
        reqs += [dist.irecv(data_in[p], p) for p in peers if len(data_in[p])]
        for r in reqs:
            r.wait()
        got = [data_in[p].cpu().numpy() for p in peers]
        return np.vstack(got) if got else np.zeros((0, cols))

    def migrate(self, own: Owned) -> Owned:
        """Atoms whose wrapped z left the slab go to their owner."""
        if self.world == 1:
            return own
        dest = self.owner(own.pos[:, 2])
        stay = dest == self.rank
        out = {}
        for p in self.peers():
            sel = dest == p
            if sel.any():
                out[p] = own.rows(sel)
        if np.any(~stay & ~np.isin(dest, self.peers())):
            raise RuntimeError("an atom moved past a neighbouring slab in one tick")
        got = self._exchange(out, _MIG)
        return own.take(stay).concat(Owned.from_rows(got))

    def halo(self, own: Owned) -> np.ndarray:
        """Rows (x y z charge mass elem) of the peers' atoms within r_c of
        this slab's boundaries."""
        if self.world == 1:
            return np.zeros((0, _HALO))
        z = own.pos[:, 2]
        near_lo = z - self.lo < self.rc
        near_hi = self.hi - z < self.rc
        rows = np.column_stack([own.pos, own.charge, own.mass, own.elem.astype(np.float64)])
        out: dict[int, list] = {}
        for sel, p in ((near_lo, (self.rank - 1) % self.world), (near_hi, (self.rank + 1) % self.world)):
            if sel.any():
                out.setdefault(p, []).append(rows[sel])
        return self._exchange({p: np.vstack(v) for p, v in out.items()}, _HALO)

    def all_sum(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t)
        return float(t.item())


def half_kick(v, a, dt):  # integrate.rs:38-45
    return v + a * (0.5 * dt)


def tick(sl: Slabs, own: Owned, force, cfg, n_total: int) -> tuple[Owned, float, float]:
    """One tick of the decomposed universe; returns (owned, K, lambda).
    `force(pos, elem, charge, mass)` gives the accelerations of every given
    atom in the full periodic box."""
    dt = cfg.dt
    h = 0.5 * np.asarray(cfg.size, dtype=np.float64)
    own.vel = half_kick(own.vel, own.acc, dt)
    own.pos = own.pos + own.vel * dt  # integrate.rs:62-66
    if cfg.enable_boundaries:  # boundary.rs:28-34: rem_euclid(x, 2h) - h
        own.pos = np.mod(own.pos, 2.0 * h) - h
    own = sl.migrate(own)
    hal = sl.halo(own)
    pos = np.vstack([own.pos, hal[:, 0:3]])
    elem = np.concatenate([own.elem, hal[:, 5].astype(np.uint8)])
    charge = np.concatenate([own.charge, hal[:, 3]])
    mass = np.concatenate([own.mass, hal[:, 4]])
    own.acc = np.asarray(force(pos, elem, charge, mass))[: own.n]
    own.vel = half_kick(own.vel, own.acc, dt)
    v2 = own.vel[:, 0] * own.vel[:, 0] + own.vel[:, 1] * own.vel[:, 1] + own.vel[:, 2] * own.vel[:, 2]
    K = sl.all_sum(float(np.sum(0.5 * own.mass * v2)))
    lam = 1.0
    if cfg.enable_thermostat and cfg.thermostat_temperature > 0.0 and n_total:  # thermostat.rs:52-71
        t = (2.0 / 3.0) * (K / n_total) / cfg.thermal_constant
        if np.isfinite(t) and t > 0.0:
            tau = max(cfg.thermostat_tau, 1.0)
            lam = float(np.sqrt(max(1.0 + (1.0 / tau) * (cfg.thermostat_temperature / t - 1.0), 0.0)))
            own.vel = own.vel * lam
    return own, K, lam
