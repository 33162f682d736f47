"""CPU restatement of the world section of a snapshot file (test oracle).

Test infrastructure only: the tests compare the device encoder
(gx_snapshot_world) with this restatement; nothing in the product imports it.

Universe::save (src/serialization/mod.rs:85-104) writes
bincode::serialize(&Snapshot { format, config, state, world }); `world` is a
Vec<EntitySnapshot> (mod.rs:38-56):

    struct EntitySnapshot { index: u32, generation: u32,
        position: Option<Position>, velocity: Option<Velocity>,
        mass: Option<Mass>, charge: Option<Charge>,
        atom_type: Option<AtomType>, bonds: Option<Bonds>,
        acceleration: Option<Acceleration> }

with Position/Velocity/Acceleration newtypes of Vec3 {x, y, z: f64}
(src/components/position.rs:7-9, src/math/mod.rs:13-18), Mass(f64) and
Charge(f64) (mass.rs:6-7, charge.rs:6-7), AtomType a unit enum declared
H, He, C, N, O, Na, Si, P, S, Fe (atom_type.rs:13-25; serde encodes a unit
variant by its declaration index, not its discriminant) and
Bonds { neighbors: Vec<EntityId> } with EntityId { index: u32,
generation: u32 } (bonds.rs:9-13, src/ecs/entity.rs:16-20).  bincode 1
(Cargo.toml: bincode = "1") with its default options: little-endian
fixed-width integers and floats, u64 sequence lengths, a u8 Option tag,
u32 enum variant indices, struct fields in declaration order.
"""
from __future__ import annotations

import struct

import numpy as np

RECORD_FIXED = 115  # 4 + 4 + 25 + 25 + 9 + 9 + 5 + 9 + 25


def encode_world(pos, vel, acc, mass, charge, elem, entity=None, generation=None, bonds=None) -> bytes:
    """bincode of Vec<EntitySnapshot>; every record carries all seven
    components, as every atom the reference spawns does
    (src/universe/mod.rs:247-273).  `bonds`: (m, 2) slot pairs; each slot's
    partners are written in ascending slot order."""
    n = len(elem)
    entity = np.arange(n, dtype=np.uint32) if entity is None else np.asarray(entity, dtype=np.uint32)
    generation = np.zeros(n, dtype=np.uint32) if generation is None else np.asarray(generation, dtype=np.uint32)
    adj = [[] for _ in range(n)]
    if bonds is not None:
        for a, b in np.asarray(bonds, dtype=np.int64).reshape(-1, 2):
            adj[a].append(int(b))
            adj[b].append(int(a))
    out = [struct.pack("<Q", n)]
    for s in range(n):
        rec = [struct.pack("<II", int(entity[s]), int(generation[s])),
               b"\x01" + struct.pack("<3d", *pos[s]),
               b"\x01" + struct.pack("<3d", *vel[s]),
               b"\x01" + struct.pack("<d", float(mass[s])),
               b"\x01" + struct.pack("<d", float(charge[s])),
               b"\x01" + struct.pack("<I", int(elem[s])),
               b"\x01" + struct.pack("<Q", len(adj[s]))]
        for q in sorted(adj[s]):
            rec.append(struct.pack("<II", int(entity[q]), int(generation[q])))
        rec.append(b"\x01" + struct.pack("<3d", *acc[s]))
        out.append(b"".join(rec))
    return b"".join(out)


def decode_world(data: bytes) -> list[dict]:
    """The inverse of encode_world for records whose components are all
    present or absent (tag 0 skips the value)."""
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from(fmt, data, off)
        off += struct.calcsize(fmt)
        return v

    (n,) = take("<Q")
    out = []
    for _ in range(n):
        r = {}
        r["index"], r["generation"] = take("<II")
        for key, fmt in (("position", "<3d"), ("velocity", "<3d"), ("mass", "<d"), ("charge", "<d"),
                         ("atom_type", "<I")):
            (tag,) = take("<B")
            r[key] = take(fmt) if tag else None
        (tag,) = take("<B")
        if tag:
            (k,) = take("<Q")
            r["bonds"] = [take("<II") for _ in range(k)]
        else:
            r["bonds"] = None
        (tag,) = take("<B")
        r["acceleration"] = take("<3d") if tag else None
        out.append(r)
    if off != len(data):
        raise ValueError(f"{len(data) - off} trailing bytes")
    return out
