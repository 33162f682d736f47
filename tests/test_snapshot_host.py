"""The snapshot world encoding restated on the CPU (oracle/snapshot.py):
record sizes, field order and a round trip through the decoder."""
from __future__ import annotations

import struct

import numpy as np

from oracle import snapshot as S


def _state(n=5, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.random(n) + 1.0,
            rng.normal(size=n), rng.integers(0, 10, size=n).astype(np.uint8))


def test_record_is_115_bytes_plus_8_per_bond():
    pos, vel, acc, mass, charge, elem = _state()
    bonds = np.array([[0, 3], [1, 3], [3, 4]], dtype=np.uint32)
    data = S.encode_world(pos, vel, acc, mass, charge, elem, bonds=bonds)
    # Vec length + 5 records + 2 partner ids per bond
    assert len(data) == 8 + 5 * S.RECORD_FIXED + 16 * len(bonds)
    assert struct.unpack_from("<Q", data, 0)[0] == 5


def test_field_order_of_the_first_record():
    pos, vel, acc, mass, charge, elem = _state(n=1)
    data = S.encode_world(pos, vel, acc, mass, charge, elem, entity=[7], generation=[3])
    off = 8
    assert struct.unpack_from("<II", data, off) == (7, 3)  # index, generation
    off += 8
    assert data[off] == 1 and struct.unpack_from("<3d", data, off + 1) == tuple(pos[0])  # Some(Position)
    off += 25
    assert data[off] == 1 and struct.unpack_from("<3d", data, off + 1) == tuple(vel[0])
    off += 25
    assert data[off] == 1 and struct.unpack_from("<d", data, off + 1)[0] == mass[0]
    off += 9
    assert data[off] == 1 and struct.unpack_from("<d", data, off + 1)[0] == charge[0]
    off += 9
    assert data[off] == 1 and struct.unpack_from("<I", data, off + 1)[0] == elem[0]  # variant index
    off += 5
    assert data[off] == 1 and struct.unpack_from("<Q", data, off + 1)[0] == 0  # Some(Bonds { neighbors: [] })
    off += 9
    assert data[off] == 1 and struct.unpack_from("<3d", data, off + 1) == tuple(acc[0])
    assert off + 25 == len(data)


def test_round_trip_with_bonds_in_slot_order():
    pos, vel, acc, mass, charge, elem = _state(n=6, seed=3)
    ent = np.array([10, 11, 12, 13, 14, 15], dtype=np.uint32)
    gen = np.array([0, 1, 0, 2, 0, 0], dtype=np.uint32)
    bonds = np.array([[2, 5], [0, 2], [2, 3]], dtype=np.uint32)
    recs = S.decode_world(S.encode_world(pos, vel, acc, mass, charge, elem, ent, gen, bonds))
    assert [r["index"] for r in recs] == list(ent)
    assert recs[2]["bonds"] == [(10, 0), (13, 2), (15, 0)]  # partners 0, 3, 5 ascending
    assert recs[5]["bonds"] == [(12, 0)]
    assert recs[1]["bonds"] == []
    for s, r in enumerate(recs):
        assert r["position"] == tuple(pos[s]) and r["acceleration"] == tuple(acc[s])
        assert r["atom_type"] == (int(elem[s]),)
