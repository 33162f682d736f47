"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker the parity tests, smoke() and the
bench's cpu_baseline / reference arm use.  The product (genesis_b200/) never
imports this module.  See oracle.h for what the oracle restates and how its
parity is pinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_D = C.c_double
_D10 = C.c_double * 10


class OrcParams(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("dt", _D), ("thermal_constant", _D),
        ("sigma", _D10), ("epsilon_k", _D10), ("charge", _D10),
        ("lj_cutoff_factor", _D), ("coulomb_constant", _D), ("coulomb_cutoff", _D),
        ("gravity_constant", _D), ("gravity_cutoff", _D), ("bond_k_bind", _D),
        ("thermostat_temperature", _D), ("thermostat_tau", _D),
        ("enable_electrostatics", C.c_int32), ("enable_gravity", C.c_int32),
        ("enable_bond_interaction", C.c_int32), ("enable_thermostat", C.c_int32),
        ("enable_boundaries", C.c_int32), ("enable_collisions", C.c_int32), ("reserved", C.c_int32 * 2),
        ("particle_radius", C.c_double),
    ]


def build(force: bool = False) -> Path:
    src = [HERE / n for n in ("oracle.cpp", "oracle_dual.cpp", "oracle_bonds.cpp", "oracle_export.cpp", "oracle.h",
                               "oracle_grid.h", "Makefile")]
    if force or not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in src):
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboracle.so"], check=True)
    return LIB


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        dp, u8p, u32p, u64p, sz = C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.POINTER(C.c_uint32), \
            C.POINTER(C.c_uint64), C.c_size_t
        pp = C.POINTER(OrcParams)
        proto = {
            "orc_lj_table": (None, [pp, dp, dp, dp, dp]),
            "orc_lj_raw": (None, [_D, _D, _D, dp, dp]),
            "orc_smooth_cutoff": (None, [_D, _D, _D, dp, dp]),
            "orc_switched": (None, [_D, _D, _D, _D, dp, dp]),
            "orc_force_switched_scalar": (None, [_D, _D, _D, _D, _D, dp, dp]),
            "orc_coulomb_raw": (None, [_D, _D, _D, _D, dp, dp]),
            "orc_gravity_raw": (None, [_D, _D, _D, _D, dp, dp]),
            "orc_bond_harmonic_raw": (None, [_D, _D, _D, dp, dp]),
            "orc_well_curvature": (_D, [_D, _D]),
            "orc_vib_period": (_D, [_D, _D, _D]),
            "orc_equilibrium_distance": (_D, [_D]),
            "orc_grid_dims": (None, [dp, _D, u32p]),
            "orc_cell_of": (None, [sz, dp, dp, _D, u32p]),
            "orc_neighbors": (sz, [sz, dp, dp, _D, _D, u32p, dp, sz]),
            "orc_min_image": (None, [dp, dp, dp]),
            "orc_forces": (sz, [pp, sz, dp, u8p, dp, dp, sz, u32p, dp, dp, dp, C.c_int]),
            "orc_half_kick": (None, [sz, dp, dp, _D]),
            "orc_drift": (None, [sz, dp, dp, _D]),
            "orc_wrap": (None, [sz, dp, dp]),
            "orc_thermostat": (C.c_int, [sz, dp, dp, _D, _D, _D, dp, dp]),
            "orc_stats": (None, [sz, dp, dp, dp, dp]),
            "orc_ticks": (C.c_int, [pp, sz, dp, dp, dp, u8p, dp, dp, sz, u32p, C.c_int, C.c_int, dp]),
            "orc_collisions": (sz, [pp, sz, dp, dp, dp]),
            "orc_xyz_frame": (sz, [sz, C.c_uint64, dp, C.POINTER(C.c_uint8), C.c_char_p, sz]),
            "orc_radial_distribution": (C.c_int, [sz, dp, dp, _D, sz, u64p, dp, dp, dp]),
            "orc_radial_distribution_between": (C.c_int, [sz, dp, u8p, C.c_uint8, C.c_uint8, dp, _D, sz, u64p, dp,
                                                          dp, dp]),
            "orc_clusters": (C.c_int, [sz, dp, u8p, dp, _D, dp, u32p, u64p, dp]),
            "orc_bound_pairs": (sz, [sz, dp, u8p, u32p, dp, _D, dp, u32p, sz]),
            "orc_adjoint_forward": (C.c_int, [pp, sz, dp, dp, dp, u8p, dp, dp, C.c_int, C.c_int, C.c_int, _D, _D,
                                              _D, C.c_int, dp, dp, dp, dp]),
            "orc_adjoint_trajectory": (C.c_int, [pp, sz, dp, dp, dp, u8p, dp, dp, C.c_int, C.c_int, dp]),
            "orc_tracker_new": (C.c_void_p, [C.c_int]),
            "orc_tracker_free": (None, [C.c_void_p]),
            "orc_tracker_close_all": (None, [C.c_void_p]),
            "orc_bond_threshold": (C.c_uint64, [pp, _D, C.c_int, C.c_int]),
            "orc_bond_observe": (C.c_int, [C.c_void_p, pp, _D, sz, u32p, u8p, C.c_uint64, dp, u64p, u32p, sz,
                                           C.POINTER(sz)]),
        }
        for name, (res, args) in proto.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def params(cfg) -> OrcParams:
    p = OrcParams()
    p.box[:] = list(cfg.size)
    p.dt = cfg.dt
    p.thermal_constant = cfg.thermal_constant
    p.sigma[:] = list(cfg.sigma)
    p.epsilon_k[:] = list(cfg.epsilon_k)
    p.charge[:] = list(cfg.charge)
    p.lj_cutoff_factor = 2.5
    p.coulomb_constant = cfg.coulomb_constant
    p.coulomb_cutoff = cfg.coulomb_cutoff
    p.gravity_constant = cfg.gravity_constant
    p.gravity_cutoff = cfg.gravity_cutoff
    p.bond_k_bind = cfg.bond_k_bind
    p.thermostat_temperature = cfg.thermostat_temperature
    p.thermostat_tau = cfg.thermostat_tau
    p.enable_electrostatics = int(cfg.enable_electrostatics)
    p.enable_gravity = int(cfg.enable_gravity)
    p.enable_bond_interaction = int(cfg.enable_bond_interaction)
    p.enable_thermostat = int(cfg.enable_thermostat)
    p.enable_boundaries = int(cfg.enable_boundaries)
    p.enable_collisions = int(cfg.enable_collisions)
    p.particle_radius = float(cfg.particle_radius)
    return p


def _out2():
    return C.c_double(), C.c_double()


def lj_table(cfg):
    lib = load()
    ps, pe = np.empty(100), np.empty(100)
    rc, ron = _out2()
    lib.orc_lj_table(C.byref(params(cfg)), _p(ps, C.c_double), _p(pe, C.c_double), C.byref(rc), C.byref(ron))
    return ps.reshape(10, 10), pe.reshape(10, 10), rc.value, ron.value


def _pair(fn, *args):
    a, b = _out2()
    fn(*args, C.byref(a), C.byref(b))
    return a.value, b.value


def lj_raw(sigma, eps, r):
    return _pair(load().orc_lj_raw, sigma, eps, r)


def smooth_cutoff(r, r_on, rc):
    return _pair(load().orc_smooth_cutoff, r, r_on, rc)


def switched(f, v, sw, dsw):
    return _pair(load().orc_switched, f, v, sw, dsw)


def force_switched_scalar(sigma, eps, r, r_on, rc):
    return _pair(load().orc_force_switched_scalar, sigma, eps, r, r_on, rc)


def coulomb_raw(k_e, qa, qb, r):
    return _pair(load().orc_coulomb_raw, k_e, qa, qb, r)


def gravity_raw(g, ma, mb, r):
    return _pair(load().orc_gravity_raw, g, ma, mb, r)


def bond_harmonic_raw(k, r_eq, r):
    return _pair(load().orc_bond_harmonic_raw, k, r_eq, r)


def well_curvature(eps, sigma):
    return load().orc_well_curvature(eps, sigma)


def vib_period(eps, sigma, mu):
    return load().orc_vib_period(eps, sigma, mu)


def equilibrium_distance(sigma):
    return load().orc_equilibrium_distance(sigma)


def grid_dims(box, min_cell):
    out = np.zeros(3, dtype=np.uint32)
    load().orc_grid_dims(_p(_f64(box), C.c_double), min_cell, _p(out, C.c_uint32))
    return tuple(int(x) for x in out)


def cell_of(pos, box, min_cell):
    pos = _f64(pos)
    out = np.empty(len(pos), dtype=np.uint32)
    load().orc_cell_of(len(pos), _p(pos, C.c_double), _p(_f64(box), C.c_double), min_cell, _p(out, C.c_uint32))
    return out


def neighbors(pos, box, min_cell, cutoff, with_normals=False):
    lib = load()
    pos = _f64(pos)
    b = _f64(box)
    total = lib.orc_neighbors(len(pos), _p(pos, C.c_double), _p(b, C.c_double), min_cell, cutoff, None, None, 0)
    pairs = np.empty((total, 2), dtype=np.uint32)
    normals = np.empty((total, 3)) if with_normals else None
    lib.orc_neighbors(len(pos), _p(pos, C.c_double), _p(b, C.c_double), min_cell, cutoff, _p(pairs, C.c_uint32),
                      _p(normals, C.c_double), total)
    return (pairs, normals) if with_normals else pairs


def min_image(d, box):
    out = np.empty(3)
    load().orc_min_image(_p(_f64(d), C.c_double), _p(_f64(box), C.c_double), _p(out, C.c_double))
    return out


def forces(cfg, pos, elem, charge, mass, bonds=None, nthreads=1):
    lib = load()
    pos, charge, mass = _f64(pos), _f64(charge), _f64(mass)
    elem = np.ascontiguousarray(elem, dtype=np.uint8)
    bonds = np.zeros((0, 2), dtype=np.uint32) if bonds is None else np.ascontiguousarray(bonds, dtype=np.uint32)
    acc = np.empty((len(elem), 3))
    V, Vb = _out2()
    npairs = lib.orc_forces(C.byref(params(cfg)), len(elem), _p(pos, C.c_double), _p(elem, C.c_uint8),
                            _p(charge, C.c_double), _p(mass, C.c_double), len(bonds), _p(bonds, C.c_uint32),
                            _p(acc, C.c_double), C.byref(V), C.byref(Vb), nthreads)
    return acc, V.value, Vb.value, int(npairs)


def half_kick(vel, acc, dt):
    vel = _f64(vel).copy()
    load().orc_half_kick(len(vel), _p(vel, C.c_double), _p(_f64(acc), C.c_double), dt)
    return vel


def drift(pos, vel, dt):
    pos = _f64(pos).copy()
    load().orc_drift(len(pos), _p(pos, C.c_double), _p(_f64(vel), C.c_double), dt)
    return pos


def wrap(pos, box):
    pos = _f64(pos).copy()
    load().orc_wrap(len(pos), _p(pos, C.c_double), _p(_f64(box), C.c_double))
    return pos


def thermostat(vel, mass, k, target, tau):
    vel = _f64(vel).copy()
    K, lam = _out2()
    applied = load().orc_thermostat(len(vel), _p(vel, C.c_double), _p(_f64(mass), C.c_double), k, target, tau,
                                    C.byref(K), C.byref(lam))
    return vel, K.value, lam.value, bool(applied)


def stats(vel, mass):
    K, sp = _out2()
    vel = _f64(vel)
    load().orc_stats(len(vel), _p(vel, C.c_double), _p(_f64(mass), C.c_double), C.byref(K), C.byref(sp))
    return K.value, sp.value


TICK_FIELDS = ("kinetic", "potential", "bond_energy", "lambda", "pairs")


def collisions(cfg, pos, vel, mass):
    """One CollisionSystem pass: (velocities after, collisions counted)."""
    lib = load()
    pos = _f64(pos)
    vel = _f64(vel).copy()
    c = lib.orc_collisions(C.byref(params(cfg)), len(pos), _p(pos, C.c_double), _p(vel, C.c_double),
                           _p(_f64(mass), C.c_double))
    return vel, int(c)


def xyz_frame(tick, pos, elem) -> bytes:
    """export::write_frame's text (src/export/mod.rs:152-172) through the C
    library's printf (oracle_export.cpp)."""
    lib = load()
    pos = _f64(pos)
    elem = np.ascontiguousarray(elem, dtype=np.uint8)
    n = len(elem)
    ep = elem.ctypes.data_as(C.POINTER(C.c_uint8))
    size = lib.orc_xyz_frame(n, int(tick), _p(pos, C.c_double), ep, None, 0)
    buf = C.create_string_buffer(size)
    lib.orc_xyz_frame(n, int(tick), _p(pos, C.c_double), ep, buf, size)
    return buf.raw[:size]


def xyz_frame_py(tick, pos, elem) -> bytes:
    """The same text from Python's own fixed-point formatting (exact value,
    ties to even), pure-Python loops for small cases: pins the C path."""
    symbols = ("H", "He", "C", "N", "O", "Na", "Si", "P", "S", "Fe")

    def f6(x):
        x = float(x)
        if x != x:
            return "NaN"
        if x in (float("inf"), float("-inf")):
            return "inf" if x > 0 else "-inf"
        return f"{x:.6f}"

    lines = [f"{len(elem)}", f"frame {int(tick)}"]
    lines += [f"{symbols[int(e)]} {f6(p[0])} {f6(p[1])} {f6(p[2])}" for p, e in zip(pos, elem)]
    return ("\n".join(lines) + "\n").encode()


def ticks(cfg, pos, vel, acc, elem, charge, mass, nticks, bonds=None, nthreads=1):
    """Runs nticks of the force schedule; returns (pos, vel, acc, stats[nticks, 5])."""
    lib = load()
    pos, vel = _f64(pos).copy(), _f64(vel).copy()
    acc = np.zeros_like(pos) if acc is None else _f64(acc).copy()
    elem = np.ascontiguousarray(elem, dtype=np.uint8)
    bonds = np.zeros((0, 2), dtype=np.uint32) if bonds is None else np.ascontiguousarray(bonds, dtype=np.uint32)
    st = np.zeros((nticks, 5))
    lib.orc_ticks(C.byref(params(cfg)), len(elem), _p(pos, C.c_double), _p(vel, C.c_double), _p(acc, C.c_double),
                  _p(elem, C.c_uint8), _p(_f64(charge), C.c_double), _p(_f64(mass), C.c_double), len(bonds),
                  _p(bonds, C.c_uint32), nticks, nthreads, _p(st, C.c_double))
    return pos, vel, acc, st


def radial_distribution(pos, box, r_max, nbins, elem=None, between=None):
    lib = load()
    pos = _f64(pos)
    nb = min(max(nbins, 1), 1 << 16)
    counts = np.zeros(nb, dtype=np.uint64)
    bins = np.zeros(nb)
    rmo, dro = _out2()
    if between is None:
        rc = lib.orc_radial_distribution(len(pos), _p(pos, C.c_double), _p(_f64(box), C.c_double), r_max, nbins,
                                         _p(counts, C.c_uint64), _p(bins, C.c_double), C.byref(rmo), C.byref(dro))
    else:
        e = np.ascontiguousarray(elem, dtype=np.uint8)
        rc = lib.orc_radial_distribution_between(len(pos), _p(pos, C.c_double), _p(e, C.c_uint8), between[0],
                                                 between[1], _p(_f64(box), C.c_double), r_max, nbins,
                                                 _p(counts, C.c_uint64), _p(bins, C.c_double), C.byref(rmo),
                                                 C.byref(dro))
    return counts, bins, rmo.value, dro.value, rc


def clusters(pos, elem, box, bond_factor, sigma):
    pos = _f64(pos)
    e = np.ascontiguousarray(elem, dtype=np.uint8)
    labels = np.empty(len(pos), dtype=np.uint32)
    st = np.zeros(4, dtype=np.uint64)
    mean = C.c_double()
    load().orc_clusters(len(pos), _p(pos, C.c_double), _p(e, C.c_uint8), _p(_f64(box), C.c_double), bond_factor,
                        _p(_f64(sigma), C.c_double), _p(labels, C.c_uint32), _p(st, C.c_uint64), C.byref(mean))
    return labels, {"monomers": int(st[0]), "aggregates": int(st[1]), "largest": int(st[2]),
                    "bound_pairs": int(st[3]), "mean_size": mean.value}


def bound_pairs(pos, elem, entity, box, k_bind, sigma):
    lib = load()
    pos = _f64(pos)
    e = np.ascontiguousarray(elem, dtype=np.uint8)
    ent = None if entity is None else np.ascontiguousarray(entity, dtype=np.uint32)
    args = (len(pos), _p(pos, C.c_double), _p(e, C.c_uint8), _p(ent, C.c_uint32), _p(_f64(box), C.c_double), k_bind,
            _p(_f64(sigma), C.c_double))
    total = lib.orc_bound_pairs(*args, None, 0)
    out = np.empty((total, 2), dtype=np.uint32)
    lib.orc_bound_pairs(*args, _p(out, C.c_uint32), total)
    return out


def adjoint_forward(cfg, pos, vel, acc, elem, charge, mass, nsteps, gr_bins=0, gr_every=1, gr_rmax=1.0,
                    gr_width=0.1, gr_support=6.0, nthreads=1, dual=False):
    """Potential per tick and time-averaged Gaussian-kernel g(r) of an NVE
    run (oracle_dual.cpp).  With ``dual`` also their exact derivatives with
    respect to (sigma[0..9], epsilon_k[0..9]): returns
    (V[nsteps], g[gr_bins], dV[nsteps, 20], dg[gr_bins, 20])."""
    lib = load()
    elem = np.ascontiguousarray(elem, dtype=np.uint8)
    n = len(elem)
    V = np.zeros(nsteps)
    g = np.zeros(max(gr_bins, 0))
    dV = np.zeros((nsteps, 20)) if dual else None
    dg = np.zeros((max(gr_bins, 0), 20)) if dual else None
    if dual and gr_bins <= 0:
        dg = None
    rc = lib.orc_adjoint_forward(C.byref(params(cfg)), n, _p(_f64(pos), C.c_double), _p(_f64(vel), C.c_double),
                                 _p(_f64(acc), C.c_double), _p(elem, C.c_uint8), _p(_f64(charge), C.c_double),
                                 _p(_f64(mass), C.c_double), nsteps, gr_bins, gr_every, gr_rmax, gr_width,
                                 gr_support, nthreads, _p(V, C.c_double), _p(g, C.c_double) if gr_bins > 0 else None,
                                 _p(dV, C.c_double), _p(dg, C.c_double))
    if rc != 0:
        raise ValueError(f"orc_adjoint_forward failed ({rc})")
    if dual and dg is None:
        dg = np.zeros((0, 20))
    return V, g, dV, dg


def adjoint_trajectory(cfg, pos, vel, acc, elem, charge, mass, nsteps, nthreads=1):
    """The dual template's T = double trajectory: (pos, vel, acc, V[nsteps])."""
    lib = load()
    pos, vel, acc = _f64(pos).copy(), _f64(vel).copy(), _f64(acc).copy()
    elem = np.ascontiguousarray(elem, dtype=np.uint8)
    V = np.zeros(nsteps)
    rc = lib.orc_adjoint_trajectory(C.byref(params(cfg)), len(elem), _p(pos, C.c_double), _p(vel, C.c_double),
                                    _p(acc, C.c_double), _p(elem, C.c_uint8), _p(_f64(charge), C.c_double),
                                    _p(_f64(mass), C.c_double), nsteps, nthreads, _p(V, C.c_double))
    if rc != 0:
        raise ValueError(f"orc_adjoint_trajectory failed ({rc})")
    return pos, vel, acc, V


BOND_STATS = ("bonded_pairs", "bonded_entities", "mean_coordination", "bonds_formed", "lifetime_sum_ticks",
              "open_episodes", "completed_episodes", "completed_ticks")


class BondTracker:
    """PairTracker + BondObservationSystem (oracle_bonds.cpp), pairs by slot."""

    def __init__(self, cfg, debounce: int = 2, min_periods: float | None = None):
        self.lib = load()
        self.p = params(cfg)
        self.min_periods = cfg.bond_min_periods if min_periods is None else min_periods
        self.t = self.lib.orc_tracker_new(debounce)

    def threshold(self, ea: int, eb: int) -> int:
        return int(self.lib.orc_bond_threshold(C.byref(self.p), self.min_periods, ea, eb))

    def observe(self, bound, elem_of_slot, tick: int):
        """bound: (k, 2) slot pairs of this tick.  Returns (stats dict with a
        10x10 'species_matrix', persistent pairs (m, 2) ascending)."""
        bound = np.ascontiguousarray(np.asarray(bound, dtype=np.uint32).reshape(-1, 2))
        elem = np.ascontiguousarray(elem_of_slot, dtype=np.uint8)
        st = np.zeros(8)
        mat = np.zeros(100, dtype=np.uint64)
        cap = max(len(bound), 1)
        out = np.zeros((cap, 2), dtype=np.uint32)
        n = C.c_size_t()
        rc = self.lib.orc_bond_observe(self.t, C.byref(self.p), self.min_periods, len(bound), _p(bound, C.c_uint32),
                                       _p(elem, C.c_uint8), tick, _p(st, C.c_double), _p(mat, C.c_uint64),
                                       _p(out, C.c_uint32), cap, C.byref(n))
        if rc != 0:
            raise ValueError("orc_bond_observe failed")
        d = dict(zip(BOND_STATS, st.tolist()))
        d["species_matrix"] = mat.reshape(10, 10)
        return d, out[: n.value].copy()

    def close_all(self):
        self.lib.orc_tracker_close_all(self.t)

    def __del__(self):
        try:
            self.lib.orc_tracker_free(self.t)
        except Exception:
            pass
