"""ctypes binding of the C ABI in include/genesis_gpu.h.

The shared library is loaded from this package directory.  There is no
fallback: if ``libgenesis_gpu.so`` is missing or a call fails, an exception
is raised.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import elements as E

LIB_PATH = Path(__file__).resolve().parent / "libgenesis_gpu.so"

GX_FP64, GX_MIXED = 0, 1
_PRECISION = {"fp64": GX_FP64, "mixed": GX_MIXED}

_D = C.c_double
_D10 = C.c_double * 10


class GxParams(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("dt", _D), ("thermal_constant", _D),
        ("sigma", _D10), ("epsilon_k", _D10), ("charge", _D10),
        ("lj_cutoff_factor", _D), ("coulomb_constant", _D), ("coulomb_cutoff", _D),
        ("gravity_constant", _D), ("gravity_cutoff", _D), ("bond_k_bind", _D),
        ("thermostat_temperature", _D), ("thermostat_tau", _D),
        ("enable_electrostatics", C.c_int32), ("enable_gravity", C.c_int32),
        ("enable_bond_interaction", C.c_int32), ("enable_thermostat", C.c_int32),
        ("enable_boundaries", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("enable_collisions", C.c_int32), ("reserved", C.c_int32 * 2), ("particle_radius", _D),
    ]


class GxTickStats(C.Structure):
    _fields_ = [("kinetic", _D), ("speed_sum", _D), ("potential", _D), ("bond_energy", _D),
                ("lambda_", _D), ("pairs", C.c_uint64)]


class GxAdjointSpec(C.Structure):
    _fields_ = [("nsteps", C.c_int32), ("checkpoint_every", C.c_int32), ("gr_bins", C.c_int32),
                ("gr_every", C.c_int32), ("gr_rmax", _D), ("gr_width", _D), ("gr_support", _D)]


class GxBondObservation(C.Structure):
    _fields_ = [("tick", C.c_uint64), ("bound_pairs", C.c_uint64), ("bonded_pairs", C.c_uint64),
                ("bonded_entities", C.c_uint64), ("mean_coordination", _D), ("bonds_formed", C.c_uint64),
                ("lifetime_sum_ticks", _D), ("open_episodes", C.c_uint64), ("completed_episodes", C.c_uint64),
                ("completed_ticks", C.c_uint64), ("species_matrix", C.c_uint64 * 100)]


TICK_DTYPE = np.dtype([("kinetic", "f8"), ("speed_sum", "f8"), ("potential", "f8"),
                       ("bond_energy", "f8"), ("lambda", "f8"), ("pairs", "u8")])

EXPORTS = (
    "gx_create", "gx_destroy", "gx_last_error", "gx_status_string", "gx_set_precision",
    "gx_set_state", "gx_get_state", "gx_num_atoms", "gx_set_bonds", "gx_half_kick",
    "gx_drift", "gx_wrap", "gx_forces", "gx_thermostat", "gx_stats", "gx_step",
    "gx_cell_assign", "gx_neighbors", "gx_radial_distribution",
    "gx_radial_distribution_between", "gx_clusters", "gx_bound_pairs",
    "gx_synchronize", "gx_profile_enable", "gx_profile_read", "gx_set_dynamic",
    "gx_timer_mark", "gx_timer_elapsed", "gx_launch_count", "gx_measure_fp32_peak", "gx_measure_fp64_peak",
    "gx_radial_distribution_noalloc", "gx_set_kernel_variant", "gx_autotune",
    "gx_batch_create", "gx_batch_destroy", "gx_batch_last_error", "gx_batch_set_state",
    "gx_batch_step", "gx_batch_get_state", "gx_adjoint_forward", "gx_adjoint_backward",
    "gx_set_list_skin", "gx_list_rebuilds", "gx_list_stats", "gx_batch_set_mode", "gx_batch_get_mode", "gx_batch_autotune", "gx_batch_set_list_skin", "gx_batch_list_rebuilds", "gx_batch_list_stats",
    "gx_get_list_config", "gx_set_list_threads", "gx_set_list_stash", "gx_set_list_brick", "gx_set_list_block", "gx_get_list_shape", "gx_set_pass_timing", "gx_pass_ms", "gx_bond_observe", "gx_bond_tracker_reset", "gx_get_bonds",
    "gx_bond_components", "gx_collisions", "gx_collision_count", "gx_xyz_frame", "gx_snapshot_world",
    "gx_set_step_async", "gx_tick_host",
)

_lib = None
_OBS_SCALARS = tuple(f for f, _ in GxBondObservation._fields_ if f != "species_matrix")


def load(path: str | Path | None = None) -> C.CDLL:
    """Loads the library (once) and declares every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m genesis_b200.build`")
    lib = C.CDLL(str(p))
    vp, sz, u32p, u64p, dp, u8p = C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), \
        C.POINTER(C.c_double), C.POINTER(C.c_uint8)
    proto = {
        "gx_create": (C.c_int, [C.POINTER(GxParams), C.POINTER(vp)]),
        "gx_destroy": (None, [vp]),
        "gx_last_error": (C.c_char_p, [vp]),
        "gx_status_string": (C.c_char_p, [C.c_int]),
        "gx_set_precision": (C.c_int, [vp, C.c_int]),
        "gx_set_state": (C.c_int, [vp, sz, dp, dp, dp, u8p, dp, dp, u32p]),
        "gx_get_state": (C.c_int, [vp, dp, dp, dp]),
        "gx_num_atoms": (sz, [vp]),
        "gx_set_bonds": (C.c_int, [vp, sz, u32p]),
        "gx_half_kick": (C.c_int, [vp]),
        "gx_drift": (C.c_int, [vp]),
        "gx_wrap": (C.c_int, [vp]),
        "gx_forces": (C.c_int, [vp, dp, dp, u64p]),
        "gx_thermostat": (C.c_int, [vp, dp, dp]),
        "gx_stats": (C.c_int, [vp, dp, dp]),
        "gx_step": (C.c_int, [vp, C.c_int, C.POINTER(GxTickStats), C.c_int]),
        "gx_cell_assign": (C.c_int, [vp, _D, u32p]),
        "gx_neighbors": (C.c_int, [vp, _D, _D, u32p, sz, C.POINTER(sz)]),
        "gx_radial_distribution": (C.c_int, [vp, _D, sz, sz, u64p, dp, dp, dp]),
        "gx_radial_distribution_between": (C.c_int, [vp, C.c_uint8, C.c_uint8, _D, sz, sz, u64p, dp, dp, dp]),
        "gx_clusters": (C.c_int, [vp, _D, u32p, u64p, dp]),
        "gx_bound_pairs": (C.c_int, [vp, _D, u32p, sz, C.POINTER(sz)]),
        "gx_synchronize": (C.c_int, [vp]),
        "gx_profile_enable": (C.c_int, [vp, C.c_int]),
        "gx_profile_read": (C.c_int, [vp, C.POINTER(C.c_char_p), u64p, dp, C.c_int, C.c_int]),
        "gx_set_dynamic": (C.c_int, [vp, dp, dp, dp]),
        "gx_tick_host": (C.c_int, [vp, dp, dp, dp, C.POINTER(GxTickStats)]),
        "gx_timer_mark": (C.c_int, [vp, C.c_int]),
        "gx_timer_elapsed": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "gx_launch_count": (C.c_uint64, [vp]),
        "gx_measure_fp32_peak": (C.c_int, [C.c_int, dp]),
        "gx_measure_fp64_peak": (C.c_int, [C.c_int, dp]),
        "gx_radial_distribution_noalloc": (C.c_int, [sz, dp, dp, _D, sz, u64p, dp, dp, dp]),
        "gx_set_kernel_variant": (C.c_int, [vp, C.c_int]),
        "gx_autotune": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), dp]),
        "gx_adjoint_forward": (C.c_int, [vp, C.POINTER(GxAdjointSpec), dp, dp]),
        "gx_set_list_skin": (C.c_int, [vp, _D]),
        "gx_list_rebuilds": (C.c_int, [vp, u64p]),
        "gx_list_stats": (C.c_int, [vp, u64p, u64p]),
        "gx_get_list_config": (C.c_int, [vp, dp, C.POINTER(C.c_int)]),
        "gx_set_list_threads": (C.c_int, [vp, C.c_int]),
        "gx_set_list_stash": (C.c_int, [vp, C.c_int]),
        "gx_set_list_brick": (C.c_int, [vp, C.c_int]),
        "gx_set_list_block": (C.c_int, [vp, C.c_int]),
        "gx_get_list_shape": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
        "gx_set_pass_timing": (C.c_int, [vp, C.c_int]),
        "gx_pass_ms": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "gx_bond_observe": (C.c_int, [vp, _D, _D, C.c_int, C.c_uint64, C.c_int, C.POINTER(GxBondObservation)]),
        "gx_bond_tracker_reset": (C.c_int, [vp]),
        "gx_get_bonds": (C.c_int, [vp, u32p, sz, C.POINTER(sz)]),
        "gx_bond_components": (C.c_int, [vp, u32p, dp, sz, C.POINTER(sz)]),
        "gx_collisions": (C.c_int, [vp, u64p]),
        "gx_collision_count": (C.c_int, [vp, u64p]),
        "gx_xyz_frame": (C.c_int, [vp, C.c_uint64, C.c_char_p, sz, C.POINTER(sz)]),
        "gx_snapshot_world": (C.c_int, [vp, u32p, C.c_void_p, sz, C.POINTER(sz)]),
        "gx_set_step_async": (C.c_int, [vp, C.c_int]),
        "gx_adjoint_backward": (C.c_int, [vp, dp, dp, dp, dp, dp, dp, dp]),
    }
    for name, (res, args) in proto.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class GxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def params(cfg, precision: str | int = "fp64", device: int = 0) -> GxParams:
    """gx_params from a :class:`genesis_b200.config.Config`."""
    p = GxParams()
    p.box[:] = list(cfg.size)
    p.dt = cfg.dt
    p.thermal_constant = cfg.thermal_constant
    p.sigma[:] = list(cfg.sigma)
    p.epsilon_k[:] = list(cfg.epsilon_k)
    p.charge[:] = list(cfg.charge)
    p.lj_cutoff_factor = E.LJ_CUTOFF_FACTOR
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
    p.precision = _PRECISION[precision] if isinstance(precision, str) else int(precision)
    p.device = device
    return p


class Handle:
    """One resident universe on one GPU (a ``gx_handle``)."""

    def __init__(self, cfg, precision: str | int = "fp64", device: int = 0):
        self.lib = load()
        self.cfg = cfg
        self._p = params(cfg, precision, device)
        h = C.c_void_p()
        rc = self.lib.gx_create(C.byref(self._p), C.byref(h))
        self.h = h
        self._check(rc)

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.gx_last_error(self.h).decode() if self.h else "gx_create failed"
            raise GxError(rc, msg)

    def close(self):
        if self.h:
            self.lib.gx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state --------------------------------------------------------------
    def set_state(self, pos, vel, elem, acc=None, charge=None, mass=None, entity=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        elem = np.ascontiguousarray(elem, dtype=np.uint8)
        n = len(elem)
        acc = None if acc is None else np.ascontiguousarray(acc, dtype=np.float64)
        charge = None if charge is None else np.ascontiguousarray(charge, dtype=np.float64)
        mass = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        entity = None if entity is None else np.ascontiguousarray(entity, dtype=np.uint32)
        self._check(self.lib.gx_set_state(self.h, n, _ptr(pos, C.c_double), _ptr(vel, C.c_double),
                                          _ptr(acc, C.c_double), _ptr(elem, C.c_uint8),
                                          _ptr(charge, C.c_double), _ptr(mass, C.c_double),
                                          _ptr(entity, C.c_uint32)))

    def set_universe(self, u, acc=None):
        self.set_state(u.pos, u.vel, u.elem, acc=acc, charge=u.charge, mass=u.mass, entity=u.entity)

    @property
    def n(self) -> int:
        return int(self.lib.gx_num_atoms(self.h))

    def get_state(self):
        n = self.n
        pos, vel, acc = (np.empty((n, 3)) for _ in range(3))
        self._check(self.lib.gx_get_state(self.h, _ptr(pos, C.c_double), _ptr(vel, C.c_double),
                                          _ptr(acc, C.c_double)))
        return pos, vel, acc

    def set_bonds(self, pairs):
        pairs = np.ascontiguousarray(np.asarray(pairs, dtype=np.uint32).reshape(-1, 2))
        self._check(self.lib.gx_set_bonds(self.h, len(pairs), _ptr(pairs, C.c_uint32)))

    def set_precision(self, precision):
        self._check(self.lib.gx_set_precision(self.h, _PRECISION.get(precision, precision)))

    def set_kernel_variant(self, variant: int):
        """Mixed pair pass: 0 automatic, 1 thread per atom, 2 warp-tiled,
        3 staged rows, 4 per-thread candidate lists, 5 persistent full
        neighbour list, 6 persistent half list with far-end atomics, 7 the
        half list with each thread's in-cutoff entries collected in shared
        memory before the warp evaluates them (same forces as 6), 8 the half
        list brick by brick with the brick's neighbourhood staged in shared
        memory (same forces as 6)."""
        self._check(self.lib.gx_set_kernel_variant(self.h, variant))

    def autotune(self, reps: int = 5):
        """Times every applicable pair-pass variant and keeps the fastest;
        returns (variant, {variant: ms}) -- ms per pass for 1-4, ms per tick
        for 5-8 and 0 (the tick of the best of 1-4)."""
        best = C.c_int()
        ms = np.full(9, -1.0)
        self._check(self.lib.gx_autotune(self.h, reps, C.byref(best), _ptr(ms, C.c_double)))
        return best.value, {v: float(t) for v, t in enumerate(ms) if t >= 0}

    def set_list_skin(self, skin: float):
        """Skin of the variant-5 neighbour list (default 0.1 r_c)."""
        self._check(self.lib.gx_set_list_skin(self.h, skin))

    def list_config(self):
        """(skin, threads per atom) of the variant-5/6 list pass."""
        skin, tpp = C.c_double(), C.c_int()
        self._check(self.lib.gx_get_list_config(self.h, C.byref(skin), C.byref(tpp)))
        return skin.value, tpp.value

    def set_pass_timing(self, on: bool):
        """CUDA events around every tick's pair pass, inside captured ticks too."""
        self._check(self.lib.gx_set_pass_timing(self.h, 1 if on else 0))

    def pass_ms(self) -> float:
        """Device time of the last tick's pair pass (pass timing on)."""
        v = C.c_double()
        self._check(self.lib.gx_pass_ms(self.h, C.byref(v)))
        return v.value

    def list_shape(self) -> dict:
        """The list pass's work shape: threads per atom, far-end block,
        variant-7 stash slots, variant-8 brick cells."""
        v = [C.c_int() for _ in range(4)]
        self._check(self.lib.gx_get_list_shape(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("threads_per_atom", "block", "stash_slots", "brick_cells"), (x.value for x in v)))

    def set_list_threads(self, threads_per_atom: int):
        self._check(self.lib.gx_set_list_threads(self.h, threads_per_atom))

    def set_list_stash(self, slots: int):
        """Stash slots per thread of the variant-7 list pass (8 or 16)."""
        self._check(self.lib.gx_set_list_stash(self.h, slots))

    def set_list_block(self, threads: int):
        """Block of the shared far-end sums of the one-lane half-list pass
        (256, 128, or 0 for every far end in global memory)."""
        self._check(self.lib.gx_set_list_block(self.h, threads))

    def set_list_brick(self, cells: int):
        """Brick length of the variant-8 list pass (4 or 8 cells)."""
        self._check(self.lib.gx_set_list_brick(self.h, cells))

    def list_stats(self) -> tuple[int, int]:
        """(entries held by the neighbour list, atoms whose list overflowed)."""
        e, o = C.c_uint64(), C.c_uint64()
        self._check(self.lib.gx_list_stats(self.h, C.byref(e), C.byref(o)))
        return e.value, o.value

    def list_rebuilds(self) -> int:
        out = C.c_uint64()
        self._check(self.lib.gx_list_rebuilds(self.h, C.byref(out)))
        return out.value

    # -- systems ------------------------------------------------------------
    def half_kick(self):
        self._check(self.lib.gx_half_kick(self.h))

    def drift(self):
        self._check(self.lib.gx_drift(self.h))

    def wrap(self):
        self._check(self.lib.gx_wrap(self.h))

    def forces(self):
        V, Vb, npairs = C.c_double(), C.c_double(), C.c_uint64()
        self._check(self.lib.gx_forces(self.h, C.byref(V), C.byref(Vb), C.byref(npairs)))
        return V.value, Vb.value, npairs.value

    def thermostat(self):
        K, lam = C.c_double(), C.c_double()
        self._check(self.lib.gx_thermostat(self.h, C.byref(K), C.byref(lam)))
        return K.value, lam.value

    def stats(self):
        K, sp = C.c_double(), C.c_double()
        self._check(self.lib.gx_stats(self.h, C.byref(K), C.byref(sp)))
        return K.value, sp.value

    def step(self, nsteps: int, stats: bool = True, graph: bool = False):
        rec = (GxTickStats * max(nsteps, 1))() if stats else None
        self._check(self.lib.gx_step(self.h, nsteps, rec, int(graph)))
        if not stats:
            return None
        return np.frombuffer(rec, dtype=TICK_DTYPE, count=nsteps).copy()

    def synchronize(self):
        self._check(self.lib.gx_synchronize(self.h))

    def set_dynamic(self, pos=None, vel=None, acc=None):
        """Per-tick sync of the dynamic columns from host arrays (slot order)."""
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (pos, vel, acc)]
        self._check(self.lib.gx_set_dynamic(self.h, *(_ptr(x, C.c_double) for x in a)))

    def tick_host(self, pos, vel, acc, stats: bool = True):
        """One tick against host columns (float64 (n, 3), slot order), updated
        in place: gx_set_dynamic + gx_step(1) + gx_get_state in one call with
        the copies overlapped (pinned arrays give the overlap)."""
        for x in (pos, vel, acc):
            if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous
                    and x.shape == (self.n, 3)):
                raise ValueError("tick_host needs C-contiguous float64 (n, 3) arrays")
        rec = (GxTickStats * 1)() if stats else None
        self._check(self.lib.gx_tick_host(self.h, _ptr(pos, C.c_double), _ptr(vel, C.c_double),
                                          _ptr(acc, C.c_double), rec))
        if not stats:
            return None
        return np.frombuffer(rec, dtype=TICK_DTYPE, count=1).copy()

    def get_state_into(self, pos=None, vel=None, acc=None):
        """gx_get_state into caller-owned (e.g. pinned) float64 (n, 3) arrays."""
        self._check(self.lib.gx_get_state(self.h, _ptr(pos, C.c_double), _ptr(vel, C.c_double),
                                          _ptr(acc, C.c_double)))

    def mark(self, slot: int):
        self._check(self.lib.gx_timer_mark(self.h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_double()
        self._check(self.lib.gx_timer_elapsed(self.h, a, b, C.byref(ms)))
        return ms.value

    @property
    def launches(self) -> int:
        return int(self.lib.gx_launch_count(self.h))

    # -- probes and lenses --------------------------------------------------
    def cell_assign(self, min_cell: float) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        self._check(self.lib.gx_cell_assign(self.h, min_cell, _ptr(out, C.c_uint32)))
        return out

    def neighbors(self, min_cell: float, cutoff: float, cap: int | None = None) -> np.ndarray:
        cap = cap if cap is not None else max(64, self.n * 64)
        out = np.empty((cap, 2), dtype=np.uint32)
        total = C.c_size_t()
        self._check(self.lib.gx_neighbors(self.h, min_cell, cutoff, _ptr(out, C.c_uint32), cap,
                                          C.byref(total)))
        return out[: total.value].copy()

    def radial_distribution(self, r_max: float, nbins: int, sample_cap: int = E.G_SAMPLE_CAP,
                            between: tuple[int, int] | None = None):
        nb = min(max(nbins, 1), 1 << 16)
        counts = np.empty(nb, dtype=np.uint64)
        bins = np.empty(nb, dtype=np.float64)
        rmo, dro = C.c_double(), C.c_double()
        if between is None:
            rc = self.lib.gx_radial_distribution(self.h, r_max, nbins, sample_cap, _ptr(counts, C.c_uint64),
                                                 _ptr(bins, C.c_double), C.byref(rmo), C.byref(dro))
        else:
            rc = self.lib.gx_radial_distribution_between(self.h, between[0], between[1], r_max, nbins,
                                                         sample_cap, _ptr(counts, C.c_uint64),
                                                         _ptr(bins, C.c_double), C.byref(rmo), C.byref(dro))
        self._check(rc)
        return counts, bins, rmo.value, dro.value

    def clusters(self, bond_factor: float = E.BOND_FACTOR):
        labels = np.empty(self.n, dtype=np.uint32)
        st = np.zeros(4, dtype=np.uint64)
        mean = C.c_double()
        self._check(self.lib.gx_clusters(self.h, bond_factor, _ptr(labels, C.c_uint32), _ptr(st, C.c_uint64),
                                         C.byref(mean)))
        return labels, {"monomers": int(st[0]), "aggregates": int(st[1]), "largest": int(st[2]),
                        "bound_pairs": int(st[3]), "mean_size": mean.value}

    def bound_pairs(self, k_bind: float, cap: int | None = None) -> np.ndarray:
        cap = cap if cap is not None else max(64, self.n * 16)
        out = np.empty((cap, 2), dtype=np.uint32)
        total = C.c_size_t()
        self._check(self.lib.gx_bound_pairs(self.h, k_bind, _ptr(out, C.c_uint32), cap, C.byref(total)))
        return out[: total.value].copy()

    # -- adjoint --------------------------------------------------------------
    def adjoint_forward(self, nsteps: int, checkpoint_every: int = 20, gr_bins: int = 0, gr_every: int = 1,
                        gr_rmax: float = 1.0, gr_width: float = 0.1, gr_support: float = 6.0):
        """Trajectory of ``nsteps`` NVE ticks from the current state (left
        unchanged): FP64 on an "fp64" handle, the mixed method (FP32 pair law,
        fixed-point force sums, FP64 state) on a "mixed" one; returns (V per
        tick, time-averaged Gaussian-kernel g(r) or None)."""
        spec = GxAdjointSpec(nsteps, checkpoint_every, gr_bins, gr_every, gr_rmax, gr_width, gr_support)
        V = np.zeros(nsteps)
        g = np.zeros(gr_bins) if gr_bins > 0 else None
        self._check(self.lib.gx_adjoint_forward(self.h, C.byref(spec), _ptr(V, C.c_double), _ptr(g, C.c_double)))
        self._adj_T, self._adj_bins = nsteps, gr_bins
        return V, g

    def adjoint_backward(self, dl_dpotential=None, dl_dgr=None, initial_state: bool = False):
        """Gradients of the loss whose cotangents are given, with respect to
        (sigma[10], epsilon_k[10]); with ``initial_state`` also with respect
        to the initial (pos, vel, acc)."""
        dV = None if dl_dpotential is None else np.ascontiguousarray(dl_dpotential, dtype=np.float64)
        dg = None if dl_dgr is None else np.ascontiguousarray(dl_dgr, dtype=np.float64)
        T, bins = getattr(self, "_adj_T", None), getattr(self, "_adj_bins", None)
        if T is not None and dV is not None and len(dV) != T:
            raise ValueError("dl_dpotential needs one entry per tick")
        if bins is not None and dg is not None and len(dg) != bins:
            raise ValueError("dl_dgr needs one entry per g(r) bin")
        gs, ge = np.zeros(10), np.zeros(10)
        st = [np.zeros((self.n, 3)) for _ in range(3)] if initial_state else [None, None, None]
        self._check(self.lib.gx_adjoint_backward(self.h, _ptr(dV, C.c_double), _ptr(dg, C.c_double),
                                                 _ptr(gs, C.c_double), _ptr(ge, C.c_double),
                                                 *(_ptr(a, C.c_double) for a in st)))
        if initial_state:
            return gs, ge, tuple(st)
        return gs, ge

    # -- bond observation ---------------------------------------------------
    def bond_observe(self, k_bind: float, min_periods: float, tick: int, debounce: int = E.DEBOUNCE,
                     apply_bonds: bool = True) -> dict:
        """One tick of bond observation on the device (gx_bond_observe)."""
        o = GxBondObservation()
        self._check(self.lib.gx_bond_observe(self.h, k_bind, min_periods, debounce, tick, int(apply_bonds),
                                             C.byref(o)))
        d = {f: getattr(o, f) for f in _OBS_SCALARS}
        d["species_matrix"] = np.ctypeslib.as_array(o.species_matrix).astype(np.uint64).reshape(10, 10)
        return d

    def bond_components(self):
        """(labels per slot: the smallest slot of the atom's bond component,
        0xFFFFFFFF for an atom in no bond; the raw pair energy of each bond in
        get_bonds() order)."""
        n = int(self.lib.gx_num_atoms(self.h))
        nb = C.c_size_t()
        self._check(self.lib.gx_bond_components(self.h, None, None, 0, C.byref(nb)))
        labels = np.empty(n, dtype=np.uint32)
        energy = np.empty(max(nb.value, 1))
        self._check(self.lib.gx_bond_components(self.h, _ptr(labels, C.c_uint32), _ptr(energy, C.c_double),
                                                len(energy), C.byref(nb)))
        return labels, energy[: nb.value].copy()

    def collisions(self) -> int:
        """One CollisionSystem pass on the resident state; the pairs that collided."""
        c = C.c_uint64()
        self._check(self.lib.gx_collisions(self.h, C.byref(c)))
        return c.value

    def collision_count(self) -> int:
        """Collisions counted by every pass so far."""
        c = C.c_uint64()
        self._check(self.lib.gx_collision_count(self.h, C.byref(c)))
        return c.value

    def bond_tracker_reset(self):
        self._check(self.lib.gx_bond_tracker_reset(self.h))

    def get_bonds(self) -> np.ndarray:
        """The handle's bond list, (m, 2) slot pairs."""
        n = C.c_size_t()
        cap = max(int(self.lib.gx_num_atoms(self.h)) * 8, 64)
        out = np.empty((cap, 2), dtype=np.uint32)
        rc = self.lib.gx_get_bonds(self.h, _ptr(out, C.c_uint32), cap, C.byref(n))
        if rc == -4:
            out = np.empty((n.value, 2), dtype=np.uint32)
            rc = self.lib.gx_get_bonds(self.h, _ptr(out, C.c_uint32), n.value, C.byref(n))
        self._check(rc)
        return out[: n.value].copy()

    def set_step_async(self, on: bool = True):
        """gx_step without records returns without waiting; its errors come
        back from the next call that waits (gx_set_step_async)."""
        self._check(self.lib.gx_set_step_async(self.h, int(on)))

    def xyz_frame(self, tick: int) -> bytes:
        """The XYZ frame of the current state as export::write_frame writes
        it (src/export/mod.rs:152-172), formatted on the device."""
        n = C.c_size_t()
        rc = self.lib.gx_xyz_frame(self.h, int(tick), None, 0, C.byref(n))
        if rc != -4:
            self._check(rc)
        buf = C.create_string_buffer(n.value)
        self._check(self.lib.gx_xyz_frame(self.h, int(tick), buf, n.value, C.byref(n)))
        return buf.raw[: n.value]

    def snapshot_world(self, generation=None) -> bytes:
        """The bincode encoding of the snapshot's Vec<EntitySnapshot>
        (src/serialization/mod.rs:38-56) for the resident atoms, encoded on
        the device (gx_snapshot_world)."""
        gen = None
        if generation is not None:
            gen = np.ascontiguousarray(generation, dtype=np.uint32)
            if gen.shape != (self.n,):
                raise ValueError("one generation per atom")
        n = C.c_size_t()
        gp = _ptr(gen, C.c_uint32) if gen is not None else None
        rc = self.lib.gx_snapshot_world(self.h, gp, None, 0, C.byref(n))
        if rc != -4:
            self._check(rc)
        buf = np.empty(n.value, dtype=np.uint8)
        self._check(self.lib.gx_snapshot_world(self.h, gp, buf.ctypes.data_as(C.c_void_p), n.value, C.byref(n)))
        return buf.tobytes()

    # -- profiling ----------------------------------------------------------
    def profile(self, on: bool = True):
        self._check(self.lib.gx_profile_enable(self.h, int(on)))

    def profile_read(self, reset: bool = True) -> dict:
        cap = 64
        names = (C.c_char_p * cap)()
        launches = np.zeros(cap, dtype=np.uint64)
        ms = np.zeros(cap, dtype=np.float64)
        k = self.lib.gx_profile_read(self.h, names, _ptr(launches, C.c_uint64), _ptr(ms, C.c_double), cap,
                                     int(reset))
        if k < 0:
            self._check(k)
        return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(min(k, cap))}


def measure_fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA throughput (TFLOP/s) of the device."""
    lib = load()
    t = C.c_double()
    rc = lib.gx_measure_fp32_peak(device, C.byref(t))
    if rc != 0:
        raise GxError(rc, "gx_measure_fp32_peak failed")
    return t.value


def measure_fp64_peak(device: int = 0) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of the device."""
    lib = load()
    t = C.c_double()
    rc = lib.gx_measure_fp64_peak(device, C.byref(t))
    if rc != 0:
        raise GxError(rc, "gx_measure_fp64_peak failed")
    return t.value


def radial_distribution_noalloc(pos, box, r_max: float, nbins: int):
    """gx_radial_distribution_noalloc: g(r) of host positions on the current
    device without any device allocation (fixed scratch, 8192-atom sample,
    at most 65536 grid cells).  Returns (counts, bins, r_max, dr)."""
    lib = load()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(box, dtype=np.float64)
    nb = min(max(nbins, 1), 1 << 16)
    counts = np.empty(nb, dtype=np.uint64)
    bins = np.empty(nb, dtype=np.float64)
    rmo, dro = C.c_double(), C.c_double()
    rc = lib.gx_radial_distribution_noalloc(len(pos), _ptr(pos, C.c_double), _ptr(b, C.c_double), r_max, nbins,
                                            _ptr(counts, C.c_uint64), _ptr(bins, C.c_double), C.byref(rmo),
                                            C.byref(dro))
    if rc != 0:
        raise GxError(rc, "gx_radial_distribution_noalloc: " + lib.gx_status_string(rc).decode())
    return counts, bins, rmo.value, dro.value


class Batch:
    """Many independent universes advanced together in one persistent launch
    (a ``gx_batch``): the temperature-sweep replicas."""

    def __init__(self, base_cfg, boxes, targets=None, device: int = 0):
        self.lib = load()
        _declare_batch(self.lib)
        self._p = params(base_cfg, "mixed", device)
        boxes = np.ascontiguousarray(np.asarray(boxes, dtype=np.float64).reshape(-1, 3))
        self.nrep = len(boxes)
        tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.float64)
        b = C.c_void_p()
        rc = self.lib.gx_batch_create(C.byref(self._p), self.nrep, _ptr(boxes, C.c_double), _ptr(tg, C.c_double),
                                      C.byref(b))
        self.b = b
        self._check(rc)
        self.natoms = None

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.gx_batch_last_error(self.b).decode() if self.b else "gx_batch_create failed"
            raise GxError(rc, msg)

    def close(self):
        if self.b:
            self.lib.gx_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_universes(self, universes):
        self.natoms = np.array([u.n for u in universes], dtype=np.uint32)
        cat = lambda f: np.ascontiguousarray(np.concatenate([getattr(u, f) for u in universes]))  # noqa: E731
        pos, vel, elem, q, m = cat("pos"), cat("vel"), cat("elem").astype(np.uint8), cat("charge"), cat("mass")
        self._check(self.lib.gx_batch_set_state(self.b, _ptr(self.natoms, C.c_uint32), _ptr(pos, C.c_double),
                                                _ptr(vel, C.c_double), None, _ptr(elem, C.c_uint8),
                                                _ptr(q, C.c_double), _ptr(m, C.c_double)))

    def step(self, nsteps: int):
        """Returns (stats[nrep, 4] = K, V, lambda, pairs; device milliseconds)."""
        st = np.zeros((self.nrep, 4))
        ms = C.c_double()
        self._check(self.lib.gx_batch_step(self.b, nsteps, _ptr(st, C.c_double), C.byref(ms)))
        return st, ms.value

    def set_mode(self, mode: int):
        """1 = persistent launch (one CTA per replica), 2 = all-replica graph,
        3 = the all-replica phases in one persistent cooperative launch,
        4 = the all-replica graph over persistent neighbour lists."""
        self._check(self.lib.gx_batch_set_mode(self.b, mode))

    @property
    def mode(self) -> int:
        m = C.c_int()
        self._check(self.lib.gx_batch_get_mode(self.b, C.byref(m)))
        return m.value

    def set_list_skin(self, skin: float):
        """Skin of mode 4's neighbour lists (default 0.15 r_c)."""
        self._check(self.lib.gx_batch_set_list_skin(self.b, skin))

    def list_rebuilds(self) -> int:
        """Mode 4's list rebuilds so far."""
        v = C.c_uint64()
        self._check(self.lib.gx_batch_list_rebuilds(self.b, C.byref(v)))
        return v.value

    def list_stats(self):
        """(entries, overflowed slots) of mode 4's current lists."""
        e, o = C.c_uint64(), C.c_uint64()
        self._check(self.lib.gx_batch_list_stats(self.b, C.byref(e), C.byref(o)))
        return e.value, o.value

    def autotune(self, ticks: int = 10):
        """Times the four modes from a snapshot, keeps the fastest: (mode, {mode: ms per tick})."""
        m = C.c_int()
        ms = np.zeros(4)
        self._check(self.lib.gx_batch_autotune(self.b, ticks, C.byref(m), _ptr(ms, C.c_double)))
        return m.value, {k + 1: float(t) for k, t in enumerate(ms) if t >= 0}

    def get_state(self):
        n = int(self.natoms.sum())
        pos, vel, acc = (np.empty((n, 3)) for _ in range(3))
        self._check(self.lib.gx_batch_get_state(self.b, _ptr(pos, C.c_double), _ptr(vel, C.c_double),
                                                _ptr(acc, C.c_double)))
        offs = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        return [(pos[a:b], vel[a:b], acc[a:b]) for a, b in zip(offs[:-1], offs[1:])]


_batch_declared = False


def _declare_batch(lib):
    global _batch_declared
    if _batch_declared:
        return
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    proto = {
        "gx_batch_create": (C.c_int, [C.POINTER(GxParams), C.c_int, dp, dp, C.POINTER(vp)]),
        "gx_batch_destroy": (None, [vp]),
        "gx_batch_last_error": (C.c_char_p, [vp]),
        "gx_batch_set_state": (C.c_int, [vp, C.POINTER(C.c_uint32), dp, dp, dp, C.POINTER(C.c_uint8), dp, dp]),
        "gx_batch_step": (C.c_int, [vp, C.c_int, dp, dp]),
        "gx_batch_get_state": (C.c_int, [vp, dp, dp, dp]),
        "gx_batch_set_mode": (C.c_int, [vp, C.c_int]),
        "gx_batch_get_mode": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "gx_batch_autotune": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), dp]),
        "gx_batch_set_list_skin": (C.c_int, [vp, C.c_double]),
        "gx_batch_list_rebuilds": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "gx_batch_list_stats": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    }
    for name, (res, args) in proto.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _batch_declared = True
