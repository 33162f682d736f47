#!/usr/bin/env python
"""Headline benchmark of the per-tick particle hot path on B200.

Workload: the 2,097,152-atom condensation quench (128^3 lattice, spacing
1.2 x max sigma, 10-element mixture with the element charges, LJ + Coulomb,
velocities at 300 K, Berendsen to 20 K, g(r) every 100 ticks with 256 bins
and r_max = 3 r_c), one tick = kick, drift, wrap, cell sort, pair pass, kick,
thermostat.  Synthetic seeded inputs; the state (~300 MB) is larger than L2,
so no flush is needed between ticks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun each rank advances its own
replica of the workload on its own GPU (the single-universe path has no
inter-GPU exchange in this build), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "atom-steps/s/GPU mixed vs plain FP64 at ≤1e-5 force err; replica-steps/s"
UNIT = "atom-steps/s"
FLOP_PER_PAIR_LJ = 67      # algorithmic FLOPs per in-cutoff pair (LJ), FMA = 2
FLOP_PER_PAIR_LJC = 75     # with Coulomb sharing the switch
# the list pass of a tick that records nothing leaves out the potential
# (its product with the switch and its sum: 2 FLOPs per term)
FLOP_PER_PAIR_LJ_NOV = 65
FLOP_PER_PAIR_LJC_NOV = 71
# Algorithmic bytes per atom of each memory-bound kernel (reads + writes of
# the arrays the kernel must touch; FP64 state, u8 element/kind, u32 ids).
BYTES_PER_ATOM = {
    "kick": 72, "drift": 72, "wrap": 48, "cell_keys": 28, "cell_count": 4, "cell_scan": 0,
    # scatter: read key, read the cell's start, write the slot; the per-cell
    # ranking: read key, the cell's start and end, write the slot (the cell's
    # segment it scans is an L1/L2 hit)
    "cell_scatter": 12, "cell_rank": 16, "reorder": 220, "stage_pos4": 45, "kinetic": 32,
    # list path: fused kick + drift + wrap + FP32 staging + displacement test
    # (read x v a 72, kind 1, home cell 4, reference float4 16; write x v 48,
    # float4 16, and zero the int64 force sums 24 for the half-list pass),
    # and fused F -> a + kick + K (read F 24, v 24, 1/m 8, m 8; write a 24,
    # v 24)
    "nl_advance": 181, "nl_finish": 112,
    # list rebuild: the sorted state copied back (12 f64 columns, 2 u8, 1 u32,
    # read and written), the staging (read x y z 24, kind 1, home 4; write
    # the float4 and its reference copy 32); the list build's own bytes
    # depend on the entries it writes (list_build_bytes_per_atom)
    "nl_copy": 204, "nl_stage": 61,
}
# kernels that run only on ticks that rebuild the neighbour list
REBUILD_KERNELS = ("cell_keys", "cell_count", "cell_scan", "cell_scatter", "cell_rank", "reorder", "nl_copy",
                   "nl_stage", "nl_build")


def list_build_bytes_per_atom(entries_per_atom: float) -> float:
    """k_nl_build: read the atom's float4 16 and home cell 4, write its count
    4 and its list entries 4 each; the candidates it tests are L1/L2 hits of
    the same float4 array."""
    return 24.0 + 4.0 * entries_per_atom



def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--n-side", type=int, default=0, help="override the lattice edge (testing only)")
    ap.add_argument("--no-extras", action="store_true", help="skip fp64/e2e/cpu legs (testing only)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="fix the mixed pair-pass variant instead of autotuning (profiling only)")
    ap.add_argument("--list-block", type=int, default=-1,
                    help="block of the shared far-end sums of the one-lane half-list pass: 256, 128 or 0 "
                         "(profiling only)")
    ap.add_argument("--skin", type=float, default=-1.0,
                    help="neighbour-list skin in length units instead of 0.1 r_c (profiling only; 0 = rebuild every tick)")
    ap.add_argument("--leg", default="",
                    choices=["", "ionic", "accuracy", "adjoint", "xyz", "sweep", "c1", "rebuild", "gr", "fp64"],
                    help="run one extra leg alone and print its JSON (profiling only)")
    ap.add_argument("--leg-steps", type=int, default=0, help="ticks of the --leg run (0: the workload's own)")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed


class Dist:
    def __init__(self, n_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = os.environ.get("GENESIS_DIST_BACKEND", "nccl")
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=60))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def all_gather_object(self, obj) -> list:
        """Every rank's `obj`, in rank order (one collective)."""
        if not self.pg:
            return [obj]
        out = [None] * self.world
        self.pg.all_gather_object(out, obj)
        return out

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: the timed region begins
            # once the first sample is in, so every sample falls inside it
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 3.0 and not Path(self.path).read_text().strip():
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and f[1].replace(".", "").isdigit():
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()) if rows else None,
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------- helpers


def workload(args):
    from genesis_b200 import workloads as W

    wl = W.WORKLOADS[args.workload]
    if args.n_side:
        wl = wl.scaled(args.n_side)
    return wl


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def ncu_figure(key: str, kernel: str) -> float | None:
    """A `key[kernel]: value` figure from the committed ncu summaries."""
    for f in (ROOT / "profiles").glob("*.txt"):
        for line in f.read_text().splitlines():
            if line.startswith(f"{key}[{kernel}]"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except Exception:
                    return None
    return None


def ncu_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch from the committed ncu summary, if present."""
    return ncu_figure("traffic_bytes_per_launch", kernel)


def hbm_peak() -> tuple[float, str]:
    hbm = measured_peaks().get("hbm_gbs")
    if hbm:
        return hbm, "MEASURED_PEAKS.json hbm_gbs (of measured)"
    # without the measured file: a copy bandwidth measured earlier on the same B200 model
    return 6650.0, "fallback 6650 GB/s (of fallback: an earlier copy-bandwidth measurement)"


XYZ_READ_BYTES_PER_ATOM = 29  # x, y, z f64 + element u8 + the slot's sorted position u32


def xyz_leg(h, elem, tick: int, cpu: bool, reps: int = 5) -> dict:
    """XYZ frame export (export::write_frame) of the resident state: the
    device formatter's kernels (profiled), end to end into a pinned host
    buffer, the bytes against the oracle's printf text, and that text's
    single-thread CPU time (the reference formats its frame in one loop)."""
    import ctypes as C

    import numpy as np
    import torch

    n = C.c_size_t()
    rc = h.lib.gx_xyz_frame(h.h, tick, None, 0, C.byref(n))
    if rc not in (0, -4):
        h._check(rc)
    size = n.value
    buf = torch.empty(size, dtype=torch.uint8, pin_memory=True)
    ptr = C.cast(C.c_void_p(buf.data_ptr()), C.c_char_p)
    for _ in range(2):
        h._check(h.lib.gx_xyz_frame(h.h, tick, ptr, size, C.byref(n)))
    h.profile(True)
    walls = []
    for _ in range(reps):
        t0 = time.perf_counter()
        h._check(h.lib.gx_xyz_frame(h.h, tick, ptr, size, C.byref(n)))
        walls.append(time.perf_counter() - t0)
    prof = h.profile_read(reset=True)
    h.profile(False)
    atoms = len(elem)
    text = bytes(buf.numpy()[:size])
    wall = float(np.median(walls))
    out = {"workload": f"one XYZ frame of the resident state: {atoms} atoms, {size} bytes of text",
           "bytes": size, "e2e": {"ms": wall * 1e3, "atoms_per_s": atoms / wall, "GB_per_s": size / wall / 1e9,
                                   "timing": "host wall clock, median of 5 gx_xyz_frame calls into pinned memory "
                                             "(both kernels, the scan, the size read-back and the D2H copy)"}}
    hbm, src = hbm_peak()
    kern = {}
    for k, (nl, kms) in prof.items():
        if k.startswith("xyz_") and nl:
            per = kms / nl
            alg = XYZ_READ_BYTES_PER_ATOM * atoms + (size if k == "xyz_write" else 0)
            kern[k] = {"launch_ms": per, "algorithmic_bytes": alg, "GB/s": alg / (per * 1e-3) / 1e9}
    out["kernels"] = kern
    if "xyz_write" in kern:
        a = kern["xyz_write"]["GB/s"]
        out["roofline"] = {"kernel": "xyz_write", "bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                           "frac": a / hbm, "peak_source": src, "traffic": ncu_traffic("xyz_write")}
    if cpu:
        from oracle import oracle

        pos, _, _ = h.get_state()
        t0 = time.perf_counter()
        want = oracle.xyz_frame(tick, pos, elem)
        tc = time.perf_counter() - t0
        out["matches_oracle"] = want == text
        out["cpu_baseline"] = {"ms": tc * 1e3, "atoms_per_s": atoms / tc, "cores": 1, "kind": "port",
                               "sample": "the same frame, C restatement (printf %.6f) on one host thread"}
        out["e2e_over_cpu"] = tc / wall
    return out


def gr_leg(h, n_atoms: int, reps: int = 3) -> dict:
    """g(r) of the resident state (radial_distribution, src/analysis/mod.rs:87-133):
    the reference's call (a subsample of at most 8192 atoms, 256 bins to
    r_max = 3 r_c = 17.25) and the whole state without the subsample, which
    gives the pair throughput.  Host wall clock around the synchronous call."""
    import numpy as np

    walls = []
    for _ in range(reps):
        t0 = time.perf_counter()
        h.radial_distribution(17.25, 256)
        walls.append(time.perf_counter() - t0)
    h.radial_distribution(17.25, 256, sample_cap=n_atoms)  # warm-up: staging sized for every atom
    t0 = time.perf_counter()
    counts, _, _, _ = h.radial_distribution(17.25, 256, sample_cap=n_atoms)
    full = time.perf_counter() - t0
    pairs = int(counts.sum())
    return {"workload": f"g(r) of the resident state, 256 bins to r_max 17.25, {n_atoms} atoms",
            "subsample": {"atoms": min(n_atoms, 8192), "ms": float(np.median(walls)) * 1e3},
            "full": {"atoms": n_atoms, "ms": full * 1e3, "pairs_within_rmax": pairs,
                     "pairs_per_s": pairs / full, "position_GB_per_s": 16.0 * n_atoms / full / 1e9},
            "timing": "host wall clock around each synchronous gx_radial_distribution call"}


def lens_leg(h, k_bind: float) -> dict:
    """The structure lenses on the resident state: friends-of-friends
    (clusters, src/analysis/mod.rs:221-307) and the bound pairs
    (bound_pairs_with_grid, src/analysis/pairs.rs:132-174).  Host wall clock
    around each synchronous call, the second of two."""
    out = {}
    for name, call in (("fof", lambda: h.clusters()), ("bound_pairs", lambda: h.bound_pairs(k_bind))):
        call()
        t0 = time.perf_counter()
        r = call()
        ms = (time.perf_counter() - t0) * 1e3
        out[name] = {"ms": ms}
        if name == "fof":
            out[name].update({k: r[1][k] for k in ("aggregates", "largest", "bound_pairs")})
        else:
            out[name]["pairs"] = int(len(r))
    out["timing"] = "host wall clock around each synchronous call (labels or pairs copied back)"
    return out


def run_ticks(h, wl, cfg, steps: int, start_tick: int, record: bool = True) -> int:
    """steps ticks through gx_step, with the workload's g(r) every gr_every
    ticks.  With `record` every tick records K, V, lambda and the in-cutoff
    pair count on the device (the reference computes the potential every
    tick, src/systems/forces.rs:347, for StatsSystem,
    src/systems/aggregate.rs:86-143); without it the pair pass leaves the
    potential and the pair count out."""
    from genesis_b200 import elements as E

    t = start_tick
    done = 0
    rc = E.LJ_CUTOFF_FACTOR * max(cfg.sigma)
    while done < steps:
        k = steps - done
        if wl.gr_every:
            k = min(k, wl.gr_every - (t % wl.gr_every))
        h.step(k, stats=record, graph=True)
        done += k
        t += k
        if wl.gr_every and t % wl.gr_every == 0:
            h.radial_distribution(wl.gr_rmax_factor * rc, wl.gr_bins, E.G_SAMPLE_CAP)
    return t


def cpu_reference(wl, cfg, u, budget_s: float, threads: int) -> dict:
    """The oracle's threaded restatement of the reference's rayon tick."""
    from oracle import oracle

    pos, vel, acc = u.pos, u.vel, None
    oracle.ticks(cfg, pos[:1], vel[:1], None, u.elem[:1], u.charge[:1], u.mass[:1], 1, nthreads=1)
    ticks, elapsed = 0, 0.0
    while elapsed < budget_s or ticks == 0:
        t0 = time.perf_counter()
        pos, vel, acc, _ = oracle.ticks(cfg, pos, vel, acc, u.elem, u.charge, u.mass, 1, nthreads=threads)
        elapsed += time.perf_counter() - t0
        ticks += 1
        if elapsed > 3 * budget_s:
            break
    return {"value": u.n * ticks / elapsed, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{ticks} full ticks of the {u.n}-atom workload ({elapsed:.1f} s), C++ restatement of the "
                      f"reference rayon tick on {threads} host threads"}


# ---------------------------------------------------------------- arms


def accuracy_leg(dev: int, steps: int = 10000) -> dict:
    """NVE energy conservation of the mixed path against the plain FP64 path
    on the C1 workload (4,096 atoms, LJ, 60 K): relative drift of E = K + V
    over `steps` ticks (slope of a straight-line fit times the run length),
    RMS of the per-tick change of E, and the L1 distance of the two final
    g(r) histograms (256 bins to r = 17.25, normalised to unit sum)."""
    import numpy as np

    from genesis_b200 import workloads as W
    from genesis_b200._lib import Handle

    wl = W.C1
    cfg = wl.config()
    u = wl.generate()
    out = {"workload": f"{wl.name}: {u.n} atoms, 60 K, NVE, {steps} ticks"}
    hists = {}
    for prec in ("fp64", "mixed"):
        with Handle(cfg, prec, dev) as h:
            h.set_universe(u)
            st = h.step(steps, stats=True, graph=True)
            E = st["kinetic"] + st["potential"]
            t = np.arange(len(E))
            slope = np.polyfit(t, E, 1)[0]
            e0 = abs(E[0])
            c, _, _, _ = h.radial_distribution(17.25, 256)
            hists[prec] = c / max(c.sum(), 1)
            out[prec] = {"drift_rel": float(slope * steps / e0), "step_rms_rel": float(np.std(np.diff(E)) / e0),
                         "E0": float(E[0]), "E_end": float(E[-1])}
    out["drift_ratio_mixed_over_fp64"] = abs(out["mixed"]["drift_rel"]) / max(abs(out["fp64"]["drift_rel"]), 1e-300)
    out["gr_L1_mixed_vs_fp64"] = float(np.abs(hists["mixed"] - hists["fp64"]).sum())
    return out


def c1_leg(dev: int, cpu: bool, steps: int = 1000, cpu_budget_s: float = 8.0) -> dict:
    """Throughput on the C1 workload (4,096 atoms, 16^3 lattice, LJ only,
    60 K NVE, 1,000 ticks; the configuration the reference runs on its CPU
    today): the mixed path and the plain FP64 path through gx_step as captured
    ticks that record K, V and pairs every tick, and with `cpu` the oracle's
    threaded restatement of the reference tick on the host cores over a
    bounded sample of the same run."""
    from genesis_b200 import workloads as W
    from genesis_b200._lib import Handle

    wl = W.C1
    cfg, u = wl.config(), wl.generate()
    out = {"workload": f"{wl.name}: {u.n} atoms, LJ, 60 K NVE, {steps} ticks",
           "timing": "CUDA events around gx_step(steps) of captured ticks, after 5 warm-up ticks"}
    for prec in ("mixed", "fp64"):
        with Handle(cfg, prec, dev) as h:
            h.set_universe(u)
            picked = None
            if prec == "mixed":
                picked, _ = h.autotune(reps=3)  # state unchanged
            h.step(5, stats=True, graph=True)
            h.synchronize()
            h.mark(0)
            h.step(steps, stats=True, graph=True)
            h.mark(1)
            ms = h.elapsed_ms(0, 1)
            out[prec] = {"value": u.n * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
                         "kernel_variant": picked}
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    if cpu:
        from oracle import oracle

        threads = os.cpu_count() or 1
        p, v, a = u.pos, u.vel, None
        ticks, el = 0, 0.0
        while (el < cpu_budget_s or ticks == 0) and ticks < steps:
            t0 = time.perf_counter()
            p, v, a, _ = oracle.ticks(cfg, p, v, a, u.elem, u.charge, u.mass, 10, nthreads=threads)
            el += time.perf_counter() - t0
            ticks += 10
        out["cpu_baseline"] = {"value": u.n * ticks / el, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"the first {ticks} ticks of the run ({el:.1f} s): C++ restatement of the "
                                         f"reference rayon tick on {threads} host threads"}
        out["mixed_over_cpu"] = out["mixed"]["value"] / out["cpu_baseline"]["value"]
    return out


def adjoint_leg(dev: int) -> dict:
    """Wall-clock cost of one adjoint gradient on the C5 workload (8,000
    atoms, 200 NVE ticks, checkpoint every 20), the cost of the 40 forward
    runs central differences need, and the largest disagreement."""
    import numpy as np

    from genesis_b200 import adjoint as adj
    from genesis_b200._lib import Handle

    _, acfg, au = adj.c5()
    spec = adj.AdjointSpec()
    target = adj.gr_target(acfg, au, spec, dev)
    with Handle(acfg, "fp64", dev) as ha:
        ha.set_universe(au)
        ha.adjoint_forward(spec.nsteps, **spec.kwargs())  # warm-up
        ha.adjoint_backward(np.full(spec.nsteps, 1.0 / spec.nsteps))
        l0 = ha.launches
        t0 = time.perf_counter()
        V, g = ha.adjoint_forward(spec.nsteps, **spec.kwargs())
        t1 = time.perf_counter()
        lv, cv = adj.potential_loss(V)
        gsV, geV = ha.adjoint_backward(dl_dpotential=cv)
        t2 = time.perf_counter()
        lg, cg = adj.gr_loss(g, target)
        gsG, geG = ha.adjoint_backward(dl_dgr=cg)
        t3 = time.perf_counter()
        launches = ha.launches - l0
    tf = time.perf_counter()
    fd = adj.fd_gradients(acfg, au, spec, target, 1e-5, dev)
    fd_s = time.perf_counter() - tf

    def err(ad, ref):
        return float(np.max(np.abs(ad - ref) / (np.abs(ref) + 1e-6 * np.abs(ref).max())))

    grad_ms = (t1 - t0 + t2 - t1) * 1e3
    return {"workload": "adjoint LJ NVE 20^3: 8000 atoms, 60 K, 200 ticks, checkpoint every 20",
            "parameters": "10 sigma + 10 epsilon_k", "precision": "fp64",
            "losses": {"potential": "<V> over the 200 ticks", "gr": "sum_k (gbar_k - target_k)^2, Gaussian kernel "
                       f"w = {spec.gr_width:.4f} (0.05 max sigma), {spec.gr_bins} centres to {spec.gr_rmax}, "
                       "target = same run with sigma x 1.02"},
            "forward_ms": (t1 - t0) * 1e3, "backward_ms": ((t2 - t1) + (t3 - t2)) * 0.5e3,
            "gradient_ms": grad_ms, "fd_ms": fd_s * 1e3, "fd_runs": 40,
            "speedup_vs_fd": fd_s * 1e3 / grad_ms, "gpu_launches": launches,
            "max_rel_err_vs_fd": {"potential": err(np.r_[gsV, geV], fd["potential"]),
                                  "gr": err(np.r_[gsG, geG], fd["gr"])},
            "fd_step": "central, 1e-5 x parameter", "loss_values": {"potential": lv, "gr": lg},
            "timing": "host wall clock around the synchronous C-ABI calls",
            "mixed_forward": mixed_adjoint(acfg, au, spec, target, fd, err, dev)}


def mixed_adjoint(acfg, au, spec, target, fd, err, dev: int) -> dict:
    """The C5 form: the forward in the mixed method (FP32 pair law,
    fixed-point force sums), the FP64 adjoint on that trajectory, against the
    central differences of the FP64 forward."""
    import numpy as np

    from genesis_b200 import adjoint as adj
    from genesis_b200._lib import Handle

    with Handle(acfg, "mixed", dev) as hm:
        hm.set_universe(au)
        hm.adjoint_forward(spec.nsteps, **spec.kwargs())  # warm-up
        t0 = time.perf_counter()
        V, g = hm.adjoint_forward(spec.nsteps, **spec.kwargs())
        t1 = time.perf_counter()
        gsV, geV = hm.adjoint_backward(dl_dpotential=adj.potential_loss(V)[1])
        t2 = time.perf_counter()
        gsG, geG = hm.adjoint_backward(dl_dgr=adj.gr_loss(g, target)[1])
    return {"precision": "FP32 pair law + 64-bit fixed-point force sums forward, FP64 adjoint",
            "forward_ms": (t1 - t0) * 1e3, "gradient_ms": (t2 - t0) * 1e3,
            "max_rel_err_vs_fd": {"potential": err(np.r_[gsV, geV], fd["potential"]),
                                  "gr": err(np.r_[gsG, geG], fd["gr"])},
            "fd": "the FP64 forward's central differences above"}


def ionic_leg(dev: int, cpu: bool, steps: int | None = None, cpu_budget_s: float = 10.0, variant: int = -1) -> dict:
    """The C2 workload run whole: 32,768 Na+/O- atoms (32^3 lattice), LJ +
    Coulomb, Berendsen at 300 K, bond observation every tick with the
    persistent pairs driving the spring from the next tick on, 5,000 ticks,
    through the mixed and the plain FP64 path; the mixed pass's force error
    against FP64 on the final state with its bonds; with `cpu`, the oracle's
    threaded tick plus the same observation on the host cores over a
    bounded sample."""
    import numpy as np

    from genesis_b200 import elements as E
    from genesis_b200 import workloads as W
    from genesis_b200._lib import Handle

    wl = W.C2
    cfg, u = wl.config(), wl.generate()
    steps = steps or wl.steps
    kb, mp = cfg.bond_k_bind, cfg.bond_min_periods
    out = {"workload": f"{wl.name}: {u.n} atoms, Na+/O- 50/50 shuffled, LJ + Coulomb, Berendsen 300 K, bond "
                       f"observation every tick (k_bind {kb}, min_periods {mp}) feeding the spring, {steps} ticks",
           "timing": "host wall clock over the whole run from the generated state: gx_step(1) as a captured "
                     "tick (queued without a wait, gx_set_step_async) + gx_bond_observe every tick"}
    final = {}
    for prec in ("mixed", "fp64"):
        with Handle(cfg, prec, dev) as h:
            h.set_universe(u)
            picked = None
            if prec == "mixed" and variant >= 0:
                h.set_kernel_variant(variant)
                picked = variant
            elif prec == "mixed":
                picked, _ = h.autotune(reps=3)  # state unchanged
            ob = None
            l0 = h.launches
            h.set_step_async(True)  # the tick is queued; the observation's wait covers both
            h.synchronize()
            t0 = time.perf_counter()
            for t in range(1, steps + 1):
                h.step(1, stats=False, graph=True)
                ob = h.bond_observe(kb, mp, t)
            h.synchronize()
            el = time.perf_counter() - t0
            h.set_step_async(False)
            launches = h.launches - l0
            final[prec] = (h.get_state(), h.get_bonds())
            # the same ticks without the observation, from the final state
            # with its final bonds: the cost of the tick alone
            h.step(3, stats=False, graph=True)
            h.synchronize()
            k2 = min(steps, 1000)
            h.mark(0)
            h.step(k2, stats=False, graph=True)
            h.mark(1)
            tick_ms = h.elapsed_ms(0, 1) / k2
            out[prec] = {"value": u.n * steps / el, "unit": UNIT, "ms_per_step": el * 1e3 / steps,
                         "tick_only_ms": tick_ms, "gpu_launches": launches,
                         "kernel_variant": picked,
                         "end": {"bound_pairs": ob["bound_pairs"], "bonded_pairs": ob["bonded_pairs"],
                                 "bonds_formed": ob["bonds_formed"], "mean_coordination": ob["mean_coordination"],
                                 "completed_episodes": ob["completed_episodes"]}}
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    (pos, vel, _), bonds = final["mixed"]
    res = {}
    for prec in ("mixed", "fp64"):
        with Handle(cfg, prec, dev) as h:
            h.set_state(pos, vel, u.elem, charge=u.charge, mass=u.mass, entity=u.entity)
            h.set_bonds(bonds)
            V, Vb, _ = h.forces()
            res[prec] = (h.get_state()[2], V, Vb)
    am, Vm, Vbm = res["mixed"]
    a64, V64, Vb64 = res["fp64"]
    out["force_rel_rms_vs_fp64"] = float(np.linalg.norm(am - a64) / np.linalg.norm(a64))
    out["potential_rel_err_vs_fp64"] = abs(Vm - V64) / abs(V64)
    out["bond_energy_rel_err_vs_fp64"] = abs(Vbm - Vb64) / abs(Vb64) if Vb64 else None
    out["bonds_in_accuracy_state"] = int(len(bonds))
    # With the workload's persistence (10 vibration periods, about 3,200
    # ticks of one uninterrupted episode) no bond forms at 300 K.  To measure
    # the spring's error as well, the same system is observed with the
    # reference's floor of 0.1 periods (bonds persist after ~32 ticks).
    mp_fast = 0.1
    with Handle(cfg, "mixed", dev) as h:
        h.set_universe(u)
        for t in range(1, 121):
            h.step(1, stats=False, graph=True)
            ob = h.bond_observe(kb, mp_fast, t)
        (pos, vel, _), bonds = h.get_state(), h.get_bonds()
    res = {}
    for prec in ("mixed", "fp64"):
        with Handle(cfg, prec, dev) as h:
            h.set_state(pos, vel, u.elem, charge=u.charge, mass=u.mass, entity=u.entity)
            h.set_bonds(bonds)
            V, Vb, _ = h.forces()
            res[prec] = (h.get_state()[2], V, Vb)
    am, Vm, Vbm = res["mixed"]
    a64, V64, Vb64 = res["fp64"]
    out["with_bonds"] = {"min_periods": mp_fast, "ticks": 120, "bonds": int(len(bonds)),
                         "bonds_formed": ob["bonds_formed"],
                         "force_rel_rms_vs_fp64": float(np.linalg.norm(am - a64) / np.linalg.norm(a64)),
                         "potential_rel_err_vs_fp64": abs(Vm - V64) / abs(V64),
                         "bond_energy_rel_err_vs_fp64": abs(Vbm - Vb64) / abs(Vb64) if Vb64 else None,
                         "bond_energy": Vb64}
    if cpu:
        from oracle import oracle

        threads = os.cpu_count() or 1
        tr = oracle.BondTracker(cfg, debounce=E.DEBOUNCE)
        p, v, a = u.pos, u.vel, None
        bl = np.zeros((0, 2), dtype=np.uint32)
        ticks, el = 0, 0.0
        while el < cpu_budget_s or ticks == 0:
            t0 = time.perf_counter()
            p, v, a, _ = oracle.ticks(cfg, p, v, a, u.elem, u.charge, u.mass, 1, bonds=bl, nthreads=threads)
            bp = oracle.bound_pairs(p, u.elem, u.entity, cfg.size, kb, cfg.sigma)
            _, bl = tr.observe(bp, u.elem, ticks + 1)
            el += time.perf_counter() - t0
            ticks += 1
        out["cpu_baseline"] = {"value": u.n * ticks / el, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"the first {ticks} ticks of the workload ({el:.1f} s): C++ restatement of "
                                         f"the reference tick on {threads} host threads + bound pairs + pair "
                                         "tracker, observed bonds fed back"}
        out["mixed_over_cpu"] = out["mixed"]["value"] / out["cpu_baseline"]["value"]
    return out


def kernel_leg(args, dev: int) -> dict:
    """Profiling legs on the quench workload (scaled by --n-side): `rebuild`
    runs eager ticks that each rebuild the neighbour list (setting the skin
    again forces one), so every launch of the rebuild kernels does its work;
    `gr` runs g(r) of the whole state (no subsample); `fp64` runs eager
    ticks of the plain FP64 path.  Prints per-kernel device times."""
    import dataclasses

    from genesis_b200 import workloads as W
    from genesis_b200._lib import Handle

    wl = W.C3 if args.n_side <= 0 else dataclasses.replace(W.C3, n_side=args.n_side)
    cfg, u = wl.config(), wl.generate()
    reps = args.leg_steps or 5
    prec = "fp64" if args.leg == "fp64" else "mixed"
    with Handle(cfg, prec, dev) as h:
        if args.variant >= 0:
            h.set_kernel_variant(args.variant)
        h.set_universe(u)
        h.step(2, stats=True)
        h.profile(True)
        if args.leg == "rebuild":
            skin, _ = h.list_config()
            for _ in range(reps):
                h.set_list_skin(skin)
                h.step(1, stats=True)
        elif args.leg == "gr":
            for _ in range(reps):
                h.radial_distribution(17.25, 256, sample_cap=u.n)
        else:
            h.step(reps, stats=True)
        prof = h.profile_read(reset=True)
        h.profile(False)
        entries, overflowed = h.list_stats()
    return {"workload": f"{wl.name} at {u.n} atoms, {prec}", "reps": reps, "list_entries": entries,
            "overflowed_atoms": overflowed,
            "kernels_ms_per_launch": {k: v[1] / max(v[0], 1) for k, v in prof.items()},
            "launches": {k: v[0] for k, v in prof.items()}}


def reference_arm(args, dist):
    if dist.rank != 0:
        return
    wl = workload(args)
    cfg = wl.config()
    u = wl.generate()
    threads = os.cpu_count() or 1
    budget = float(os.environ.get("GENESIS_REF_BUDGET_S", "60"))
    cb = cpu_reference(wl, cfg, u, budget, threads)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "atoms": u.n, "host_threads": threads},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ours_arm(args, dist):
    import numpy as np

    from genesis_b200 import _lib
    from genesis_b200._lib import Handle

    wl = workload(args)
    cfg = wl.config()
    u = wl.generate(salt=dist.rank)
    dev = dist.local
    K, Wm = args.steps, max(args.warmup, 0)
    extras = {}

    h = Handle(cfg, "mixed", dev)
    if args.skin >= 0:
        h.set_list_skin(args.skin)
    if args.list_block >= 0:
        h.set_list_block(args.list_block)
    h.set_universe(u)
    if args.variant >= 0:
        h.set_kernel_variant(args.variant)
        variant, tune_ms = args.variant, {}
    else:
        variant, tune_ms = h.autotune(reps=3)  # picks the pair-pass work shape; state unchanged
    tick = run_ticks(h, wl, cfg, Wm, 0)
    h.synchronize()
    dist.barrier()
    rb0 = h.list_rebuilds()  # synchronises
    clocks = Clocks(dev)
    clocks.start()
    l0 = h.launches
    h.mark(0)
    tick = run_ticks(h, wl, cfg, K, tick)  # the reference's full tick: K, V and pairs every tick
    h.mark(1)
    ms = h.elapsed_ms(0, 1)
    clk = clocks.stop()
    h.synchronize()
    rebuilds = h.list_rebuilds() - rb0  # also counts the kernels of the rebuilds that ran
    launches = h.launches - l0
    dist.barrier()
    ms_max = dist.max(ms)
    value = dist.world * u.n * K / (ms_max * 1e-3)
    # the same ticks with the energy-free pair pass (nothing recorded)
    h.mark(2)
    tick = run_ticks(h, wl, cfg, K, tick, record=False)
    h.mark(3)
    ms_nov = dist.max(h.elapsed_ms(2, 3))

    # per-kernel device times over a profiled pass of the same (recording,
    # eagerly launched) ticks; the in-cutoff pair count from one recorded tick
    pairs = float(h.step(1, stats=True)["pairs"][0])
    h.profile(True)
    h.step(min(K, 50), stats=True)
    prof = h.profile_read(reset=True)
    # the rebuild kernels timed on ticks that each rebuild (setting the skin
    # again forces one), so that no launch of them returns at the rebuild gate
    skin_now, _ = h.list_config()
    n_rb = 8
    rbp0 = h.list_rebuilds()
    for _ in range(n_rb):
        h.set_list_skin(skin_now)
        h.step(1, stats=True)
    rb_ran = h.list_rebuilds() - rbp0
    prof_rb = h.profile_read(reset=True)
    h.profile(False)
    entries, overflowed = h.list_stats()
    force_k = "force_nl" if "force_nl" in prof else "force_mixed"
    f_launch, f_ms = prof.get(force_k, (1, float("nan")))
    force_ms_eager = f_ms / max(f_launch, 1)
    tot_ms = sum(v[1] for k, v in prof.items() if k != "nl_rebuild")
    # the pair pass as the timed ticks run it: two events captured into the
    # replayed tick around the pass (external event nodes), 40 recording ticks
    # (the state keeps condensing, so the tick time, the pair count and the
    # pass time are all taken on these ticks, the pairs from their records)
    h.step(5, stats=True, graph=True)
    h.mark(4)
    h.step(40, stats=True, graph=True)
    h.mark(5)
    tick_ms_here = h.elapsed_ms(4, 5) / 40
    h.set_pass_timing(True)
    pass_ms, pass_pairs = [], []
    for _ in range(40):
        pass_pairs.append(float(h.step(1, stats=True, graph=True)["pairs"][0]))
        pass_ms.append(h.pass_ms())
    h.set_pass_timing(False)
    force_ms = float(np.median(pass_ms))
    pairs = float(np.mean(pass_pairs))
    flop_pp = FLOP_PER_PAIR_LJC if cfg.enable_electrostatics else FLOP_PER_PAIR_LJ
    achieved = pairs * flop_pp / (force_ms * 1e-3) / 1e12
    try:
        peak = _lib.measure_fp32_peak(dev)
        peak_src = "measured: FP32 FMA loop on all SMs (gx_measure_fp32_peak)"
    except Exception as e:  # noqa: BLE001
        peak, peak_src = 74.4, f"nominal 148 SM x 128 lanes x 2 x 1.965 GHz ({e})"
    traffic = ncu_traffic(force_k)
    l1 = ncu_figure("l1tex_throughput_frac", force_k)
    roof = {"kernel": force_k, "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
            "limiter": None if l1 is None else {
                "unit": "L1/TEX throughput, fraction of peak (ncu)", "frac": l1,
                "note": "the pass is bound by its neighbour gathers and far-end integer reductions in L1/TEX, "
                        "not by the FP32 pipe (profiles/k_nl_force__c3_262144_atoms.txt)"},
            "flop_per_launch": pairs * flop_pp, "flop_per_pair": flop_pp, "pairs_per_launch": pairs,
            "launch_ms": force_ms, "share_of_step": force_ms / tick_ms_here, "tick_ms_at_these_ticks": tick_ms_here,
            "launch_ms_min_max": [float(np.min(pass_ms)), float(np.max(pass_ms))],
            "launch_ms_eager": force_ms_eager, "share_of_eager_step": f_ms / tot_ms if tot_ms else None,
            "timing": "median over 40 recording graph ticks of CUDA events captured into the tick around the "
                      "energy-carrying pass (gx_set_pass_timing), after the timed, energy-free and profiled "
                      "ticks (the quench has condensed further by then: more pairs than in the timed ticks), "
                      "pairs from those ticks' records, share against 40 graph ticks just before them; "
                      "launch_ms_eager: events around each launch of the profiled eager ticks"}
    hbm, hbm_src = hbm_peak()
    epa = entries / u.n if u.n else 0.0
    mem = {}
    for src, keys in ((prof, ("nl_advance", "nl_finish", "kick", "drift", "wrap", "kinetic", "stage_pos4")),
                      (prof_rb, REBUILD_KERNELS)):
        for k in keys:
            if k not in src or not src[k][0]:
                continue
            nl, kms = src[k]
            bpa = list_build_bytes_per_atom(epa) if k == "nl_build" else BYTES_PER_ATOM.get(k, 0)
            if not bpa:
                continue
            gbs = bpa * u.n / (kms / nl * 1e-3) / 1e9
            mem[k] = {"launch_ms": kms / nl, "bytes_per_atom": bpa, "GB/s": gbs, "frac": gbs / hbm if hbm else None,
                      "launches": "every tick" if src is prof else "rebuild ticks only (each timed launch ran)"}
    every = {k: v for k, v in mem.items() if v["launches"] == "every tick"}
    top_mem = max(every.items(), key=lambda kv: kv[1]["launch_ms"]) if every else None
    roof_hbm = None
    if top_mem:
        roof_hbm = {"kernel": top_mem[0], "bound": "hbm", "achieved": top_mem[1]["GB/s"], "peak": hbm,
                    "unit": "GB/s", "frac": top_mem[1]["frac"], "peak_source": hbm_src,
                    "traffic": ncu_traffic(top_mem[0])}
    roof_rebuild = None
    if "nl_rebuild" in prof_rb and rb_ran:
        rb_ms = prof_rb["nl_rebuild"][1] / max(prof_rb["nl_rebuild"][0], 1)
        rb_bytes = sum(v["bytes_per_atom"] for k, v in mem.items() if k in REBUILD_KERNELS) * u.n
        roof_rebuild = {"kernel": "nl_rebuild (the whole rebuild: keys, sort, reorder, copy, staging, list build)",
                        "bound": "hbm", "achieved": rb_bytes / (rb_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                        "frac": rb_bytes / (rb_ms * 1e-3) / 1e9 / hbm, "peak_source": hbm_src, "ms": rb_ms,
                        "algorithmic_bytes": rb_bytes, "rebuilds_timed": int(rb_ran),
                        "list_entries_per_atom": epa, "overflowed_atoms": int(overflowed)}
    kernels = {k: {"launches": v[0], "ms": v[1], "share": v[1] / tot_ms if tot_ms else None}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1]) if k != "nl_rebuild"}

    if not args.no_extras:
        # plain FP64 GPU path on the same state
        try:
            pos, vel, acc = h.get_state()
            h64 = Handle(cfg, "fp64", dev)
            h64.set_state(pos, vel, u.elem, acc=acc, charge=u.charge, mass=u.mass, entity=u.entity)
            K64 = max(10, min(K, 60))
            run_ticks(h64, wl, cfg, 3, tick)
            h64.synchronize()
            h64.mark(0)
            run_ticks(h64, wl, cfg, K64, tick + 3)
            h64.mark(1)
            ms64 = dist.max(h64.elapsed_ms(0, 1))
            v64 = dist.world * u.n * K64 / (ms64 * 1e-3)
            # force accuracy of the mixed pass against the FP64 pass (which
            # matches the oracle to 1e-12) on one state
            hm = Handle(cfg, "mixed", dev)
            pos, vel, acc = h64.get_state()
            hm.set_state(pos, vel, u.elem, charge=u.charge, mass=u.mass, entity=u.entity)
            h64.set_state(pos, vel, u.elem, charge=u.charge, mass=u.mass, entity=u.entity)
            Vm, _, _ = hm.forces()
            V64, _, _ = h64.forces()
            am = hm.get_state()[2]
            a64 = h64.get_state()[2]
            rel = float(np.linalg.norm(am - a64) / np.linalg.norm(a64))
            # the FP64 pair pass against the FP64 pipe: each unique in-cutoff
            # pair's algorithmic FLOPs (the same count as the mixed pass) over
            # the pass time (the full list visits every pair from both ends)
            h64.set_state(pos, vel, u.elem, acc=acc, charge=u.charge, mass=u.mass, entity=u.entity)
            h64.step(2, stats=True)
            h64.profile(True)
            pairs64 = float(h64.step(10, stats=True)["pairs"].mean())
            p64 = h64.profile_read(reset=True)
            h64.profile(False)
            k64 = "force_nl" if "force_nl" in p64 else "force_f64"
            nl64, t64 = p64.get(k64, (1, float("nan")))
            pass64_ms = t64 / max(nl64, 1)
            try:
                peak64 = _lib.measure_fp64_peak(dev)
                peak64_src = "measured: FP64 FMA loop on all SMs (gx_measure_fp64_peak)"
            except Exception as e:  # noqa: BLE001
                peak64, peak64_src = 37.0, f"nominal ({e})"
            ach64 = pairs64 * flop_pp / (pass64_ms * 1e-3) / 1e12
            extras["fp64"] = {"value": v64, "ms_per_step": ms64 / K64, "steps": K64,
                              "mixed_over_fp64": value / v64,
                              "tick": "the same tick on the plain FP64 path: the persistent full neighbour list, "
                                      "the reference's FP64 per-pair arithmetic (k_nl_force64)",
                              "roofline": {"kernel": k64, "bound": "fp64", "achieved": ach64, "peak": peak64,
                                           "unit": "TFLOP/s", "frac": ach64 / peak64, "peak_source": peak64_src,
                                           "launch_ms": pass64_ms, "flop_per_pair": flop_pp}}
            extras["force_rel_rms_vs_fp64"] = rel
            extras["potential_rel_err_vs_fp64"] = abs(Vm - V64) / abs(V64)
            hm.close()
            h64.close()
        except Exception as e:  # noqa: BLE001
            extras["fp64_error"] = repr(e)

        # end to end through the C ABI: host ECS columns synced every tick
        try:
            import torch

            n = u.n
            pin = [torch.empty((n, 3), dtype=torch.float64, pin_memory=True) for _ in range(3)]
            arr = [p.numpy() for p in pin]
            pos, vel, acc = h.get_state()
            arr[0][:] = pos
            arr[1][:] = vel
            arr[2][:] = acc
            Ke = max(5, min(K, 20))
            he = Handle(cfg, "mixed", dev)
            he.set_state(arr[0], arr[1], u.elem, acc=arr[2], charge=u.charge, mass=u.mass, entity=u.entity)
            he.step(2)
            he.tick_host(arr[0], arr[1], arr[2])  # the first call allocates its staging
            he.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            for _ in range(Ke):
                stt = he.tick_host(arr[0], arr[1], arr[2])
            he.synchronize()
            te = time.perf_counter() - t0
            te = dist.max(te)
            extras["e2e"] = {"value": dist.world * n * Ke / te, "unit": UNIT,
                             "h2d_bytes_per_step": 3 * n * 24, "d2h_bytes_per_step": 3 * n * 24 + stt.nbytes,
                             "steps": Ke, "timing": "host wall clock, pinned host buffers, one gx_tick_host per "
                             "tick (Position, Velocity, Acceleration in and out, copies overlapped with the tick)"}
            # the same ticks through the three separate calls a host system could make
            dist.barrier()
            t0 = time.perf_counter()
            for _ in range(Ke):
                he.set_dynamic(arr[0], arr[1], arr[2])
                stt = he.step(1, stats=True)
                he.get_state_into(arr[0], arr[1], arr[2])
            he.synchronize()
            t3 = dist.max(time.perf_counter() - t0)
            extras["e2e_three_calls"] = {"value": dist.world * n * Ke / t3, "unit": UNIT, "steps": Ke,
                                         "timing": "host wall clock, pinned host buffers, gx_set_dynamic + "
                                         "gx_step(1) + gx_get_state every tick (no overlap)"}
            he.close()
        except Exception as e:  # noqa: BLE001
            extras["e2e_error"] = repr(e)

        # g(r) of the resident state: the reference's subsampled call and the whole state
        try:
            extras["gr"] = gr_leg(h, u.n)
        except Exception as e:  # noqa: BLE001
            extras["gr_error"] = repr(e)

        # the structure lenses (FoF, bound pairs) on the resident state
        try:
            extras["lenses"] = lens_leg(h, cfg.bond_k_bind)
        except Exception as e:  # noqa: BLE001
            extras["lenses_error"] = repr(e)

        # XYZ frame export of the resident state (export::write_frame)
        try:
            extras["xyz_frame"] = xyz_leg(h, u.elem, tick, cpu=dist.rank == 0 and dist.world == 1)
        except Exception as e:  # noqa: BLE001
            extras["xyz_frame_error"] = repr(e)

        # batched temperature sweep: replica-steps/s in one persistent launch vs
        # the same replicas one after another through gx_step
        try:
            from genesis_b200 import sweep

            # one sweep of 256 replicas shared over the ranks (size-balanced,
            # no collective until the per-replica results are gathered)
            wls = sweep.make_replicas(256, seed=0)
            sizes = [wl.n_atoms for wl in wls]
            parts = sweep.partition(sizes, dist.world)
            mine = [wls[i] for i in parts[dist.rank]]
            sweep_steps = 2000
            _, stb, msb = sweep.run_batched(mine, sweep_steps, dev, mode=2)
            _, _, msp = sweep.run_batched(mine, sweep_steps, dev, mode=1)
            _, stc, msc = sweep.run_batched(mine, sweep_steps, dev, mode=3)
            _, stl, msl = sweep.run_batched(mine, sweep_steps, dev, mode=4)
            seq_steps = 50
            _, mss = sweep.run_sequential(mine, seq_steps, dev)
            msb, msp, msc, msl, mss = dist.max(msb), dist.max(msp), dist.max(msc), dist.max(msl), dist.max(mss)
            vb = len(wls) * sweep_steps / (msb * 1e-3)
            vp = len(wls) * sweep_steps / (msp * 1e-3)
            vc = len(wls) * sweep_steps / (msc * 1e-3)
            vl = len(wls) * sweep_steps / (msl * 1e-3)
            vs = len(wls) * seq_steps / (mss * 1e-3)
            stats = sweep.assemble(parts, dist.all_gather_object(np.asarray(stl if vl >= vb else stb).tolist()))
            best = max(vb, vp, vc, vl)
            mode_name = {vb: "all-replica graph", vp: "persistent launch, a CTA per replica",
                         vc: "persistent cooperative launch", vl: "all-replica graph over neighbour lists"}[best]
            extras["replica_sweep"] = {
                "metric": "replica-steps/s", "replicas": len(wls), "atoms": sweep.atoms(wls),
                "scaling": "strong: one sweep shared over the ranks",
                "atoms_per_rank": [int(sum(sizes[i] for i in p)) for p in parts],
                "batched": {"value": best, "steps": sweep_steps, "mode": mode_name,
                            "all_replica_graph": {"value": vb, "ms": msb},
                            "persistent_launch": {"value": vp, "ms": msp},
                            "persistent_cooperative_launch": {"value": vc, "ms": msc,
                                                              "same_bits_as_graph": bool(np.array_equal(stb, stc))},
                            "neighbour_lists": {"value": vl, "ms": msl,
                                                "note": "the same pairs in the list grid's frame: the last FP32 "
                                                        "bits differ from the graph mode's, and over 2,000 chaotic "
                                                        "ticks the trajectories decorrelate; the thermostatted "
                                                        "kinetic energies agree to within their fluctuations",
                                                "final_kinetic_max_rel_dev_from_graph": float(
                                                    np.max(np.abs(np.asarray(stl)[:, 0] - np.asarray(stb)[:, 0])
                                                           / np.abs(np.asarray(stb)[:, 0])))}},
                "sequential": {"value": vs, "steps_per_replica": seq_steps, "ms": mss},
                "batched_over_sequential": best / vs,
                "final_kinetic_sum": float(stats[:, 0].sum()), "final_pairs_sum": float(stats[:, 3].sum()),
                "workload": "256 replicas, n^3 atoms with n = round(N^(1/3)) in [8, 25], N log-uniform in "
                            "[512, 16384], 10-element LJ mixture, Berendsen T uniform in [20, 120] K"}
        except Exception as e:  # noqa: BLE001
            extras["replica_sweep_error"] = repr(e)

        # adjoint (C5): gradients of <V> and of the g(r) fitting loss with
        # respect to the 10 sigma + 10 epsilon_k, against 40 central differences
        try:
            extras["accuracy"] = accuracy_leg(dev)
        except Exception as e:  # noqa: BLE001
            extras["accuracy_error"] = repr(e)
        try:
            extras["adjoint"] = adjoint_leg(dev)
        except Exception as e:  # noqa: BLE001
            extras["adjoint_error"] = repr(e)
        try:
            extras["c1"] = c1_leg(dev, cpu=dist.rank == 0 and dist.world == 1)
        except Exception as e:  # noqa: BLE001
            extras["c1_error"] = repr(e)
        try:
            extras["ionic"] = ionic_leg(dev, cpu=dist.rank == 0 and dist.world == 1)
        except Exception as e:  # noqa: BLE001
            extras["ionic_error"] = repr(e)

        if dist.rank == 0 and dist.world == 1:
            try:
                threads = os.cpu_count() or 1
                extras["cpu_baseline"] = cpu_reference(wl, cfg, u, 12.0, threads)
            except Exception as e:  # noqa: BLE001
                extras["cpu_baseline_error"] = repr(e)

    list_cfg = h.list_config()
    list_shape = h.list_shape()
    h.close()
    if dist.rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": K, "warmup": Wm,
                "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 pair arithmetic, i64 fixed-point accumulation, f64 state",
                "data": "synthetic",
                "config": {"workload": wl.name, "atoms": u.n, "precision": "mixed", "thermostat_target_K":
                           cfg.thermostat_temperature, "electrostatics": cfg.enable_electrostatics,
                           "gr_every": wl.gr_every, "l2": "inputs larger than L2 (state ~300 MB > 126 MB); no flush",
                           "parallelism": f"{dist.world} independent replicas (one per GPU)",
                           "pair_pass_variant": variant, "autotune_ms": tune_ms,
                           "neighbour_list_rebuilds_in_timed_ticks": rebuilds,
                           "neighbour_list_skin_and_threads_per_atom": list_cfg,
                           "list_pass_shape": list_shape,
                           "cuda_graph": True},
                "gpu_launches": launches, "clocks": clk, "roofline": roof, "roofline_hbm": roof_hbm,
                "roofline_rebuild": roof_rebuild,
                "tick": "the reference's tick: kick, drift, wrap, list check (rebuild when flagged), pair pass "
                        "with the potential and the in-cutoff pair count, second kick, Berendsen; K, V, lambda "
                        "and pairs recorded on the device every tick",
                "energy_free_ticks": {"value": dist.world * u.n * K / (ms_nov * 1e-3), "ms_per_step": ms_nov / K,
                                      "steps": K, "note": "the same ticks with a pair pass that leaves the "
                                      "potential and pair count out (ticks that record nothing)"},
                "kernels": kernels, "memory_kernels": mem, "pairs_per_tick": pairs}
        line.update(extras)
        if "e2e" not in line:
            line["e2e"] = None
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            reference_arm(args, dist)
        elif args.leg:
            dev = dist.local
            if args.leg == "ionic":
                out = ionic_leg(dev, cpu=False, steps=args.leg_steps or None, variant=args.variant)
            elif args.leg == "accuracy":
                out = accuracy_leg(dev, args.leg_steps or 10000)
            elif args.leg == "c1":
                out = c1_leg(dev, cpu=True, steps=args.leg_steps or 1000)
            elif args.leg == "sweep":
                from genesis_b200 import sweep

                wls = sweep.make_replicas(256, seed=0)
                steps = args.leg_steps or 2000
                mode = args.variant if args.variant in (1, 2, 3, 4) else 2
                _, _, ms = sweep.run_batched(wls, steps, dev, mode=mode)
                out = {"workload": f"256 replicas, batch mode {mode}", "steps": steps, "ms": ms,
                       "replica_steps_per_s": len(wls) * steps / (ms * 1e-3), "atoms": sweep.atoms(wls)}
            elif args.leg == "xyz":
                import dataclasses

                from genesis_b200 import workloads as W
                from genesis_b200._lib import Handle

                wl = W.C3 if args.n_side <= 0 else dataclasses.replace(W.C3, n_side=args.n_side)
                cfg, u = wl.config(), wl.generate()
                h = Handle(cfg, "mixed", dev)
                h.set_universe(u)
                h.step(2)
                out = xyz_leg(h, u.elem, 2, cpu=True)
                h.close()
            elif args.leg in ("rebuild", "gr", "fp64"):
                out = kernel_leg(args, dev)
            else:
                out = adjoint_leg(dev)
            if dist.rank == 0:
                print(json.dumps({"leg": args.leg, **out}), flush=True)
        else:
            ours_arm(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
