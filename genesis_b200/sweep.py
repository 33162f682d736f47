"""The batched temperature sweep (replicas of uneven size, one launch) and
its sequential counterpart, used by bench.py and the tests.

The reference runs the sweep one universe after another
(examples/temperature_sweep.rs:70-113); :func:`run_batched` advances all
replicas together with gx_batch_step, :func:`run_sequential` runs the same
replicas one after another through gx_step (CUDA-graph replay).
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W
from ._lib import Batch, Handle


def make_replicas(count: int = 256, seed: int = 0):
    return [W.replica_workload(r) for r in W.sweep_replicas(count, seed)]


def run_batched(wls, steps: int, device: int = 0, mode: int = 2):
    """Returns (replica-steps/s from the step call's CUDA-event time, stats,
    ms).  mode 1: one persistent launch, one CTA per replica; mode 2: every
    phase as one kernel over all replicas, CUDA-graph replay; mode 3: mode
    2's phases in one persistent cooperative launch; mode 4: mode 2 over
    persistent neighbour lists."""
    base = wls[0].config()
    b = Batch(base, [wl.config().size for wl in wls], [wl.thermostat_temperature for wl in wls], device)
    b.set_mode(mode)
    b.set_universes([wl.generate() for wl in wls])
    b.step(2)  # warm-up (and, in mode 2, graph capture)
    st, ms = b.step(steps)
    b.close()
    return len(wls) * steps / (ms * 1e-3), st, ms


def run_sequential(wls, steps: int, device: int = 0):
    """Each replica through its own gx_handle, one after another; device time
    per replica from stream-ordered CUDA events.  Returns (replica-steps/s, ms)."""
    total_ms = 0.0
    for wl in wls:
        h = Handle(wl.config(), "mixed", device)
        h.set_universe(wl.generate())
        h.step(2, stats=False, graph=True)
        h.mark(0)
        h.step(steps, stats=False, graph=True)
        h.mark(1)
        total_ms += h.elapsed_ms(0, 1)
        h.close()
    return len(wls) * steps / (total_ms * 1e-3), total_ms


def atoms(wls) -> int:
    return int(sum(wl.n_atoms for wl in wls))


def partition(sizes, world: int) -> list[list[int]]:
    """Shards a sweep over `world` GPUs: replicas are independent, so each
    rank advances its own share in one gx_batch with no collective on the
    data path.  Size-balanced greedy packing: the largest replica first,
    each to the rank with the fewest atoms so far (ties to the lower rank).
    Returns each rank's replica indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda r: (loads[r], r))
        parts[r].append(i)
        loads[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def assemble(parts: list[list[int]], per_rank_stats: list) -> np.ndarray:
    """Puts the per-replica rows each rank returned (in its partition's
    order) back into the sweep's replica order."""
    n = sum(len(p) for p in parts)
    rows = [np.asarray(s) for s in per_rank_stats]
    width = next((r.shape[1] for r in rows if r.size), 0)
    out = np.zeros((n, width))
    seen = np.zeros(n, dtype=bool)
    for idx, r in zip(parts, rows):
        if len(idx) != len(r):
            raise ValueError("a rank returned a different number of replicas than it was given")
        for k, i in enumerate(idx):
            if seen[i]:
                raise ValueError(f"replica {i} returned twice")
            seen[i] = True
            out[i] = r[k]
    if not seen.all():
        raise ValueError("replicas missing from the gathered results")
    return out
