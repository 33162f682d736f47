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
    phase as one kernel over all replicas, CUDA-graph replay."""
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
