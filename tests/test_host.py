"""Host-side logic on the CPU: config reader, pair tracker, persistence
threshold, generator, the C-ABI library's exported symbols and struct layout
(no device calls)."""
from __future__ import annotations

import ctypes
import json
import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from genesis_b200 import config as G
from genesis_b200 import elements as E
from genesis_b200 import synth
from genesis_b200 import workloads as W

ROOT = Path(__file__).resolve().parent.parent
CASES = {c["id"]: c for c in json.loads((ROOT / "tests/golden/reference_known_answers.json").read_text())["cases"]}

BASE = """
[universe]
name = "t"
size = { x = 10.0, y = 10.0, z = 10.0 }
dt = 0.02
initial_atoms = 100
stats_history = 256
[rng]
seed = 1
[physics]
initial_temperature = 300.0
speed_limit = 1000.0
"""


# ---------------------------------------------------------------- config (src/config/mod.rs:456-605)


def test_config_requires_mandatory_fields():
    with pytest.raises(G.ConfigError):
        G.from_toml(BASE)  # gravity_constant missing (config/mod.rs:484-504)


def test_config_partial_optional_knobs():
    c = G.from_toml(BASE + "gravity_constant = 6.674e-11\n[systems]\nenable_electrostatics = true\n"
                    "enable_bond_observation = true\nenable_bond_interaction = true\n")
    assert c.enable_electrostatics and c.enable_bond_observation and c.enable_bond_interaction
    assert c.coulomb_constant == 1.0 and c.bond_min_periods == 10.0 and c.thermostat_tau == 20.0


def test_config_invalid_toml_is_an_error():
    with pytest.raises(G.ConfigError):
        G.from_toml("this is not [valid toml\n")


def test_config_reads_reference_style_file(tmp_path):
    text = BASE + """gravity_constant = 6.674e-11
thermostat_temperature = 80.0
[physics.elements]
Na = { sigma = 2.2, epsilon_k = 130.0, charge = 1.0 }
[systems]
enable_thermostat = true
[stats]
bond_k_bind = 1.4
"""
    p = tmp_path / "u.toml"
    p.write_text(text)
    c = G.from_file(p)
    na = E.by_name("Na")
    assert c.sigma[na] == 2.2 and c.epsilon_k[na] == 130.0 and c.charge[na] == 1.0
    assert c.thermostat_temperature == 80.0 and c.enable_thermostat and c.bond_k_bind == 1.4


def test_config_partial_affinity_override_stays_partial():
    # affinity_table_parses_and_roundtrips (config/mod.rs:536-573): O sets only
    # its charge, so its sigma and epsilon stay the built-in ones
    c = G.from_toml(BASE + "gravity_constant = 6.674e-11\n[physics.elements]\n"
                    "Na = { sigma = 2.2, epsilon_k = 130.0, charge = 1.0 }\nO = { charge = -2.0 }\n"
                    "[systems]\nenable_electrostatics = true\n")
    o, na = E.by_name("O"), E.by_name("Na")
    assert c.charge[o] == -2.0
    assert c.sigma[o] == E.SIGMA[o] and c.epsilon_k[o] == E.EPSILON_K[o]
    assert (c.sigma[na], c.epsilon_k[na], c.charge[na]) == (2.2, 130.0, 1.0)


def test_config_unknown_affinity_symbol_is_named_in_the_error():
    # affinity_table_with_unknown_symbol_is_rejected (config/mod.rs:575-605)
    with pytest.raises(G.ConfigError, match="Faux"):
        G.from_toml(BASE + "gravity_constant = 6.674e-11\n[physics.elements]\nFaux = { charge = -2.0 }\n"
                    "[systems]\nenable_electrostatics = true\n")


def test_element_names():
    assert E.by_name("Na") == 5 and E.by_name("Sodium") == 5 and E.by_name("sodium") == 5
    assert E.by_name("Xx") is None


# ---------------------------------------------------------------- tracker and persistence


def test_bond_debounce_constant():
    assert E.DEBOUNCE == 2  # src/systems/bonds.rs:27


# ---------------------------------------------------------------- generator


def test_generator_is_deterministic_and_momentum_free():
    a = W.C1.scaled(8).generate()
    b = W.C1.scaled(8).generate()
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel) and np.array_equal(a.elem, b.elem)
    p = (a.vel * a.mass[:, None]).sum(0)
    assert np.abs(p).max() < 1e-9
    c = W.C1.scaled(8).generate(salt=1)
    assert not np.array_equal(a.pos, c.pos)


def test_generator_shapes_and_species():
    u = W.C2.scaled(10).generate()
    assert u.n == 1000
    na, o = E.by_name("Na"), E.by_name("O")
    assert set(np.unique(u.elem)) == {na, o} and (u.elem == na).sum() == 500
    assert np.all(u.charge[u.elem == na] == 1.0) and np.all(u.charge[u.elem == o] == -1.0)
    s = 1.2 * max(E.SIGMA)
    assert abs(W.C1.config().size[0] - 16 * s) < 1e-12
    # sites (i + 1/2) s - L/2 plus 2% Gaussian jitter stay within a few sigma of the site
    L = 10 * s
    site = (np.floor((u.pos + L / 2) / s) + 0.5) * s - L / 2
    assert np.abs(u.pos - site).max() < 0.2 * s


def test_xoshiro_reference_vector():
    # xoshiro256++ published algorithm: a state of (1, 2, 3, 4) yields 41943041 first.
    st = synth.AtomStreams(0, 1)
    st.s = [np.array([1], dtype=np.uint64), np.array([2], dtype=np.uint64), np.array([3], dtype=np.uint64),
            np.array([4], dtype=np.uint64)]
    assert int(st.next_u64()[0]) == 41943041


def test_sweep_replicas_shape():
    reps = W.sweep_replicas(256)
    assert len(reps) == 256
    assert all(8 <= r.n_side <= 25 and 20.0 <= r.temperature <= 120.0 for r in reps)


# ---------------------------------------------------------------- the C-ABI library (no GPU calls)


def _header_symbols():
    text = (ROOT / "include" / "genesis_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(gx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from genesis_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from genesis_b200.build import build
        build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    syms = _header_symbols()
    assert len(syms) >= 30
    for s in syms:
        getattr(lib, s)
    assert set(_lib.EXPORTS) <= set(syms)


def test_params_layout_matches_header():
    from genesis_b200._lib import GxAdjointSpec, GxBondObservation, GxParams, GxTickStats
    src = """
#include <stddef.h>
#include <stdio.h>
#include "genesis_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(gx_params), offsetof(gx_params, enable_electrostatics),
         offsetof(gx_params, precision), offsetof(gx_params, device), sizeof(gx_tick_stats),
         offsetof(gx_tick_stats, pairs));
  printf("%zu %zu %zu\\n", sizeof(gx_adjoint_spec), offsetof(gx_adjoint_spec, gr_rmax),
         offsetof(gx_adjoint_spec, gr_support));
  printf("%zu %zu %zu\\n", sizeof(gx_bond_observation), offsetof(gx_bond_observation, lifetime_sum_ticks),
         offsetof(gx_bond_observation, species_matrix));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "l.c"
        c.write_text(src)
        exe = Path(d) / "l"
        subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(c), "-o", str(exe)], check=True)
        got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(GxParams), GxParams.enable_electrostatics.offset, GxParams.precision.offset,
            GxParams.device.offset, ctypes.sizeof(GxTickStats), GxTickStats.pairs.offset,
            ctypes.sizeof(GxAdjointSpec), GxAdjointSpec.gr_rmax.offset, GxAdjointSpec.gr_support.offset,
            ctypes.sizeof(GxBondObservation), GxBondObservation.lifetime_sum_ticks.offset,
            GxBondObservation.species_matrix.offset]
    assert got == want


def test_oracle_params_layout_matches_its_header():
    from oracle.oracle import OrcParams
    src = """
#include <stddef.h>
#include <stdio.h>
#include "oracle.h"
int main(void) { printf("%zu %zu\\n", sizeof(orc_params), offsetof(orc_params, enable_boundaries)); return 0; }
"""
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "l.c"
        c.write_text(src)
        exe = Path(d) / "l"
        subprocess.run(["gcc", f"-I{ROOT / 'oracle'}", str(c), "-o", str(exe)], check=True)
        got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(OrcParams), OrcParams.enable_boundaries.offset]


def test_scheduler_counts_executions_after_the_schedule():
    """Scheduler::run adds its executions to StatsCollector.systems_run once
    the whole schedule ran (src/scheduler/mod.rs:83-89), so a system sees the
    previous ticks' count; the collector keeps a bounded history
    (src/stats/mod.rs:194-201)."""
    from genesis_b200.systems import Scheduler, StatsCollector, System, SystemContext, Time, World

    seen = []

    class Probe(System):
        def name(self):
            return "probe"

        def run(self, ctx):
            seen.append(ctx.stats.systems_run)
            ctx.stats.record({"tick": ctx.time.tick})

    class Noop(System):
        def name(self):
            return "noop"

        def run(self, ctx):
            pass

    s = Scheduler()
    s.add_system(Noop())
    s.add_system(Probe())
    z = np.zeros((0, 3))
    w = World(pos=z, vel=z, acc=z, elem=np.zeros(0, np.uint8), mass=np.zeros(0), charge=np.zeros(0),
              entity=np.zeros(0, np.uint32))
    stats = StatsCollector(history_cap=3)
    t = Time(0.1)
    for _ in range(5):
        t.advance()
        s.run(SystemContext(w, {}, t, t.dt, stats))
    assert seen == [0, 2, 4, 6, 8] and stats.systems_run == 10
    assert [h["tick"] for h in stats.history] == [3, 4, 5] and stats.snapshot["tick"] == 5
