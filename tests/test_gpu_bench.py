"""bench.py's own arm end to end on a small lattice: one JSON line with the
contract's keys (the full legs run only in the default bench)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def test_bench_prints_one_contract_line(gpu):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--steps", "5", "--warmup", "3", "--n-side", "24",
                          "--no-extras"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "gpu_launches", "clocks", "roofline"):
        assert k in d, k
    assert d["value"] > 0 and d["steps"] == 5 and d["gpu_launches"] > 0
    assert d["config"]["atoms"] == 24 ** 3
    assert d["roofline"]["frac"] > 0
