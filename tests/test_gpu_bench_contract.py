"""bench.py's output contract, both arms, on a short run: one JSON line each with the keys and
units the measurement contract names (the engine arm: value, e2e with its copy bytes, roofline,
clocks, launch count, CPU baseline; the reference arm: impl, cpu_baseline and e2e of its own), and
the same metric, unit and config in both."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def _run(*extra):
    env = dict(os.environ)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--steps", "3", "--warmup", "3", *extra],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_engine_and_reference_lines(cuda):
    ours = _run("--no-batch", "--cpu-rows", "64")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "gpu_launches", "clocks", "cpu_baseline"):
        assert k in ours, k
    assert ours["n_gpus"] == 1 and ours["steps"] == 3 and ours["warmup"] >= 3 and ours["higher_is_better"] is True
    assert ours["value"] > 0 and ours["ms_per_step"] > 0 and ours["gpu_launches"] > 0
    e2e = ours["e2e"]
    assert e2e["unit"] == ours["unit"] and e2e["value"] > 0
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    rf = ours["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in rf, k
    assert 0 < rf["frac"] < 1.5 and abs(rf["achieved"] / rf["peak"] - rf["frac"]) < 1e-3
    assert set(ours["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    cb = ours["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] > 0
    assert "workload" in ours["config"]

    ref = _run("--impl", "reference")
    assert ref["impl"] == "reference"
    if "unavailable" in ref:
        pytest.skip(ref["unavailable"])
    for k in ("metric", "unit", "config", "higher_is_better"):
        assert ref[k] == ours[k], k
    assert ref["value"] > 0 and ref["cpu_baseline"]["value"] == ref["value"]
    assert ref["e2e"]["value"] == ref["value"] and ref["e2e"]["unit"] == ref["unit"]
