"""bench.py's output contract on a small workload: both arms print one JSON
line with every key the benchmark driver reads, with sane values."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--n", "64", "--rays", "20000", "--steps", "3", "--warmup", "3", "--serving-requests", "40",
         "--cpu-seconds", "1"]


def _run(extra):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + SMALL + extra, cwd=ROOT,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def test_sloth_arm_line():
    d = _run([])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and "workload" in d["config"]
    r = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert r["bound"] == "fp32_pipe" and r["achieved"] > 0 and r["peak"] > 0 and 0 < r["frac"] < 1.5
    assert r["hbm"]["peak_gbs"] > 0
    c = d["cpu_baseline"]
    assert c["value"] > 0 and c["cores"] >= 1 and c["kind"] in ("port", "reference") and c["sample"]
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] == 4 * 3          # keys, scan, scatter, trace per timed step
    assert d["clocks"] is None or "sm_mhz" in d["clocks"]
    assert d["serving"]["requests"] == 40 and d["serving"]["p99_ms"] >= d["serving"]["p50_ms"]
    assert d["adjoint"]["grad_vs_fd"]["max_abs_err_rel_to_max"] < 1e-2
    assert d["diagnostics"]["ms"] > 0
    assert d["fp32_vs_fp64"]["position_rel_L_max"] < 1e-6
    assert d["config"]["field_samples_per_ray_step"] == 3 and d["rk4"]["field_samples_per_ray_step"] == 4
    assert d["rk4"]["fp32_vs_fp64"]["position_rel_L_max"] < 1e-6


def test_reference_arm_line():
    d = _run(["--impl", "reference"])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "ray-steps/s"
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
