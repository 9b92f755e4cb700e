"""bench.py's JSON line on small cases: the keys the line promises and their
consistency (throughput against time per step, roofline fractions against
their peak, the e2e block, the per-kernel bytes behind the step roofline)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + list(args), cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_two_phase_line():
    d = _line("--nx", "24", "--ny", "24", "--nz", "12", "--steps", "3", "--warmup", "3", "--no-cpu", "--no-forms")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "data", "config", "roofline", "clocks", "e2e", "gpu_launches", "solver"):
        assert k in d, k
    assert d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert abs(d["value"] * d["ms_per_step"] / 1000.0 - 1.0) < 1e-6
    assert d["gpu_launches"] > 0
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    assert 0 < r["step"]["frac"] < 1.5 and r["step"]["algorithmic_bytes_per_step"] > 0
    assert r["kernel"] and r["launches"] > 0 and r["algorithmic_bytes_per_launch"] > 0
    e = d["e2e"]
    assert e["unit"] == d["unit"] and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert 0 < e["value"] <= d["value"] * 1.05


def test_heat_line_and_kernel_profile():
    d = _line("--workload", "heat", "--nx", "32", "--ny", "32", "--steps", "3", "--warmup", "3", "--no-cpu",
              "--kernel-profile")
    assert d["metric"] == "Newton-steps/s" and d["value"] > 0
    prof = d["kernel_profile"]
    assert prof and abs(sum(v["share"] for v in prof.values()) - 1.0) < 0.01
    # every solver kernel states its algorithmic bytes
    for name in ("bicg_spmv_omega", "bilu_lower", "bilu_upper", "bicg_xr"):
        if name in prof:
            assert prof[name].get("bytes_per_launch", 0) > 0, name
