"""The bench.py result line: one JSON object on stdout carrying the keys a
benchmark harness reads (metric, value and timing fields, the roofline, the
end-to-end figure, the clocks, the launch count).  The reference arm runs the
reference's kernels on the host, so its contract is checked on the CPU; the
B200 arm needs a GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BASE_KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
             "vs_baseline", "dtype", "data", "config")


def _line(args, timeout):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       timeout=timeout, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _line(["--impl", "reference", "--size", "32x16x16", "--steps", "2", "--warmup", "1"], 300)
    for k in BASE_KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"] == "sphere_pack_32x16x16"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.gpu
def test_b200_arm_line():
    d = _line(["--size", "64x32x32", "--steps", "3", "--warmup", "3", "--no-cpu-baseline", "--no-reference-cuda",
               "--no-batch"], 900)
    for k in BASE_KEYS:
        assert k in d, k
    assert d["value"] > 0 and d["steps"] == 3 and d["warmup"] == 3 and d["dtype"] == "f32"
    r = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["achieved"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    assert r["pattern_copy"]["achieved"] > 0
    e = d["e2e"]
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in e, k
    assert e["value"] > 0 and e["d2h_bytes_per_step"] > 0 and len(e["runs_mlups"]) == 3
    assert d["gpu_launches"] == 3   # one fused launch per step
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    assert set(d["forms"]) == {"f16", "bf16", "f16q", "f64"}
    for form in d["forms"].values():
        # the default kernel of every form: one cell per thread on the natural layout
        assert form["layout"] == "natural" and form["kernel"] == "k_coupled_step"
        assert form["roofline"]["achieved"] > 0 and form["pattern_copy"]["achieved"] > 0
