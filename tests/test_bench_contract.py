"""The JSON line of bench.py: the keys and types the benchmark contract asks
for, from the reference arm on CPU and from a small GPU run."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
BASE_KEYS = {"metric": str, "value": float, "unit": str, "n_gpus": int, "steps": int,
             "warmup": int, "ms_per_step": float, "higher_is_better": bool, "scaling": str,
             "dtype": str, "data": str, "config": dict}


def _run(args, timeout):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True,
                       text=True, timeout=timeout, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def _check_base(d):
    for k, t in BASE_KEYS.items():
        assert k in d, k
        assert isinstance(d[k], (int, float) if t is float else t), (k, d[k])
    assert "vs_baseline" in d
    assert "workload" in d["config"]


def test_reference_arm_line():
    d = _run(["--impl", "reference", "--steps", "1", "--warmup", "0"], timeout=900)
    _check_base(d)
    assert d["impl"] == "reference"
    assert d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # ms_per_step is the measured time of the timed sample, not a scaled figure
    n = d["config"]["cpu_sample_n"]
    assert abs(d["value"] * d["ms_per_step"] * 1e-3 - n ** 3) <= 1e-6 * n ** 3
    assert f"{n}^3" in cb["sample"]


def test_reference_arm_maps_no_product_library():
    """The reference arm runs the reference's own host model with inputs made on
    the oracle side: the product's shared library is never loaded."""
    code = (
        "import sys, types; sys.argv = ['bench.py']; sys.path.insert(0, '.');"
        "import bench;"
        "a = types.SimpleNamespace(warmup=0, steps=1, n=512, gpus=1);"
        "import io, contextlib; buf = io.StringIO();"
        "ctx = contextlib.redirect_stdout(buf); ctx.__enter__(); bench.run_reference(a); ctx.__exit__(None, None, None);"
        "maps = open('/proc/self/maps').read();"
        "print('PRODUCT' if 'libastaroth_b200' in maps else 'CLEAN');"
        "print('ORACLE' if 'oracle/' in maps else 'NO-ORACLE')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "CLEAN" in r.stdout and "ORACLE" in r.stdout, r.stdout


@pytest.mark.gpu
def test_gpu_line_small():
    d = _run(["--n", "64", "--steps", "2", "--warmup", "3", "--no-ensemble", "--no-cfl1024",
              "--accuracy-steps", "2"], timeout=900)
    _check_base(d)
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    c = d["clocks"]
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(c)
    assert d["cpu_baseline"]["value"] > 0
    assert d["fp32comp"]["rel_linf_vs_fp64"]["max"] <= 1e-5
    a = d["adjoint"]
    assert a["value"] > 0 and a["forward_ms"] > 0 and a["backward_ms"] > 0
