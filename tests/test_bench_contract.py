"""bench.py's JSON line: the keys and types the benchmark contract fixes, for
the reference arm (CPU, runs here) and the engine arm (GPU)."""
import json
import os
import subprocess
import sys

import pytest
from conftest import ROOT

from oracle import oracle as O


def _run(args, timeout):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                       timeout=timeout, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref/lgf_ref not built")
def test_reference_arm_line():
    d = _run(["--impl", "reference", "--steps", "1", "--warmup", "1", "--ref-procs", "2", "--ref-shape", "8,8,8,8"],
             600)
    assert d["impl"] == "reference" and d["metric"] == "site-RK3-steps/s" and d["unit"] == "site-RK3-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.gpu
def test_engine_arm_line():
    d = _run(["--steps", "1", "--warmup", "3", "--no-forms", "--no-cpu-baseline"], 900)
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "clocks", "gpu_launches", "flow_only"):
        assert k in d, k
    assert d["metric"] == d["unit"] == "site-RK3-steps/s" and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["warmup"] >= 3 and d["value"] > 0 and d["dtype"] == "f64" and d["scaling"] == "weak"
    assert "workload" in d["config"]
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] == 48 * 24 ** 3 * 576 and e["d2h_bytes_per_step"] > 0
    r = d["roofline"]
    # the stage kernel is bound by the FP64 FMA pipe; its HBM figures sit beside
    assert r["bound"] == "fp64" and r["unit"] == "TFLOP/s"
    assert r["achieved"] > 0 and r["peak"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    h = r["hbm"]
    assert h["unit"] == "GB/s" and h["achieved"] > 0 and abs(h["frac"] - h["achieved"] / h["peak"]) < 1e-9
    assert r["traffic"] is None or r["traffic"] > 0
    assert d["gpu_launches"] == 3 * 300 + 3 * 31
    assert set(d["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
