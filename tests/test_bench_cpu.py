"""bench.py pieces that run without a GPU: the algorithmic bytes behind the
roofline figure, the clock sampler's fallback, and the reference arm (the
oracle's OpenMP step on the host cores), whose JSON line must carry the keys
the measurement contract names."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_stage_launch_bytes():
    n, nx, ny, nz = 1000, 8, 8, 8
    gh = nx * ny * (nz + 3)
    # plain: stage 1 reads 19 and writes 22 FP64 attributes, stages 2-5 read 29
    assert bench.stage_launch_bytes(n, nx, ny, nz, "plain", later_only=True) == 408 * n + 128 * gh
    assert bench.stage_launch_bytes(n, nx, ny, nz, "plain") == pytest.approx((328 + 4 * 408) / 5 * n + 128 * gh)
    # mixed: FP64 position, volume, delta_pos; FP32 the rest; FP32 records
    assert bench.stage_launch_bytes(n, nx, ny, nz, "mixed", later_only=True) == 256 * n + 64 * gh
    assert bench.stage_launch_bytes(n, nx, ny, nz, "mixed") == pytest.approx((208 + 4 * 256) / 5 * n + 64 * gh)


def test_step_roofline():
    r = bench.step_roofline(4.0e8, "plain", 6554.2, "measured")
    assert r["achieved"] == pytest.approx(4.0e8 * 2700 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6554.2)
    assert bench.step_roofline(5.0e8, "mixed", 6554.2, "measured")["bytes_per_parcel_step"] == 1740


def test_clock_sampler_without_gpu():
    c = bench.ClockSampler(0)
    c.start()
    out = c.stop()
    assert set(out) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert isinstance(out["reasons"], list)


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--no-full-check"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["unit"] == bench.UNIT and line["metric"] == bench.METRIC
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
