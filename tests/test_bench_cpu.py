"""bench.py's host-side helpers on the CPU: the whole-job arithmetic, the
roofline keys taken from the committed ncu profile, the peak fallback, and the
reference arm's JSON line (a one-step oracle run on a small slice)."""
import json
import os
import subprocess
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_replica_value_is_whole_job():
    # 4 ranks, each 1e8 tokens per step, 5 steps in 2 s on the slowest rank
    assert bench.replica_value(100_000_000, 5, 4, 2.0) == pytest.approx(1e9)


def test_roofline_profile_keys():
    mid = types.SimpleNamespace(K=1000, n_tokens=1000)
    r = bench.roofline_profile("mid", mid)
    assert r["kernel"] == "z_sweep_kernel"
    tpt = bench.measured_traffic_per_token()
    assert tpt and 10.0 < tpt < 1000.0
    assert r["traffic"] == pytest.approx(tpt * 1000)
    assert bench.roofline_profile("large_k1000", mid)["traffic"] is None
    big = types.SimpleNamespace(K=10000, n_tokens=1000)
    r = bench.roofline_profile("large_k10000", big)
    assert r["kernel"] == "z_sweep_pairs_kernel" and r["traffic"] is None


def test_peaks_measured_or_fallback():
    value, kind = bench.peaks()
    assert kind in ("measured", "fallback") and value > 1000.0
    if not os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert (value, kind) == (6650.0, "fallback")


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cpu-seconds", "1"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "gibbs_tokens_per_sec" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
