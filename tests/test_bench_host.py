"""Host-side arithmetic of bench.py's roofline objects (no GPU): the
algorithmic bytes of the two large kernels, the live-timed achieved rate, the
DRAM traffic attached only to the workload it was captured on."""
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _inputs():
    w = {"photons": 10_000_000, "k": 64}
    sc = types.SimpleNamespace(ntri=132_620)
    bvh = {"nodes": 33_781}
    return w, sc, bvh


def test_algorithmic_bytes_and_achieved():
    import bench
    w, sc, bvh = _inputs()
    out = bench.rooflines(w, sc, bvh, nreq=1_000, paths=9_000_000, k_trace_ms=4.0, k_gather_ms=2.0, hbm=6000.0,
                          src="measured", default_workload=True)
    scene = 33_781 * 64 + 132_620 * (80 + 36)
    tr = out["k_trace"]
    assert tr["algorithmic_bytes_per_launch"] == 10_000_000 * 32 + 9_000_000 * 8 + scene
    assert tr["achieved"] == pytest.approx(tr["algorithmic_bytes_per_launch"] / 4e-3 / 1e9)
    assert tr["frac"] == pytest.approx(tr["achieved"] / 6000.0)
    ga = out["k_gather"]
    assert ga["algorithmic_bytes_per_launch"] == 1_000 * (64 * 40 + 44)
    assert ga["achieved"] == pytest.approx(ga["algorithmic_bytes_per_launch"] / 2e-3 / 1e9)
    for r in out.values():
        assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] == 6000.0
    # the dominant kernel is the one with the longer launch
    assert max(out, key=lambda k: out[k]["ms_per_launch"]) == "k_trace"


def test_traffic_only_on_the_captured_workload():
    import bench
    w, sc, bvh = _inputs()
    on = bench.rooflines(w, sc, bvh, 1_000, 9_000_000, 4.0, 2.0, 6000.0, "measured", default_workload=True)
    off = bench.rooflines(w, sc, bvh, 1_000, 9_000_000, 4.0, 2.0, 6000.0, "measured", default_workload=False)
    for k in ("k_trace", "k_gather"):
        assert on[k]["traffic"] == bench.DRAM_TRAFFIC.get(k)
        assert off[k]["traffic"] is None


def test_zero_time_gives_zero_rate():
    import bench
    w, sc, bvh = _inputs()
    out = bench.rooflines(w, sc, bvh, 0, 0, 0.0, 0.0, 6000.0, "fallback", default_workload=False)
    assert out["k_trace"]["achieved"] == 0.0 and out["k_gather"]["achieved"] == 0.0
