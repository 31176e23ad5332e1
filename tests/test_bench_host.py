"""Host-side arithmetic of bench.py's roofline objects (no GPU): the tracer's
flops from its counted work, the gather's algorithmic bytes, the live-timed
achieved rates, the DRAM traffic attached only to the workload it was
captured on."""
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


WORK = (9_000_000, 30_000_000, 900_000_000, 2_000_000_000)   # paths, rays, node visits, triangle tests


def test_algorithmic_bytes_and_achieved():
    import bench
    w, sc, bvh = _inputs()
    out = bench.rooflines(w, sc, bvh, nreq=1_000, paths=9_000_000, k_trace_ms=4.0, k_gather_ms=2.0, work=WORK,
                          hbm=6000.0, src="measured", default_workload=True)
    tr = out["k_trace"]
    flop = 2 * 20 * 900_000_000 + 86 * 2_000_000_000
    assert tr["flop_per_launch"] == flop and tr["bound"] == "fp32" and tr["unit"] == "TFLOP/s"
    assert tr["achieved"] == pytest.approx(flop / 4e-3 / 1e12)
    assert tr["peak"] == pytest.approx(148 * 128 * 2 * 1.965e9 / 1e12)
    assert tr["frac"] == pytest.approx(tr["achieved"] / tr["peak"])
    assert tr["mrays_per_s"] == pytest.approx(30_000_000 / 4e-3 / 1e6)
    scene = 33_781 * 64 + 132_620 * (80 + 36)
    assert tr["hbm_view"]["algorithmic_bytes_per_launch"] == 10_000_000 * 32 + 9_000_000 * 8 + scene
    ga = out["k_gather"]
    assert ga["algorithmic_bytes_per_launch"] == 1_000 * (64 * 28 + 24)
    assert ga["achieved"] == pytest.approx(ga["algorithmic_bytes_per_launch"] / 2e-3 / 1e9)
    assert ga["bound"] == "hbm" and ga["unit"] == "GB/s" and ga["peak"] == 6000.0
    # the dominant kernel is the one with the longer launch
    assert max(out, key=lambda k: out[k]["ms_per_launch"]) == "k_trace"


def test_traffic_only_on_the_captured_workload():
    import bench
    w, sc, bvh = _inputs()
    on = bench.rooflines(w, sc, bvh, 1_000, 9_000_000, 4.0, 2.0, WORK, 6000.0, "measured", default_workload=True)
    off = bench.rooflines(w, sc, bvh, 1_000, 9_000_000, 4.0, 2.0, WORK, 6000.0, "measured", default_workload=False)
    for k in ("k_trace", "k_gather"):
        assert on[k]["traffic"] == bench.DRAM_TRAFFIC.get(k) and on[k]["traffic_source"]
        assert off[k]["traffic"] is None


def test_zero_time_gives_zero_rate():
    import bench
    w, sc, bvh = _inputs()
    out = bench.rooflines(w, sc, bvh, 0, 0, 0.0, 0.0, (0, 0, 0, 0), 6000.0, "fallback", default_workload=False)
    assert out["k_trace"]["achieved"] == 0.0 and out["k_gather"]["achieved"] == 0.0


def test_reference_arm_times_its_sample(monkeypatch):
    """The reference arm (CPU, no GPU): one step is a bounded sample whose own
    wall time is ms_per_step; value is the workload's Mphotons/s scaled from
    it, and the photon pass is scaled by the sample's exact path count."""
    import bench
    from oracle import REF_SO
    if not os.path.exists(REF_SO):
        pytest.skip("reference host harness not built")
    from photonmap import scenes
    sc, cs, w = scenes.workload("cornell_small")
    monkeypatch.setattr(scenes, "workload", lambda name: (sc, cs, w))
    monkeypatch.setenv("RANK", "0")
    args = types.SimpleNamespace(workload="cornell_small", steps=1, warmup=0, gpus=1)
    line = bench.run_reference(args)
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "reference"
    assert line["value"] == pytest.approx(w["photons"] / (line["ms_per_frame_estimated"] / 1e3) / 1e6)
    assert 0 < line["ms_per_step"] < 600_000
    assert "paths [0, 16384)" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
