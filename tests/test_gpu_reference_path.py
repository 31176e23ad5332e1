"""The CUDA tracer against the reference's GPU path.

oracle/ref_host/ref_trace.cu's device pass compiles the reference's device
build of its tracer (CudaPhotonMapping/PhotonTracing.cu and what it calls, its
vec3 arithmetic rounded toward zero, CudaPhotonMapping/vec3.cuh:18-20) and
runs it one photon path per thread with the same injected streams.  The CUDA
tracer keeps the reference's host (CPU-mode) numerics, so the two differ by
rounding: on a path whose decisions all agree, every photon position is
within 1e-5 relative of the reference's GPU path; a rounding difference can
flip a decision (a Russian-roulette draw, a triangle edge, a rejection
sample), after which the two paths part.  The test measures both rates.
"""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import ref_cases  # noqa: E402

from oracle import REF_TRACE_SO  # noqa: E402

REL = 1e-5


def compare_paths(a, b, n):
    """Per path: the same photon counts and bounce indices (decisions agree),
    and then the largest relative position error of its photons."""
    ca, cb = np.asarray(a["counts"]).reshape(-1, 2), np.asarray(b["counts"]).reshape(-1, 2)
    same = (ca == cb).all(1)
    err = np.full(n, np.inf)
    for key, k in (("g", 0), ("c", 1)):
        oa = np.concatenate([[0], np.cumsum(ca[:, k])])
        ob = np.concatenate([[0], np.cumsum(cb[:, k])])
        pa, pb = np.asarray(a[f"{key}_pos"]), np.asarray(b[f"{key}_pos"])
        ba, bb = np.asarray(a[f"{key}_bounce"]), np.asarray(b[f"{key}_bounce"])
        for i in np.nonzero(same)[0]:
            x, y = pa[oa[i]:oa[i + 1]], pb[ob[i]:ob[i + 1]]
            if not np.array_equal(ba[oa[i]:oa[i + 1]], bb[ob[i]:ob[i + 1]]):
                same[i] = False
                continue
            e = float((np.linalg.norm(x - y, axis=1) / np.maximum(np.linalg.norm(y, axis=1), 1e-30)).max()) \
                if x.size else 0.0
            err[i] = e if not np.isfinite(err[i]) else max(err[i], e)
    err[~same] = np.inf
    return same, err


@pytest.mark.skipif(not os.path.exists(REF_TRACE_SO), reason="reference tracer harness not built (make -C oracle ref)")
@pytest.mark.parametrize("name", ["cornell_small", "stress_glass", "heightfield", "heightfield_albedo"])
def test_cuda_tracer_against_the_reference_gpu_path(name):
    import photonmap
    from oracle import RefTrace
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build, seed, cap, p0, end, sub = ref_cases.CASES[name]
    n = min(end - p0, 20_000)
    sc = build()
    rs = RefTrace().scene(sc)
    ref_gpu = rs.gpu_trace_paths(seed, cap, p0, p0 + n)
    ref_host = rs.trace_paths(seed, cap, p0, p0 + n)
    ctx = photonmap.Context(0)
    ctx.set_scene(sc)
    o = ctx.trace_paths(seed, ref_cases.MAX_BOUNCES, cap, p0, p0 + n)
    ours = {k: v.cpu().numpy() for k, v in o.items()}
    # the CUDA tracer is the reference's host path bit for bit (its bounce indices are the host path's)
    assert np.array_equal(ours["g_pos"], ref_host["g_pos"]) and np.array_equal(ours["c_pos"], ref_host["c_pos"])
    ours["g_bounce"], ours["c_bounce"] = ref_host["g_bounce"], ref_host["c_bounce"]
    same, err = compare_paths(ours, ref_gpu, n)
    within = float((err <= REL).mean())
    print(f"\n{name}: {n} paths; decisions agree on {same.mean():.4%}; photons within {REL:g} on "
          f"{within:.4%} of paths; median error of agreeing paths {np.median(err[same]):.2e}")
    assert (ref_gpu["draws"] > 0).all()
    assert same.mean() >= 0.97
    assert within >= 0.95
