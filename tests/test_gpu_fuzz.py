"""The CUDA path against the oracle on seeded random rooms (tests/fuzz_scenes.py:
random light offsets, sphere sizes and tessellations, random triangle blobs
with degenerate triangles and diffuse / mirror / glossy / glass / translucent
materials; odd seeds add a heightfield floor with per-triangle albedo), through
the C ABI:
  * photon pass with a caustic map: both photon lists bit for bit;
  * grid of each map: dims, cell, cell starts and sizes bit for bit;
  * kNN gather on 2,000 queries: neighbour id sets bit for bit, estimates
    within 1e-4;
  * a 64x48 frame with the caustic estimate: radiance within 1e-4 of the
    oracle's render, 8-bit pixels at most one level apart."""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import fuzz_scenes  # noqa: E402

RTOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return photonmap.Context(0)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("seed", range(6))
def test_random_room_matches_oracle(ctx, orc, seed):
    import photonmap
    sc = fuzz_scenes.random_scene(seed, per_triangle_albedo=seed % 2 == 1)
    ctx.set_scene(sc)
    s = orc.scene(sc)
    assert np.array_equal(ctx.scene_aabb(), s.aabb())
    ng, nc = 30_000, 3_000
    ctx.trace_photons(seed, 10, ng, nc)
    tr = s.trace_photons(seed, 10, ng, nc)
    g, c = ctx.photons(0, sorted_=False), ctx.photons(1, sorted_=False)
    for key, arr in (("g_pos", g["list_pos"]), ("g_dir", g["list_dir"]), ("g_pow", g["list_power"]),
                     ("c_pos", c["list_pos"]), ("c_dir", c["list_dir"]), ("c_pow", c["list_power"])):
        assert np.array_equal(_np(arr), tr[key]), f"seed {seed}: {key}"
    ctx.build_grid(0)
    ctx.build_grid(1)
    grids = []
    for map_id, pre in ((0, "g"), (1, "c")):
        ph = ctx.photons(map_id)
        og = orc.grid_build(tr[pre + "_pos"], tr[pre + "_pow"], tr[pre + "_dir"], s.aabb(), sub_div=ph["sub_div"])
        assert tuple(og.dims) == tuple(ph["dims"]) and np.float32(og.cell) == np.float32(ph["cell"])
        assert np.array_equal(og.starts, _np(ph["cell_starts"]).astype(np.uint32))
        assert np.array_equal(og.sizes, _np(ph["cell_sizes"]).astype(np.uint32))
        grids.append(og)
    rng = np.random.default_rng(seed)
    q = (tr["g_pos"][rng.integers(0, ng, 2000)] + rng.normal(scale=0.02, size=(2000, 3))).astype(np.float32)
    qn = rng.normal(size=(2000, 3)).astype(np.float32)
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    for k, r in ((64, 0.1), (7, 0.03)):
        ids_o, cnt_o, _, rad_o = orc.gather(grids[0], q, qn, r, k, heap_mode=False)
        rad, ids, cnt = ctx.gather(torch.from_numpy(q), torch.from_numpy(qn), k, r, want_ids=True)
        assert np.array_equal(_np(cnt), cnt_o)
        assert np.array_equal(_np(ids).astype(np.uint32), ids_o)
        np.testing.assert_allclose(_np(rad), rad_o, rtol=RTOL, atol=1e-8)
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 64, 48)
    rgb, rad = ctx.render(cam, 50, 0.1, 4, k_caustic=20, r_caustic=0.2, faithful_caustic=False)
    out = s.render(cam.as_vector(), 64, 48, grids[0], 50, 0.1, 4, c=grids[1], k_c=20, r_c=0.2,
                   faithful_caustic=False)
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)
    d = np.abs(_np(rgb).reshape(-1, 3).astype(np.int32) - out["rgb8"].astype(np.int32))
    assert d.max() <= 1
    assert ctx.status() == 0
