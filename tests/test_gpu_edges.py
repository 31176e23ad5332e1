"""Edge cases of the CUDA path against the oracle (through the C ABI):
  * a 1x1 frame, and eye depths 0 and 1 (no specular / refraction plans);
  * k = 1 with a radius that finds nothing for most requests (zero radiance),
    and k = 256 (the largest) with a radius that leaves many requests short
    of k photons;
  * a photon map of one photon: its grid and every gather;
  * a minimal scene (the light and one diffuse triangle below it);
  * queries outside the scene box (clamped into the boundary cells, as the
    reference's hash does).
Photon lists, grids and kNN id sets bit for bit; radiance within 1e-4."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from photonmap import scenes  # noqa: E402

RTOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return photonmap.Context(0)


def _np(t):
    return t.detach().cpu().numpy()


def _frame_vs_oracle(ctx, orc, sc, W, H, k, r, depth, photons=40_000, seed=2):
    import photonmap
    ctx.set_scene(sc)
    s = orc.scene(sc)
    ctx.trace_photons(seed, 8, photons)
    ctx.build_grid(0)
    tr = s.trace_photons(seed, 8, photons)
    ph = ctx.photons(0)
    g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb(), sub_div=ph["sub_div"])
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, W, H)
    rgb, rad = ctx.render(cam, k, r, depth)
    out = s.render(cam.as_vector(), W, H, g, k, r, depth)
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)
    assert np.abs(_np(rgb).reshape(-1, 3).astype(int) - out["rgb8"].astype(int)).max() <= 1
    assert ctx.status() == 0
    return _np(rad)


@pytest.mark.parametrize("W,H,depth", [(1, 1, 4), (33, 17, 0), (33, 17, 1)])
def test_tiny_frames_and_shallow_eye_paths(ctx, orc, W, H, depth):
    sc, _, _ = scenes.workload("cornell_small")
    _frame_vs_oracle(ctx, orc, sc, W, H, 50, 0.1, depth)


def test_k1_tiny_radius_and_k256(ctx, orc):
    sc, _, _ = scenes.workload("cornell_small")
    rad = _frame_vs_oracle(ctx, orc, sc, 48, 36, 1, 1e-4, 2)
    assert (rad == 0).mean() > 0.5          # most requests find no photon within 1e-4
    _frame_vs_oracle(ctx, orc, sc, 48, 36, 256, 0.02, 2)


def test_one_photon_map(ctx, orc):
    sc, _, _ = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    s = orc.scene(sc)
    ctx.trace_photons(4, 8, 1)
    tr = s.trace_photons(4, 8, 1)
    lst = ctx.photons(0, sorted_=False)
    assert lst["count"] == 1 and np.array_equal(_np(lst["list_pos"]), tr["g_pos"])
    ctx.build_grid(0)
    ph = ctx.photons(0)
    g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb(), sub_div=ph["sub_div"])
    assert tuple(g.dims) == tuple(ph["dims"])
    assert np.array_equal(g.starts, _np(ph["cell_starts"]).astype(np.uint32))
    rng = np.random.default_rng(0)
    q = (tr["g_pos"] + rng.normal(scale=0.3, size=(256, 3))).astype(np.float32)
    qn = rng.normal(size=(256, 3)).astype(np.float32)
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    for k, r in ((1, 0.5), (8, 2.0)):
        ids_o, cnt_o, _, rad_o = orc.gather(g, q, qn, r, k, heap_mode=False)
        rad, ids, cnt = ctx.gather(torch.from_numpy(q), torch.from_numpy(qn), k, r, want_ids=True)
        assert np.array_equal(_np(cnt), cnt_o) and cnt_o.max() == 1
        assert np.array_equal(_np(ids).astype(np.uint32), ids_o)
        np.testing.assert_allclose(_np(rad), rad_o, rtol=RTOL, atol=1e-12)


def test_minimal_scene(ctx, orc):
    light = scenes._quad((-0.25, 0.999, -0.25), (0.25, 0.999, -0.25), (0.25, 0.999, 0.25), (-0.25, 0.999, 0.25),
                         (0, -1, 0))
    floor_p = np.array([[[-1, -1, -1], [0, -1, 1], [1, -1, -1]]], np.float64)
    floor_n = np.tile(np.array([0.0, 1.0, 0.0]), (1, 3, 1))
    pos = np.concatenate([floor_p, light[0]]).astype(np.float32)
    nrm = np.concatenate([floor_n, light[1]]).astype(np.float32)
    mats = np.stack([scenes.material(diffuse=(0.7, 0.7, 0.7)), scenes.material(emission=(1, 1, 1))])
    sc = scenes.Scene(pos, nrm, np.array([0, 1, 1], np.int32), mats, light_model=1,
                      light_intensity=np.ones(3, np.float32))
    _frame_vs_oracle(ctx, orc, sc, 40, 30, 20, 0.2, 4, photons=5_000)


def test_queries_outside_the_scene_box(ctx, orc):
    sc, _, _ = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    s = orc.scene(sc)
    ctx.trace_photons(6, 8, 30_000)
    ctx.build_grid(0)
    tr = s.trace_photons(6, 8, 30_000)
    ph = ctx.photons(0)
    g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb(), sub_div=ph["sub_div"])
    rng = np.random.default_rng(1)
    q = rng.uniform(-1.3, 1.3, size=(2000, 3)).astype(np.float32)   # partly outside [-1, 1]^3
    qn = rng.normal(size=(2000, 3)).astype(np.float32)
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    ids_o, cnt_o, _, rad_o = orc.gather(g, q, qn, 0.25, 32, heap_mode=False)
    rad, ids, cnt = ctx.gather(torch.from_numpy(q), torch.from_numpy(qn), 32, 0.25, want_ids=True)
    assert np.array_equal(_np(cnt), cnt_o)
    assert np.array_equal(_np(ids).astype(np.uint32), ids_o)
    np.testing.assert_allclose(_np(rad), rad_o, rtol=RTOL, atol=1e-9)
