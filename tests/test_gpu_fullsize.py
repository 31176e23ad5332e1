"""The benched frame itself against the oracle: cornell_hf_1080p at full size
(10M photons, 1920x1080, k 64, r 0.05, automatic sub-division, the frame's
Morton-ordered gather), checked on seeded samples.

  * the oracle builds its grid from the frame's 10M photons: dims, cell size,
    cell starts and sizes equal the GPU's;
  * 20,000 of the frame's kNN requests: neighbour id sets equal the oracle's
    canonical (distance, index) selection bit for bit; the estimates the frame
    used (its Morton-ordered gather) are within 1e-4 of the oracle's;
  * 8 rows of pixels (15,360): the oracle renders them over its grid; radiance
    within 1e-4 relative, 8-bit pixels at most one level apart.
The photon pass at this size is checked by its properties in
tests/test_gpu_parity.py and path by path against the oracle and the
reference's own tracer on the same scene (tests/test_tracer_pin.py)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL = 1e-4


@pytest.fixture(scope="module")
def frame():
    import photonmap
    from photonmap import scenes
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sc, cs, w = scenes.workload("cornell_hf_1080p")
    ctx = photonmap.Context(0)
    ctx.set_scene(sc)
    cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
    rgb, rad, _ = ctx.frame(w["seed"], w["max_bounces"], w["photons"], cam, w["k"], w["radius"], w["max_depth"])
    ph = ctx.photons(0)
    req = {k: v.cpu().numpy() for k, v in ctx.requests().items()}
    out = dict(ctx=ctx, sc=sc, cs=cs, w=w, cam=cam, rgb=rgb.cpu().numpy().reshape(-1, 3),
               rad=rad.cpu().numpy().reshape(-1, 3), req=req, sub_div=ph["sub_div"], dims=tuple(ph["dims"]),
               cell=np.float32(ph["cell"]), starts=ph["cell_starts"].cpu().numpy().astype(np.uint32),
               sizes=ph["cell_sizes"].cpu().numpy().astype(np.uint32))
    lst = ctx.photons(0, sorted_=False)
    out["pos"], out["dir"], out["pow"] = (lst[k].cpu().numpy() for k in ("list_pos", "list_dir", "list_power"))
    return out


@pytest.fixture(scope="module")
def oracle_grid(frame, orc):
    s = orc.scene(frame["sc"])
    g = orc.grid_build(frame["pos"], frame["pow"], frame["dir"], s.aabb(), sub_div=frame["sub_div"])
    return s, g


def test_grid_of_the_frame(frame, oracle_grid):
    _, g = oracle_grid
    assert tuple(g.dims) == frame["dims"] and np.float32(g.cell) == frame["cell"]
    assert np.array_equal(g.starts, frame["starts"]) and np.array_equal(g.sizes, frame["sizes"])


def test_knn_sets_and_estimates_of_the_frame(frame, orc, oracle_grid):
    _, g = oracle_grid
    ctx, w, req = frame["ctx"], frame["w"], frame["req"]
    gl = np.nonzero(req["b"][:, 3].view(np.uint32) & 1)[0]
    pick = np.sort(np.random.default_rng(3).choice(gl, 20_000, replace=False))
    qp = np.ascontiguousarray(req["a"][pick, :3])
    qn = np.ascontiguousarray(req["b"][pick, :3])
    ids_o, cnt_o, _, rad_o = orc.gather(g, qp, qn, w["radius"], w["k"], heap_mode=False)
    rad, ids, cnt = ctx.gather(torch.from_numpy(qp), torch.from_numpy(qn), w["k"], w["radius"], want_ids=True)
    assert np.array_equal(cnt.cpu().numpy(), cnt_o)
    assert np.array_equal(ids.cpu().numpy().astype(np.uint32), ids_o)
    np.testing.assert_allclose(rad.cpu().numpy(), rad_o, rtol=RTOL, atol=1e-9)
    # the estimates the frame itself used (gathered in Morton order of the hit points)
    np.testing.assert_allclose(req["est_global"][pick], rad_o, rtol=RTOL, atol=1e-9)


def test_pixel_rows_of_the_frame(frame, orc, oracle_grid):
    s, g = oracle_grid
    w, cs = frame["w"], frame["cs"]
    W, H = cs.width, cs.height
    cv = orc.camera(cs)
    for y in np.linspace(0, H - 1, 8).astype(int):
        out = s.render(cv, W, H, g, w["k"], w["radius"], w["max_depth"], y0=int(y), y1=int(y) + 1)
        sl = slice(int(y) * W, (int(y) + 1) * W)
        np.testing.assert_allclose(frame["rad"][sl], out["radiance"], rtol=RTOL, atol=1e-7)
        d = np.abs(frame["rgb"][sl].astype(int) - out["rgb8"].astype(int))
        assert d.max() <= 1
