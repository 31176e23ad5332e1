"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the
reference-generated golden files.

Tolerances: photon positions / directions / powers, grid arrays, kNN id sets:
bit-exact.  Radiance: 1e-4 relative (the estimate and the tone map use CUDA's
expf / powf, the oracle glibc's).  8-bit pixels: at most 1 level apart.
"""
import os

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


# ------------------------------------------------------------------- scan
@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 100_003, 1_000_000])
def test_scan_matches_sequential_sum(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 1000, n).astype(np.int32)
    x = torch.from_numpy(a).cuda()
    inc = _np(ctx.scan_u32(x, True)).astype(np.uint32)
    exc = _np(ctx.scan_u32(x, False)).astype(np.uint32)
    ref = np.cumsum(a.astype(np.uint64)).astype(np.uint32)
    assert np.array_equal(inc, ref)
    if n:
        assert exc[0] == 0 and np.array_equal(exc[1:], ref[:-1])


def test_scan_known_answer_of_reference(ctx):
    # CudaPhotonMapping/DynamicArrayTest.cu:165-172 input, checked against a sequential sum
    n = 1_000_000
    i = np.arange(n)
    a = np.where(i % 7 != 0, (i % 3 + 1) % 2, i % 2).astype(np.int32)
    a[0] = 512 * 44
    inc = _np(ctx.scan_u32(torch.from_numpy(a).cuda(), True)).astype(np.uint64)
    assert np.array_equal(inc, np.cumsum(a.astype(np.uint64)))


# ----------------------------------------------------------------- tracer
@pytest.fixture(scope="module")
def cornell(orc, ctx):
    sc, cam, w = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    s = orc.scene(sc)
    return sc, cam, w, s


def test_scene_aabb_and_tracer_matches_oracle(ctx, cornell):
    sc, cam, w, s = cornell
    assert np.array_equal(ctx.scene_aabb(), s.aabb())
    n = w["photons"]
    paths = ctx.trace_photons(w["seed"], w["max_bounces"], n)
    tr = s.trace_photons(w["seed"], w["max_bounces"], n)
    assert paths >= tr["paths"]
    ph = ctx.photons(0, sorted_=False)
    assert ph["count"] == n
    assert np.array_equal(_np(ph["list_pos"]), tr["g_pos"])
    assert np.array_equal(_np(ph["list_dir"]), tr["g_dir"])
    assert np.array_equal(_np(ph["list_power"]), tr["g_pow"])


def test_traced_map_grid_arrays_written_when_asked(ctx, orc, cornell):
    # a traced map's direction / power lists and its grid's sorted power are
    # written by the first photons() call after the photon pass / grid build;
    # the grid itself equals the oracle's grid of the same photons
    sc, cam, w, s = cornell
    ctx.set_scene(sc)
    ctx.trace_photons(4, w["max_bounces"], 40_000, 3_000)
    ctx.build_grid(0)
    ctx.build_grid(1)
    tr = s.trace_photons(4, w["max_bounces"], 40_000, 3_000)
    for map_id, key in ((0, "g"), (1, "c")):
        ph = ctx.photons(map_id)
        g = orc.grid_build(tr[f"{key}_pos"], tr[f"{key}_pow"], tr[f"{key}_dir"], s.aabb(), sub_div=ph["sub_div"])
        sp = _np(ph["sorted_pos"])
        assert np.array_equal(sp[:, :3], g.spos) and np.array_equal(sp[:, 3].view(np.uint32), g.sid)
        assert np.array_equal(_np(ph["sorted_dir"]), g.sdir)
        assert np.array_equal(_np(ph["sorted_power"]), g.spow)
        lst = ctx.photons(map_id, sorted_=False)
        assert np.array_equal(_np(lst["list_dir"]), tr[f"{key}_dir"])
        assert np.array_equal(_np(lst["list_power"]), tr[f"{key}_pow"])
    assert ctx.status() == 0


def test_trace_with_caustic_map(ctx, cornell):
    sc, cam, w, s = cornell
    paths = ctx.trace_photons(3, 8, 20_000, 2_000)
    tr = s.trace_photons(3, 8, 20_000, 2_000)
    g = ctx.photons(0, sorted_=False)
    c = ctx.photons(1, sorted_=False)
    assert np.array_equal(_np(g["list_pos"]), tr["g_pos"])
    assert np.array_equal(_np(c["list_pos"]), tr["c_pos"])
    assert np.array_equal(_np(c["list_dir"]), tr["c_dir"])
    assert np.array_equal(_np(c["list_power"]), tr["c_pow"])


def test_trace_stress_scene_nested_glass(ctx, orc):
    # the stress room: five glass bodies of four IORs, 16 bounces, a caustic map
    sc, cam, w = scenes.workload("cornell_stress_4k")
    ctx.set_scene(sc)
    s = orc.scene(sc)
    ctx.trace_photons(5, w["max_bounces"], 30_000, 10_000)
    tr = s.trace_photons(5, w["max_bounces"], 30_000, 10_000)
    g = ctx.photons(0, sorted_=False)
    c = ctx.photons(1, sorted_=False)
    for key, arr in (("g_pos", g["list_pos"]), ("g_dir", g["list_dir"]), ("c_pos", c["list_pos"]),
                     ("c_dir", c["list_dir"]), ("c_pow", c["list_power"])):
        assert np.array_equal(_np(arr), tr[key]), key
    assert ctx.status() == 0


def test_trace_paths_heightfield_subset(ctx, orc):
    # the 130k-triangle scene: the BVH must return the reference's closest hits
    sc = scenes.cornell(sphere_level=3, heightfield_n=256, seed=0)
    ctx.set_scene(sc)
    s = orc.scene(sc)
    p0, p1, B = 5000, 6500, 10
    out = ctx.trace_paths(0, B, 10_000_000, p0, p1)
    ref = s.trace_paths(0, B, 10_000_000, p0, p1)
    assert np.array_equal(_np(out["counts"]), ref["counts"])
    assert np.array_equal(_np(out["g_pos"]), ref["g_pos"])
    assert np.array_equal(_np(out["g_dir"]), ref["g_dir"])
    assert np.array_equal(_np(out["c_pos"]), ref["c_pos"])


@pytest.mark.parametrize("name", ["cornell_small", "stress_glass", "heightfield", "heightfield_albedo"])
def test_trace_paths_match_reference_tracer(ctx, name):
    """The CUDA tracer against the reference's own tracer (CudaPhotonMapping/
    PhotonTracing.cu compiled as host code, records in tests/golden/tracer_ref.npz
    written by tests/golden/make_golden.py): per-path photon counts, positions
    and directions of both maps, bit for bit, at the reference's 10 bounces."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import ref_cases
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tracer_ref.npz"))
    build, seed, cap, p0, _, sub = ref_cases.CASES[name]
    ctx.set_scene(build())
    out = ctx.trace_paths(seed, ref_cases.MAX_BOUNCES, cap, p0, sub)
    assert np.array_equal(_np(out["counts"]), f[f"{name}__counts"])
    for key in ("g_pos", "g_dir", "c_pos", "c_dir"):
        assert np.array_equal(_np(out[key]), f[f"{name}__{key}"]), key
    assert ctx.status() == 0


@pytest.mark.parametrize("which", ["cornell_small", "heightfield", "cornell_stress_4k"])
def test_device_bvh_gives_the_same_photons_and_image(ctx, which):
    """The device LBVH and the host SAH tree answer every closest-hit query the
    same (smallest (t, triangle index)), so the photon lists, the caustic map
    and the image are bit-identical; only the tree (and its speed) differs."""
    import photonmap
    if which == "heightfield":
        sc = scenes.cornell(sphere_level=3, heightfield_n=256, seed=0)
    else:
        sc = scenes.workload(which)[0]
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 160, 90)
    out = {}
    for builder in ("host_sah", "device_lbvh"):
        ctx.set_bvh_builder(builder)
        ctx.set_scene(sc)
        info = ctx.bvh_info()
        assert info["builder"] == builder and info["nodes"] >= 1 and info["build_ms"] >= 0.0
        ctx.trace_photons(3, 12, 40_000, 8_000)
        g = ctx.photons(0, sorted_=False)
        c = ctx.photons(1, sorted_=False)
        ctx.build_grid(0)
        ctx.build_grid(1)
        rgb, rad = ctx.render(cam, 64, 0.1, 4, k_caustic=32, r_caustic=0.1)
        out[builder] = [_np(t) for t in (g["list_pos"], g["list_dir"], g["list_power"], c["list_pos"],
                                         c["list_dir"], rgb, rad)]
        assert ctx.status() == 0
    ctx.set_bvh_builder("host_sah")
    for a, b in zip(out["host_sah"], out["device_lbvh"]):
        assert np.array_equal(a, b)


def test_heightfield_render_matches_oracle(ctx, orc):
    # eye rays through the BVH of the 130k-triangle scene, small photon map
    sc = scenes.cornell(sphere_level=3, heightfield_n=256, seed=0)
    ctx.set_scene(sc)
    s = orc.scene(sc)
    ctx.trace_photons(0, 10, 30_000)
    ctx.build_grid(0)
    import photonmap
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 96, 54)
    rgb, rad = ctx.render(cam, 64, 0.1, 4)
    tr = s.trace_photons(0, 10, 30_000)
    g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
    out = s.render(cam.as_vector(), 96, 54, g, 64, 0.1, 4)
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)


# ------------------------------------------------------------------- grid
def _oracle_grid(orc, pos, pw, dr, aabb, desired=1000, sub_div=1):
    return orc.grid_build(pos, pw, dr, aabb, desired=desired, sub_div=sub_div)


def _check_grid(ctx, orc, pos, pw, dr, aabb, desired=1000, map_id=0, auto=False):
    ph = ctx.photons(map_id)
    g = _oracle_grid(orc, pos, pw, dr, aabb, desired, sub_div=ph["sub_div"])
    if auto:   # the automatic sub-division is the same rule on both sides
        assert _oracle_grid(orc, pos, pw, dr, aabb, desired, sub_div=0).sub_div == ph["sub_div"]
    ks = _np(ph["key_starts"]).astype(np.int64)
    S3 = ph["sub_div"] ** 3
    assert ks[-1] == len(pos) and np.array_equal(ks[:-1:S3][:len(g.starts)], g.starts.astype(np.int64))
    assert tuple(ph["dims"]) == tuple(g.dims) and np.float32(ph["cell"]) == np.float32(g.cell)
    assert np.array_equal(_np(ph["cell_sizes"]).astype(np.uint32), g.sizes)
    assert np.array_equal(_np(ph["cell_starts"]).astype(np.uint32), g.starts)
    sp = _np(ph["sorted_pos"])
    assert np.array_equal(sp[:, :3], g.spos)
    assert np.array_equal(sp[:, 3].view(np.uint32), g.sid)
    assert np.array_equal(_np(ph["sorted_dir"]), g.sdir)
    assert np.array_equal(_np(ph["sorted_power"]), g.spow)
    return g


def test_grid_build_matches_oracle(ctx, orc, cornell):
    sc, cam, w, s = cornell
    ctx.set_scene(sc)
    tr = s.trace_photons(w["seed"], w["max_bounces"], w["photons"])
    ctx.set_photons(0, tr["g_pos"], tr["g_pow"], tr["g_dir"])
    for sub in (0, 1, 2, 8):
        ctx.build_grid(0, sub_div=sub)
        _check_grid(ctx, orc, tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb(), auto=sub == 0)


def test_grid_regrid_path_and_multi_pass_radix(ctx, orc):
    # clustered photons force the re-grid (max cell > 5x desired); > 65536 cells (3 radix passes)
    rng = np.random.default_rng(5)
    n = 300_000
    pos = np.concatenate([rng.normal(0.3, 0.02, (n // 2, 3)), rng.uniform(-1, 1, (n - n // 2, 3))]).astype(np.float32)
    pos = np.clip(pos, -1, 1)
    dr = rng.normal(size=(n, 3)).astype(np.float32)
    pw = np.full((n, 3), 1e-5, np.float32)
    aabb = np.array([-1, -1, -1, 1, 1, 1], np.float32)
    ctx.set_photons(0, pos, pw, dr)
    ctx.build_grid(0, desired=10, aabb=aabb, sub_div=1)
    g = _check_grid(ctx, orc, pos, pw, dr, aabb, desired=10)
    assert g.sizes.size > 256 * 256   # re-gridded; cell ids need three 8-bit passes


@pytest.mark.parametrize("cluster,sub_div", [(5_000, 1), (5_000, 8), (20_000, 2), (40_000, 1)])
def test_grid_dense_keys_and_radix_fallback(ctx, orc, cluster, sub_div):
    # a tight cluster puts `cluster` photons into one cell and one sub-cell
    # (its key's run in every radix pass is thousands of photons long), the
    # rest are spread over the box
    rng = np.random.default_rng(9)
    n = cluster + 50_000
    pos = np.concatenate([rng.normal(0.25, 1e-4, (cluster, 3)), rng.uniform(-1, 1, (n - cluster, 3))]).astype(np.float32)
    pos = rng.permutation(np.clip(pos, -1, 1))
    dr = rng.normal(size=(n, 3)).astype(np.float32)
    pw = rng.uniform(1e-6, 1e-5, (n, 3)).astype(np.float32)
    aabb = np.array([-1, -1, -1, 1, 1, 1], np.float32)
    ctx.set_photons(0, pos, pw, dr)
    ctx.build_grid(0, aabb=aabb, sub_div=sub_div)
    g = _check_grid(ctx, orc, pos, pw, dr, aabb)
    assert g.sizes.max() >= cluster
    assert ctx.status() == 0


def test_grid_fixture100(ctx, orc, golden_dir):
    f = np.load(os.path.join(golden_dir, "fixture100.npz"))
    ctx.set_photons(0, f["pos"], f["power"], f["dir"])
    ctx.build_grid(0, desired=int(f["desired"]), aabb=f["aabb"])
    ph = ctx.photons(0)
    assert tuple(ph["dims"]) == tuple(f["dims"])
    assert np.array_equal(_np(ph["cell_starts"]).astype(np.uint32), f["starts"])
    assert np.array_equal(_np(ph["cell_sizes"]).astype(np.uint32), f["sizes"])
    # the reference's own find_nearests / get_color on this grid (golden)
    k, r = int(f["k"]), float(f["r"])
    rad, ids, cnt = ctx.gather(torch.from_numpy(f["q"]), torch.from_numpy(f["qn"]), k, r, want_ids=True)
    assert np.array_equal(_np(cnt), f["ref_cnt"])
    ids = _np(ids).astype(np.uint32)
    for a, b, c in zip(ids, f["ref_ids"], f["ref_cnt"]):
        assert set(a[:c]) == set(b[:c])
    np.testing.assert_allclose(_np(rad), f["ref_rad"], rtol=RTOL, atol=1e-9)


# ----------------------------------------------------------------- gather
def test_gather_matches_oracle(ctx, orc, cornell):
    sc, cam, w, s = cornell
    ctx.set_scene(sc)
    tr = s.trace_photons(w["seed"], w["max_bounces"], w["photons"])
    ctx.set_photons(0, tr["g_pos"], tr["g_pow"], tr["g_dir"])
    ctx.build_grid(0)
    g = _oracle_grid(orc, tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
    rng = np.random.default_rng(11)
    q = (tr["g_pos"][rng.integers(0, len(tr["g_pos"]), 4000)] + rng.normal(scale=0.02, size=(4000, 3))).astype(np.float32)
    qn = rng.normal(size=(4000, 3)).astype(np.float32)
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    for sub in (1, 4, 8):
        ctx.build_grid(0, sub_div=sub)
        for k, r in [(100, 0.1), (1, 0.05), (16, 0.3), (256, 0.2)]:
            ids_o, cnt_o, rk_o, rad_o = orc.gather(g, q, qn, r, k, heap_mode=False)
            rad, ids, cnt = ctx.gather(torch.from_numpy(q), torch.from_numpy(qn), k, r, want_ids=True)
            assert np.array_equal(_np(cnt), cnt_o)
            assert np.array_equal(_np(ids).astype(np.uint32), ids_o)
            np.testing.assert_allclose(_np(rad), rad_o, rtol=RTOL, atol=1e-8)


# ----------------------------------------------------------------- render
def test_render_matches_reference_golden(ctx, orc, golden_dir):
    f = np.load(os.path.join(golden_dir, "cornell_ref.npz"))
    sc, _, _ = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    s = orc.scene(sc)
    tr = s.trace_photons(int(f["seed"]), int(f["max_bounces"]), int(f["photons"]))
    ctx.set_photons(0, tr["g_pos"], tr["g_pow"], tr["g_dir"])
    ctx.build_grid(0)
    import photonmap
    W, H = int(f["render_w"]), int(f["render_h"])
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, W, H)
    assert np.array_equal(cam.as_vector(), f["cam_vecs"][0])
    rgb, rad = ctx.render(cam, int(f["render_k"]), float(f["render_r"]), int(f["render_depth"]))
    rgb = _np(rgb).reshape(-1, 3).astype(np.int32)
    ref = f["ref_rgb8"].astype(np.int32)
    assert np.abs(rgb - ref).max() <= 1
    assert (rgb != ref).mean() < 0.01
    g = _oracle_grid(orc, tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
    out = s.render(orc.camera(scenes.default_camera(W, H)), W, H, g, int(f["render_k"]), float(f["render_r"]),
                   int(f["render_depth"]), heap_mode=False)
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)


def test_render_full_small_workload_matches_oracle(ctx, orc, cornell):
    sc, _, w, s = cornell
    ctx.set_scene(sc)
    paths = ctx.trace_photons(w["seed"], w["max_bounces"], w["photons"])
    ctx.build_grid(0)
    import photonmap
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, w["width"], w["height"])
    rgb, rad = ctx.render(cam, w["k"], w["radius"], w["max_depth"])
    tr = s.trace_photons(w["seed"], w["max_bounces"], w["photons"])
    g = _oracle_grid(orc, tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
    out = s.render(cam.as_vector(), w["width"], w["height"], g, w["k"], w["radius"], w["max_depth"])
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)
    d = np.abs(_np(rgb).reshape(-1, 3).astype(np.int32) - out["rgb8"].astype(np.int32))
    assert d.max() <= 1


def test_render_with_caustic_map(ctx, orc, cornell):
    sc, _, w, s = cornell
    ctx.set_scene(sc)
    ctx.trace_photons(1, 8, 40_000, 4_000)
    ctx.build_grid(0)
    ctx.build_grid(1)
    import photonmap
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 64, 48)
    rgb, rad = ctx.render(cam, 50, 0.1, 4, k_caustic=20, r_caustic=0.2, faithful_caustic=True)
    tr = s.trace_photons(1, 8, 40_000, 4_000)
    # the faithful caustic estimate reads the global map's arrays with caustic slot
    # numbers, so both sides must use the same in-cell order (sub-division) per map
    g = _oracle_grid(orc, tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb(), sub_div=ctx.photons(0)["sub_div"])
    c = _oracle_grid(orc, tr["c_pos"], tr["c_pow"], tr["c_dir"], s.aabb(), sub_div=ctx.photons(1)["sub_div"])
    out = s.render(cam.as_vector(), 64, 48, g, 50, 0.1, 4, c=c, k_c=20, r_c=0.2, faithful_caustic=True)
    np.testing.assert_allclose(_np(rad), out["radiance"], rtol=RTOL, atol=1e-7)


# ------------------------------------------------------- full-size checks
def test_full_size_photon_pass_properties(ctx):
    """cornell_hf_1080p photon pass (10M photons): size-independent properties."""
    sc, cam, w = scenes.workload("cornell_hf_1080p")
    ctx.set_scene(sc)
    n = w["photons"]
    ctx.trace_photons(w["seed"], w["max_bounces"], n)
    ctx.build_grid(0)
    ph = ctx.photons(0)
    aabb = ctx.scene_aabb()
    lp = ph["list_pos"]
    lo = torch.from_numpy(aabb[:3]).cuda() - 1e-4
    hi = torch.from_numpy(aabb[3:]).cuda() + 1e-4
    assert bool(((lp >= lo) & (lp <= hi)).all())
    pw = ph["list_power"]
    assert bool((pw == pw[0]).all()) and abs(float(pw[0, 0]) - 1.0 / n) < 1e-12
    sizes = ph["cell_sizes"].long()
    starts = ph["cell_starts"].long()
    assert int(sizes.sum()) == n
    assert bool((starts[1:] == torch.cumsum(sizes, 0)[:-1]).all()) and int(starts[0]) == 0
    sp = ph["sorted_pos"]
    ids = sp[:, 3].contiguous().view(torch.int32).long()
    assert bool((torch.sort(ids).values == torch.arange(n, device=ids.device)).all())   # a permutation
    # every photon sits in the cell / sub-cell its position hashes to (IEEE float32
    # division on the host, as CudaPhotonMapping/PhotonGrid.cu:10-38 computes it), and
    # photons of one sub-cell keep trace order
    gx, gy, gz = ph["dims"]
    cell = np.float32(ph["cell"])
    S = ph["sub_div"]
    spn = _np(sp[:, :3])
    u = (spn - aabb[:3]) / cell
    c3 = np.minimum(np.maximum(u.astype(np.int32), 0), np.array([gx - 1, gy - 1, gz - 1], np.int32))
    s3 = np.minimum(np.maximum(((u - c3.astype(np.float32)) * np.float32(S)).astype(np.int32), 0), S - 1)
    key = ((c3[:, 0] + c3[:, 1] * gx + c3[:, 2] * gx * gy).astype(np.int64) * S ** 3 +
           s3[:, 0] + S * (s3[:, 1] + S * s3[:, 2]))
    ks = ph["key_starts"].long()
    slot_key = torch.repeat_interleave(torch.arange(ks.numel() - 1, device=ks.device), ks[1:] - ks[:-1])
    assert bool((torch.from_numpy(key).cuda() == slot_key).all())
    slot_cell = torch.div(slot_key, S ** 3, rounding_mode="floor")
    assert bool((torch.repeat_interleave(torch.arange(sizes.numel(), device=sizes.device), sizes) == slot_cell).all())
    same = slot_key[1:] == slot_key[:-1]
    assert bool((ids[1:][same] > ids[:-1][same]).all())
    assert np.array_equal(_np(ph["list_pos"])[_np(ids)[:1000]], _np(sp[:1000, :3]))


def test_frame_call_equals_the_three_calls(ctx):
    """pm_frame (eye pass beside the grid build) gives the photons and the image
    of pm_trace_photons + pm_build_grid + pm_render, with and without a caustic map."""
    import photonmap
    sc, cs, w = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 128, 96)
    for caustic, kc in ((0, 0), (8_000, 32)):
        ctx.trace_photons(7, 8, 60_000, caustic)
        ctx.build_grid(0)
        if caustic:
            ctx.build_grid(1)
        rgb_a, rad_a = ctx.render(cam, 64, 0.1, 4, k_caustic=kc, r_caustic=0.1)
        rgb_a, rad_a = rgb_a.clone(), rad_a.clone()
        pos_a = _np(ctx.photons(0, sorted_=False)["list_pos"])
        rgb_b, rad_b, paths = ctx.frame(7, 8, 60_000, cam, 64, 0.1, 4, caustic_capacity=caustic, k_caustic=kc,
                                        r_caustic=0.1)
        assert paths > 0
        assert np.array_equal(_np(ctx.photons(0, sorted_=False)["list_pos"]), pos_a)
        assert torch.equal(rgb_b, rgb_a)
        assert torch.equal(rad_b, rad_a)
        assert ctx.status() == 0
        # the kernels timed alone lie inside their stages
        st = ctx.stage_times()
        assert 0 < st["k_trace_ms"] <= st["trace_ms"]
        assert 0 < st["k_gather_ms"] <= st["gather_ms"]


def test_photon_pass_batches_equal_the_path_range(ctx):
    """pm_trace_photons (a pilot batch, then batches sized by the measured
    yield, cut at the capacity) gives the first 150,000 global photons of
    pm_trace_paths over the same paths in canonical order (heightfield room)."""
    sc, cam, w = scenes.workload("cornell_hf_1080p")
    ctx.set_scene(sc)
    seed, nb = 11, 10
    n_paths = ctx.trace_photons(seed, nb, 150_000)
    assert n_paths >= 1 << 16
    lst = ctx.photons(0, sorted_=False)
    part = ctx.trace_paths(seed, nb, 150_000, 0, n_paths)
    cnt = _np(part["counts"])
    g = int(cnt[:, 0].sum())
    assert g >= 150_000
    # canonical order (path, then bounce) cut at the capacity: the list is the
    # first 150,000 global photons of the path-ordered records
    assert np.array_equal(_np(part["g_pos"])[:150_000], _np(lst["list_pos"]))
    assert np.array_equal(_np(part["g_dir"])[:150_000], _np(lst["list_dir"]))
    assert ctx.status() == 0
