"""Pins of the CPU oracle against the reference's own results (no GPU).

The golden files were produced by tests/golden/make_golden.py, which runs the
reference's host code (compiled from its sources) and reads its photon dump.
"""
import os

import numpy as np
import pytest

from photonmap import scenes


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def test_philox_known_answers(orc):
    # Random123 known-answer vectors for Philox-4x32-10 (Salmon et al., SC'11)
    assert list(orc.philox_raw([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(orc.philox_raw([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(orc.philox_raw([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_uniform_stream_range(orc):
    u = orc.philox(1234, 0, 77, 4096)
    assert u.min() > 0.0 and u.max() <= 1.0
    assert abs(float(u.mean()) - 0.5) < 0.02
    # counter-based: the stream of a path does not depend on how it is consumed
    assert np.array_equal(orc.philox(1234, 0, 77, 10), u[:10])


def test_scan_known_answer(orc):
    # the reference's scan test input (CudaPhotonMapping/DynamicArrayTest.cu:165-172), checked
    # against a sequential sum as the reference does (:128-144)
    n = 1_000_000
    i = np.arange(n)
    a = np.where(i % 7 != 0, (i % 3 + 1) % 2, i % 2).astype(np.uint32)
    a[0] = 512 * 44
    inc = orc.scan_u32(a, True)
    exc = orc.scan_u32(a, False)
    ref = np.cumsum(a.astype(np.uint64))
    assert np.array_equal(inc, ref.astype(np.uint32))
    assert np.array_equal(exc[1:], inc[:-1]) and exc[0] == 0


def test_fixture100_grid_and_gather(orc, golden_dir):
    f = _load(golden_dir, "fixture100.npz")
    g = orc.grid_build(f["pos"], f["power"], f["dir"], f["aabb"], desired=int(f["desired"]))
    assert np.array_equal(g.dims, f["dims"]) and np.float32(g.cell) == f["cell"]
    assert np.array_equal(g.starts, f["starts"]) and np.array_equal(g.sizes, f["sizes"])
    k, r = int(f["k"]), float(f["r"])
    ids, cnt, rk, rad = orc.gather(g, f["q"], f["qn"], r, k, heap_mode=True)
    assert np.array_equal(cnt, f["ref_cnt"])
    assert np.array_equal(ids, f["ref_ids"])
    assert np.array_equal(rad, f["ref_rad"])          # bit-exact with the reference heap order
    ids_c, cnt_c, _, rad_c = orc.gather(g, f["q"], f["qn"], r, k, heap_mode=False)
    assert np.array_equal(cnt_c, cnt)
    for a, b, c in zip(ids_c, ids, cnt):
        assert set(a[:c]) == set(b[:c])
    np.testing.assert_allclose(rad_c, rad, rtol=1e-5, atol=1e-12)


def test_cornell_camera_rays_hdr_rayops(orc, golden_dir):
    f = _load(golden_dir, "cornell_ref.npz")
    cams = [scenes.default_camera(80, 60),
            scenes.CameraSpec((0.3, 0.2, 3.0), (-0.1, -0.05, -1.0), (0, 1, 0), 60.0, 64, 48),
            scenes.CameraSpec((0.0, 0.5, 2.5), (0.0, -0.3, -1.0), (0, 1, 0), 45.0, 1920, 1080)]
    for c, ref in zip(cams, f["cam_vecs"]):
        assert np.array_equal(orc.camera(c), ref)
    d = orc.camera_rays(f["cam_vecs"][2], 1920, 1080, f["eye_xs"], f["eye_ys"])
    assert np.array_equal(d, f["eye_dirs"])
    assert np.array_equal(orc.hdr(f["hdr_in"]), f["hdr_out"])
    a, b, ok = orc.ray_ops(f["op_dir"], f["op_from"], f["op_nrm"], f["op_etas"])
    assert np.array_equal(ok, f["ref_refract_ok"])
    assert np.array_equal(a, f["ref_reflect"])
    assert np.array_equal(b[ok == 1], f["ref_refract"][ok == 1])


def test_cornell_intersection(orc, golden_dir):
    f = _load(golden_dir, "cornell_ref.npz")
    sc, _, _ = scenes.workload("cornell_small")
    s = orc.scene(sc)
    t, m, tri, n = s.intersect(f["ray_orig"], f["ray_dir"])
    assert np.array_equal(m, f["ref_model"])
    hit = m >= 0
    p = (f["ray_dir"] * t[:, None]).astype(np.float32) + f["ray_orig"]
    assert np.array_equal(p[hit], f["ref_point"][hit])
    assert np.array_equal(n[hit], f["ref_normal"][hit])


def _cornell_map(orc, f):
    sc, _, _ = scenes.workload("cornell_small")
    s = orc.scene(sc)
    tr = s.trace_photons(int(f["seed"]), int(f["max_bounces"]), int(f["photons"]))
    h = np.concatenate([tr["g_pos"].ravel(), tr["g_dir"].ravel(), tr["g_pow"].ravel()]).view(np.uint32)
    chk = int(np.bitwise_xor.reduce(h * np.arange(1, h.size + 1, dtype=np.uint32)))
    assert chk == int(f["photons_checksum"])
    g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
    return s, g


def test_cornell_gather_matches_reference(orc, golden_dir):
    f = _load(golden_dir, "cornell_ref.npz")
    s, g = _cornell_map(orc, f)
    ids, cnt, rk, rad = orc.gather(g, f["gather_q"], f["gather_n"], 0.1, 100, heap_mode=True)
    assert np.array_equal(cnt, f["ref_gather_cnt"])
    assert np.array_equal(ids, f["ref_gather_ids"])
    assert np.array_equal(rad, f["ref_gather_rad"])


def test_cornell_render_matches_reference_cpu_mode(orc, golden_dir):
    f = _load(golden_dir, "cornell_ref.npz")
    s, g = _cornell_map(orc, f)
    cam = scenes.default_camera(int(f["render_w"]), int(f["render_h"]))
    out = s.render(orc.camera(cam), cam.width, cam.height, g, int(f["render_k"]), float(f["render_r"]),
                   int(f["render_depth"]), heap_mode=True)
    assert out["overflow"] == 0
    assert np.array_equal(out["ldr"], f["ref_ldr"])
    assert np.array_equal(out["rgb8"], f["ref_rgb8"])
    # canonical (distance, id) selection agrees with the heap within rounding
    out2 = s.render(orc.camera(cam), cam.width, cam.height, g, int(f["render_k"]), float(f["render_r"]),
                    int(f["render_depth"]), heap_mode=False)
    np.testing.assert_allclose(out2["radiance"], out["radiance"], rtol=1e-5, atol=1e-7)
