"""The seeded synthetic workloads hold the shapes, sizes and value
distributions of the configurations they stand in for (CPU only).

The reference measures on no public data set; its photon-mapping runs use a
Cornell-style room built in code.  The workloads here are generated by
photonmap.scenes: the small room at the reference's CPU-runnable size, the
same room with a 256 x 256-vertex heightfield floor at 10M photons / 1080p,
the nested-glass stress room at 100M photons / 4K, and the 64-instance
batch.  These tests pin each generator to the configuration it is named for.
"""
import math

import numpy as np
import pytest

from photonmap import scenes

DIFFUSE, SPECULAR, EMISSION, IOR, OPAQUE = slice(0, 3), slice(3, 6), slice(6, 9), 9, 10


def model_tris(sc, name):
    m = sc.names.index(name)
    return sc.tri_pos[sc.tri_model == m], sc.materials[m]


def sphere_fit(pos):
    """Centre and radii of the vertices of an icosphere."""
    v = pos.reshape(-1, 3).astype(np.float64)
    c = 0.5 * (v.min(0) + v.max(0))
    return c, np.linalg.norm(v - c, axis=1)


def check_room(sc, light_offset=(0.0, 0.0, 0.0), glass_r=0.3, mirror_r=0.3):
    # the room spans [-1, 1]^3 and its front side (z = +1) is open
    assert np.allclose(sc.aabb()[[0, 2, 3, 4, 5]], [-1, -1, 1, 1, 1], atol=1e-6)
    for name in ("ceiling", "back", "left", "right"):
        tris, _ = model_tris(sc, name)
        assert tris.shape[0] == 2
    assert not any(np.all(np.isclose(sc.tri_pos[sc.tri_model == m][..., 2], 1.0))
                   for m in range(sc.nmodel)), "no wall closes the front side"
    # walls: left red, right green, the others white
    assert np.allclose(model_tris(sc, "left")[1][DIFFUSE], (0.75, 0.25, 0.25))
    assert np.allclose(model_tris(sc, "right")[1][DIFFUSE], (0.25, 0.75, 0.25))
    for name in ("ceiling", "back", "floor"):
        assert np.allclose(model_tris(sc, name)[1][DIFFUSE], 0.75)
    # a 0.5 x 0.5 square light at y = 0.999 facing down, 1 W
    lt, lm = model_tris(sc, "light")
    assert sc.names[sc.light_model] == "light" and lt.shape[0] == 2
    v = lt.reshape(-1, 3)
    assert np.allclose(v[:, 1], 0.999)
    assert np.allclose(v[:, [0, 2]].max(0) - v[:, [0, 2]].min(0), 0.5, atol=1e-6)
    assert np.allclose(0.5 * (v[:, [0, 2]].max(0) + v[:, [0, 2]].min(0)), [light_offset[0], light_offset[2]],
                       atol=1e-6)
    assert np.allclose(lm[EMISSION], 1.0) and np.allclose(sc.light_intensity, 1.0)
    assert np.allclose(sc.tri_nrm[sc.tri_model == sc.light_model][..., 1], -1.0)
    # glass sphere at (-0.4, -0.7, 0.2), IOR 1.5; mirror sphere at (0.45, -0.7, -0.3)
    for name, centre, r, ior, opaque in (("glass", (-0.4, -0.7, 0.2), glass_r, 1.5, 0.0),
                                         ("mirror", (0.45, -0.7, -0.3), mirror_r, None, 1.0)):
        tris, m = model_tris(sc, name)
        c, radii = sphere_fit(tris)
        assert np.allclose(c, centre, atol=1e-5)
        assert np.allclose(radii, r, rtol=1e-5)
        assert np.allclose(m[SPECULAR], 1.0) and np.allclose(m[DIFFUSE], 0.0)
        assert m[OPAQUE] == opaque
        if ior is not None:
            assert m[IOR] == pytest.approx(ior)


def test_small_room_workload():
    sc, cam, w = scenes.workload("cornell_small")
    check_room(sc)
    floor, _ = model_tris(sc, "floor")
    assert floor.shape[0] == 2 and np.allclose(floor[..., 1], -1.0)
    # 5 walls + the light = 12 triangles before the spheres
    assert sum(model_tris(sc, n)[0].shape[0] for n in ("floor", "ceiling", "back", "left", "right", "light")) == 12
    assert (w["photons"], w["max_bounces"], w["k"], w["radius"], w["seed"]) == (100_000, 8, 100, 0.1, 0)
    assert (cam.width, cam.height, cam.fov_deg) == (320, 240, 45.0)
    assert cam.position == (0.0, 0.0, 3.5) and cam.direction == (0.0, 0.0, -1.0) and cam.up == (0.0, 1.0, 0.0)


def test_heightfield_workload():
    sc, cam, w = scenes.workload("cornell_hf_1080p")
    check_room(sc)
    floor, _ = model_tris(sc, "floor")
    assert floor.shape[0] == 2 * 255 ** 2                          # 256 x 256 vertices
    assert sc.ntri == 132_620
    y = floor[..., 1]
    assert y.min() >= -1.05 - 1e-6 and y.max() <= -1.0 + 0.05 + 1e-6 and y.max() - y.min() > 0.02
    # per-triangle albedo U[0.3, 0.8] on the floor, grey
    alb = sc.tri_diffuse[sc.tri_model == sc.names.index("floor")]
    assert np.all(alb[:, 0] == alb[:, 1]) and np.all(alb[:, 1] == alb[:, 2])
    assert alb.min() >= 0.3 and alb.max() <= 0.8
    assert abs(alb[:, 0].mean() - 0.55) < 0.01                        # uniform over [0.3, 0.8]
    assert (w["photons"], w["max_bounces"], w["k"], w["radius"]) == (10_000_000, 10, 64, 0.05)
    assert (cam.width, cam.height) == (1920, 1080)


def test_stress_workload():
    sc, cam, w = scenes.workload("cornell_stress_4k")
    check_room(sc)
    small = [m for m in range(sc.nmodel) if sc.names[m] == "glass_small"]
    assert len(small) == 4
    for m in small:
        mat = sc.materials[m]
        assert 1.3 <= mat[IOR] <= 1.7 and mat[OPAQUE] == 0.0
    big, mat = model_tris(sc, "glass_big")
    assert big.shape[0] == 81_920 >= 64_000                           # icosphere level 6
    assert mat[OPAQUE] == 0.0 and mat[IOR] == pytest.approx(1.5)
    assert sc.ntri == 89_612
    assert (w["photons"], w["max_bounces"], w["k"], w["radius"]) == (100_000_000, 16, 200, 0.02)
    assert (cam.width, cam.height) == (3840, 2160)


def test_batch_instances():
    insts = scenes.batch_instances(n=64, seed=0)
    assert len(insts) == 64
    photons = np.array([d["photons"] for d in insts])
    edges = np.array([d["camera_spec"].width for d in insts])
    assert all(d["camera_spec"].height == d["camera_spec"].width for d in insts)
    assert photons.min() >= 10_000 and photons.max() <= 2_000_000
    assert edges.min() >= 128 and edges.max() <= 1024
    assert {d["k"] for d in insts} <= {32, 64, 128} and len({d["k"] for d in insts}) == 3
    # log-uniform: log counts spread evenly over their range (mean near the middle)
    mid = 0.5 * (math.log(10_000) + math.log(2_000_000))
    assert abs(np.log(photons).mean() - mid) < 0.6
    assert abs(np.log(edges).mean() - 0.5 * (math.log(128) + math.log(1024))) < 0.4
    for d in insts[:8]:
        sc = d["scene"]
        lt, _ = model_tris(sc, "light")
        off = 0.5 * (lt.reshape(-1, 3).max(0) + lt.reshape(-1, 3).min(0))
        assert abs(off[0]) <= 0.2 + 1e-6 and abs(off[2]) <= 0.2 + 1e-6
        check_room(sc, light_offset=(off[0], 0.0, off[2]),
                   glass_r=sphere_fit(model_tris(sc, "glass")[0])[1].mean(),
                   mirror_r=sphere_fit(model_tris(sc, "mirror")[0])[1].mean())
        for name in ("glass", "mirror"):
            r = sphere_fit(model_tris(sc, name)[0])[1].mean()
            assert 0.15 <= r <= 0.4
    # seeded: the same seed gives the same instances, another seed others
    again = scenes.batch_instances(n=64, seed=0)
    assert [(d["photons"], d["k"], d["seed"]) for d in again] == [(d["photons"], d["k"], d["seed"]) for d in insts]
    other = scenes.batch_instances(n=64, seed=1)
    assert [d["photons"] for d in other] != list(photons)
