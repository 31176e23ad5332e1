"""Cases of the pins against the reference's own code, shared by
tests/golden/make_golden.py (which writes the reference's results into
tracer_ref.npz and grid_sizing_ref.npz) and the tests that check them.

CASES (photon tracer): a scene, the stream seed, the power capacity (photon
power = intensity / capacity) and the path range traced.  The bounce limit is
the reference's fixed PHOTON_BOUNCE_NUM (10, CudaPhotonMapping/PhotonTracing.cu:20).

GRID_CASES (grid sizing): seeded photon positions in a scene box and the
desired photons per cell (CudaPhotonMapping/PhotonGrid.cu:41-56, 92-141).
"""
import numpy as np

from photonmap import scenes


def _heightfield_uniform():
    sc = scenes.cornell(sphere_level=3, heightfield_n=256, seed=0)
    sc.tri_diffuse = None          # the 130k-triangle floor as one model of one material
    return sc


def _heightfield_per_triangle():
    # a 16 x 16-vertex floor (450 triangles) with per-triangle albedo, written as
    # one reference model per triangle
    return scenes.split_model(scenes.cornell(sphere_level=3, heightfield_n=16, seed=1), 0)


CASES = {
    # name: (scene builder, seed, power capacity, first path, end path, golden subset end)
    "cornell_small": (lambda: scenes.cornell(sphere_level=3, seed=0), 0, 100_000, 0, 100_000, 4_000),
    "stress_glass": (lambda: scenes.cornell(sphere_level=3, stress=True, seed=0), 3, 1_000_000, 0, 5_000, 2_000),
    "heightfield": (_heightfield_uniform, 5, 10_000_000, 0, 2_000, 2_000),
    "heightfield_albedo": (_heightfield_per_triangle, 9, 1_000_000, 0, 20_000, 4_000),
}

MAX_BOUNCES = 10
FIELDS = ("counts", "draws", "g_pos", "g_dir", "g_bounce", "c_pos", "c_dir", "c_bounce")


def checksum(out):
    """Order-sensitive checksum of a trace_paths result over FIELDS."""
    import numpy as np
    h = np.concatenate([np.ascontiguousarray(out[f]).view(np.uint32).ravel() for f in FIELDS])
    return int(np.bitwise_xor.reduce(h * np.arange(1, h.size + 1, dtype=np.uint32)))


def _room_surfaces(n, seed, aabb):
    """n points on the floor, ceiling and three walls of the box, the floor
    holding half of them within 0.05 of its plane (a heightfield's spread)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(aabb[:3], np.float64), np.asarray(aabb[3:], np.float64)
    p = lo + rng.random((n, 3)) * (hi - lo)
    face = rng.integers(0, 8, n)
    p[face < 4, 1] = lo[1] + 0.05 * rng.random(int((face < 4).sum()))
    p[face == 4, 1] = hi[1]
    p[face == 5, 2] = lo[2]
    p[face == 6, 0] = lo[0]
    p[face == 7, 0] = hi[0]
    return p.astype(np.float32)


def _uniform(n, seed, aabb):
    """n points uniform in the box: no cell far above the mean, no re-grid."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(aabb[:3], np.float64), np.asarray(aabb[3:], np.float64)
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def _clustered(n, seed, aabb):
    """n points, 40 % of them inside one small ball: the density re-grid case."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(aabb[:3], np.float64), np.asarray(aabb[3:], np.float64)
    p = lo + rng.random((n, 3)) * (hi - lo)
    k = int(0.4 * n)
    p[:k] = np.array([0.2, -0.9, 0.1]) + 0.03 * rng.normal(size=(k, 3))
    return np.clip(p, lo, hi).astype(np.float32)


def _oracle_small_map():
    from oracle import Oracle
    sc = scenes.cornell(sphere_level=3, seed=0)
    s = Oracle().scene(sc)
    return s.trace_photons(0, 8, 100_000)["g_pos"], s.aabb()


def _hf_box():
    return scenes.cornell(sphere_level=3, heightfield_n=256, seed=0).aabb()


GRID_CASES = {
    # name: (positions builder -> (pos, aabb), desired per cell)
    "cornell_small_100k": (_oracle_small_map, 1000),
    "room_10M": (lambda: (_room_surfaces(10_000_000, 11, _hf_box()), _hf_box()), 1000),
    "clustered_200k": (lambda: (_clustered(200_000, 12, _hf_box()), _hf_box()), 1000),
    "room_1M_desired_50": (lambda: (_room_surfaces(1_000_000, 13, _hf_box()), _hf_box()), 50),
    "uniform_2M": (lambda: (_uniform(2_000_000, 14, _hf_box()), _hf_box()), 1000),
}
