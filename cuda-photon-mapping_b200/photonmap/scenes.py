"""Seeded synthetic scenes for the photon-mapping workloads.

A scene is a triangle soup grouped into models (the reference's ``Model``,
CudaPhotonMapping/Model.cuh:24-28), one material per model
(CudaPhotonMapping/Material.cuh:4-31), optional per-triangle diffuse albedo,
and one area light (the model named ``light`` in the reference,
CudaPhotonMapping/Initializer.cu:70).  Triangles are stored sorted by model, so
the (model, triangle) order of the reference's closest-hit loop
(CudaPhotonMapping/Model.cuh:366-446) is the plain triangle index order.

Workloads (sizes in ``WORKLOADS``):
  cornell_small   room [-1,1]^3 from 10 triangles, open front, 0.5 x 0.5 light at
                  y = 0.999 (1 W), glass sphere (IOR 1.5) and mirror sphere (r 0.3),
                  100k photons, 320x240, k 100, r 0.1
  cornell_hf_1080p  the same room with a 256 x 256-vertex seeded value-noise
                  heightfield floor (130,050 triangles, amplitude 0.05, per-triangle
                  albedo U[0.3, 0.8]), 10M photons, depth 10, 1920x1080, k 64, r 0.05
  cornell_stress_4k the small room with 4 more glass spheres (IOR U[1.3, 1.7]) and an
                  81,920-triangle glass icosphere, 100M photons, depth 16, 3840x2160,
                  k 200, r 0.02
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

# material row layout shared with the C ABI: diffuse3 specular3 emission3 ior opaque shininess
MAT_FLOATS = 12


@dataclasses.dataclass
class Scene:
    tri_pos: np.ndarray          # (T, 3, 3) float32, vertices v0 v1 v2
    tri_nrm: np.ndarray          # (T, 3, 3) float32, vertex normals
    tri_model: np.ndarray        # (T,) int32, non-decreasing
    materials: np.ndarray        # (M, 12) float32
    light_model: int
    light_intensity: np.ndarray  # (3,) float32
    default_ior: float = 1.0
    tri_diffuse: Optional[np.ndarray] = None   # (T, 3) float32 per-triangle albedo override
    names: tuple = ()

    @property
    def ntri(self) -> int:
        return int(self.tri_pos.shape[0])

    @property
    def nmodel(self) -> int:
        return int(self.materials.shape[0])

    def aabb(self) -> np.ndarray:
        """Union of the model AABBs (CudaPhotonMapping/Initializer.cu:197-200)."""
        p = self.tri_pos.reshape(-1, 3)
        return np.concatenate([p.min(0), p.max(0)]).astype(np.float32)


@dataclasses.dataclass
class CameraSpec:
    position: tuple
    direction: tuple
    up: tuple
    fov_deg: float
    width: int
    height: int


def material(diffuse=(0, 0, 0), specular=(0, 0, 0), emission=(0, 0, 0), ior=1.0, opaque=1.0, shininess=16.0):
    return np.array(list(diffuse) + list(specular) + list(emission) + [ior, opaque, shininess], dtype=np.float32)


def _quad(a, b, c, d, n):
    """Two triangles (a,b,c), (a,c,d) with a shared flat normal n."""
    p = np.array([[a, b, c], [a, c, d]], dtype=np.float64)
    nn = np.tile(np.asarray(n, dtype=np.float64), (2, 3, 1))
    return p, nn


def icosphere(center, radius, level):
    """Subdivided icosahedron; smooth normals = normalised vertex directions."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(x, dtype=np.float64) / np.linalg.norm(x) for x in verts]
    for _ in range(level):
        cache = {}
        nf = []

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = v[i] + v[j]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.stack(v)
    F = np.asarray(faces, dtype=np.int64)
    nrm = V[F]
    pos = np.asarray(center, dtype=np.float64) + radius * nrm
    return pos, nrm


def _value_noise(rng, n, lattice=16):
    """Seeded value noise on an n x n vertex grid (smoothstep-interpolated lattice)."""
    g = rng.random((lattice + 1, lattice + 1))
    u = np.linspace(0.0, lattice, n)
    i0 = np.minimum(u.astype(np.int64), lattice - 1)
    f = u - i0
    s = f * f * (3 - 2 * f)
    a = g[i0][:, i0]
    b = g[i0][:, i0 + 1]
    c = g[i0 + 1][:, i0]
    d = g[i0 + 1][:, i0 + 1]
    sx = s[None, :]
    sz = s[:, None]
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def heightfield(n, amplitude, rng):
    """n x n vertices over [-1,1]^2 at y = -1 + amplitude * noise; 2 (n-1)^2 triangles."""
    h = _value_noise(rng, n)
    xs = np.linspace(-1.0, 1.0, n)
    X, Z = np.meshgrid(xs, xs)            # [z][x]
    Y = -1.0 + amplitude * h
    P = np.stack([X, Y, Z], -1)
    # smooth vertex normals from central differences of the height
    dx = 2.0 / (n - 1)
    gy = np.gradient(Y, dx)
    dYdz, dYdx = gy[0], gy[1]
    N = np.stack([-dYdx, np.ones_like(Y), -dYdz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    i = np.arange(n - 1)
    zz, xx = np.meshgrid(i, i, indexing="ij")
    a = np.stack([zz, xx], -1).reshape(-1, 2)
    def idx(dz, dx_):
        return (a[:, 0] + dz, a[:, 1] + dx_)
    v00, v01, v10, v11 = idx(0, 0), idx(0, 1), idx(1, 0), idx(1, 1)
    t1 = np.stack([P[v00], P[v10], P[v11]], 1)
    t2 = np.stack([P[v00], P[v11], P[v01]], 1)
    n1 = np.stack([N[v00], N[v10], N[v11]], 1)
    n2 = np.stack([N[v00], N[v11], N[v01]], 1)
    pos = np.stack([t1, t2], 1).reshape(-1, 3, 3)
    nrm = np.stack([n1, n2], 1).reshape(-1, 3, 3)
    return pos, nrm


def cornell(sphere_level=3, heightfield_n=0, seed=0, light_offset=(0.0, 0.0, 0.0),
            glass_radius=0.3, mirror_radius=0.3, stress=False):
    """The Cornell-style room shared by the workloads.

    Models (ids = indices): 0 floor, 1 ceiling, 2 back wall, 3 left wall (red),
    4 right wall (green), 5 light, 6 glass sphere, 7 mirror sphere.
    stress: also 4 small glass spheres (r 0.15, IOR uniform in [1.3, 1.7],
    seeded) and a large glass icosphere of 81,920 triangles (subdivision level
    6, the first icosphere above 64k triangles; r 0.3, IOR 1.5), models 8-12.
    """
    white = (0.75, 0.75, 0.75)
    parts = []   # (pos, nrm, material, per-tri diffuse or None, name)
    rng = np.random.default_rng(seed)
    if heightfield_n:
        p, n = heightfield(heightfield_n, 0.05, rng)
        alb = rng.uniform(0.3, 0.8, size=(p.shape[0], 1)).repeat(3, 1)
        parts.append((p, n, material(diffuse=white), alb, "floor"))
    else:
        p, n = _quad((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1), (0, 1, 0))
        parts.append((p, n, material(diffuse=white), None, "floor"))
    p, n = _quad((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1), (0, -1, 0))
    parts.append((p, n, material(diffuse=white), None, "ceiling"))
    p, n = _quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (0, 0, 1))
    parts.append((p, n, material(diffuse=white), None, "back"))
    p, n = _quad((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1), (1, 0, 0))
    parts.append((p, n, material(diffuse=(0.75, 0.25, 0.25)), None, "left"))
    p, n = _quad((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1), (-1, 0, 0))
    parts.append((p, n, material(diffuse=(0.25, 0.75, 0.25)), None, "right"))
    lx, ly, lz = light_offset
    y = 0.999
    p, n = _quad((-0.25 + lx, y, -0.25 + lz), (0.25 + lx, y, -0.25 + lz), (0.25 + lx, y, 0.25 + lz),
                 (-0.25 + lx, y, 0.25 + lz), (0, -1, 0))
    parts.append((p, n, material(emission=(1, 1, 1)), None, "light"))
    p, n = icosphere((-0.4, -0.7, 0.2), glass_radius, sphere_level)
    parts.append((p, n, material(specular=(1, 1, 1), ior=1.5, opaque=0.0), None, "glass"))
    p, n = icosphere((0.45, -0.7, -0.3), mirror_radius, sphere_level)
    parts.append((p, n, material(specular=(1, 1, 1), opaque=1.0), None, "mirror"))
    if stress:
        for c in ((-0.65, -0.85, -0.6), (0.0, -0.85, -0.7), (0.65, -0.85, 0.55), (-0.15, -0.85, 0.7)):
            ior = float(rng.uniform(1.3, 1.7))
            p, n = icosphere(c, 0.15, sphere_level)
            parts.append((p, n, material(specular=(1, 1, 1), ior=ior, opaque=0.0), None, "glass_small"))
        p, n = icosphere((0.1, 0.05, 0.1), 0.3, 6)
        parts.append((p, n, material(specular=(1, 1, 1), ior=1.5, opaque=0.0), None, "glass_big"))

    pos = np.concatenate([q[0] for q in parts]).astype(np.float32)
    nrm = np.concatenate([q[1] for q in parts]).astype(np.float32)
    tri_model = np.concatenate([np.full(q[0].shape[0], i, np.int32) for i, q in enumerate(parts)])
    mats = np.stack([q[2] for q in parts]).astype(np.float32)
    tri_diffuse = None
    if any(q[3] is not None for q in parts):
        tri_diffuse = np.concatenate([
            (q[3] if q[3] is not None else np.tile(q[2][0:3], (q[0].shape[0], 1))) for q in parts
        ]).astype(np.float32)
    return Scene(pos, nrm, tri_model, mats, light_model=5,
                 light_intensity=np.ones(3, np.float32), default_ior=1.0,
                 tri_diffuse=tri_diffuse, names=tuple(q[4] for q in parts))


def split_model(sc: Scene, model: int) -> Scene:
    """The same scene with `model` split into one model per triangle, each with
    the model's material and its triangle's albedo as diffuse.  The reference
    holds one material per model (CudaPhotonMapping/Model.cuh:24-28), so this is
    how a per-triangle albedo is written in its terms; the models after `model`
    (and the light's index) move up by its triangle count minus one."""
    tri = np.nonzero(sc.tri_model == model)[0]
    n = tri.size
    mats = sc.materials
    split = np.repeat(mats[model:model + 1], n, 0).copy()
    if sc.tri_diffuse is not None:
        split[:, 0:3] = sc.tri_diffuse[tri]
    new_mats = np.concatenate([mats[:model], split, mats[model + 1:]]).astype(np.float32)
    tm = sc.tri_model.astype(np.int64).copy()
    tm[sc.tri_model > model] += n - 1
    tm[tri] = model + np.arange(n)
    names = tuple(sc.names[:model]) + tuple(f"{sc.names[model]}_{i}" for i in range(n)) + tuple(sc.names[model + 1:]) \
        if sc.names else ()
    light = sc.light_model + (n - 1 if sc.light_model > model else 0)
    return Scene(sc.tri_pos, sc.tri_nrm, tm.astype(np.int32), new_mats, light_model=light,
                 light_intensity=sc.light_intensity, default_ior=sc.default_ior, tri_diffuse=None, names=names)


def default_camera(width, height):
    return CameraSpec((0.0, 0.0, 3.5), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 45.0, width, height)


# Workload table: the plain method at the reference's CPU-runnable size and at scale.
WORKLOADS = {
    "cornell_small": dict(scene=dict(sphere_level=3), photons=100_000, caustic=0, max_bounces=8,
                          width=320, height=240, k=100, radius=0.1, max_depth=4, seed=0),
    "cornell_hf_1080p": dict(scene=dict(sphere_level=3, heightfield_n=256), photons=10_000_000, caustic=0,
                             max_bounces=10, width=1920, height=1080, k=64, radius=0.05, max_depth=4, seed=0),
    "cornell_stress_4k": dict(scene=dict(sphere_level=3, stress=True), photons=100_000_000, caustic=0,
                              max_bounces=16, width=3840, height=2160, k=200, radius=0.02, max_depth=4, seed=0),
}


def workload(name):
    w = dict(WORKLOADS[name])
    sc = cornell(**w["scene"], seed=w["seed"])
    cam = default_camera(w["width"], w["height"])
    return sc, cam, w


def batch_instances(n=64, seed=0, photons_range=(10_000, 2_000_000), res_range=(128, 1024), ks=(32, 64, 128),
                    radius=0.1, max_bounces=8, max_depth=4):
    """Seeded instances of the batched workload: the small room with the light
    jittered uniformly by +-0.2 (x, z), sphere radii uniform in [0.15, 0.4],
    photon counts log-uniform in photons_range, square images with edge
    log-uniform in res_range, k drawn from ks.  Returns dicts of scene, camera
    spec and parameters."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        lx, lz = rng.uniform(-0.2, 0.2, 2)
        rg, rm = rng.uniform(0.15, 0.4, 2)
        sc = cornell(sphere_level=3, seed=seed + i, light_offset=(float(lx), 0.0, float(lz)),
                     glass_radius=float(rg), mirror_radius=float(rm))
        photons = int(round(math.exp(rng.uniform(math.log(photons_range[0]), math.log(photons_range[1])))))
        edge = int(round(math.exp(rng.uniform(math.log(res_range[0]), math.log(res_range[1])))))
        out.append(dict(scene=sc, camera_spec=default_camera(edge, edge), seed=seed * 1000 + i, photons=photons,
                        max_bounces=max_bounces, k=int(rng.choice(ks)), radius=radius, max_depth=max_depth))
    return out
