"""Seeded random variants of the room for the fuzz parity tests.

Each scene is the room of photonmap.scenes.cornell (random light offset,
sphere sizes and tessellation, optionally a small heightfield floor) plus a
few random triangle blobs, each one model with a random material: diffuse,
mirror, glossy (partial specular), glass (opaque 0) or translucent (opaque
between 0 and 1) with an IOR in [1.2, 1.9].  Some blobs carry degenerate
triangles (collinear or repeated vertices).  Normals are the flat normals of
the triangles, so a blob is closed or open at random."""
import numpy as np

from photonmap import scenes


def _blob(rng, n_tris, degenerate):
    c = rng.uniform([-0.7, -0.8, -0.7], [0.7, 0.7, 0.7])
    size = rng.uniform(0.05, 0.35)
    pos = c + rng.normal(scale=size, size=(n_tris, 3, 3))
    pos = np.clip(pos, -0.98, 0.98)
    if degenerate:
        k = rng.integers(0, n_tris)
        pos[k, 2] = pos[k, 0] + 0.5 * (pos[k, 1] - pos[k, 0])      # collinear
        k = rng.integers(0, n_tris)
        pos[k, 1] = pos[k, 0]                                      # repeated vertex
    e1 = pos[:, 1] - pos[:, 0]
    e2 = pos[:, 2] - pos[:, 0]
    n = np.cross(e1, e2)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(ln > 0, n / np.where(ln > 0, ln, 1), np.array([0.0, 1.0, 0.0]))
    nrm = np.repeat(n[:, None, :], 3, axis=1)
    return pos, nrm


def _material(rng):
    kind = rng.choice(["diffuse", "mirror", "glossy", "glass", "translucent"])
    if kind == "diffuse":
        return scenes.material(diffuse=tuple(rng.uniform(0.1, 0.9, 3)))
    if kind == "mirror":
        return scenes.material(specular=(1, 1, 1), opaque=1.0)
    if kind == "glossy":
        return scenes.material(diffuse=tuple(rng.uniform(0.1, 0.6, 3)), specular=tuple(rng.uniform(0.2, 0.8, 3)),
                               shininess=float(rng.uniform(4, 64)))
    ior = float(rng.uniform(1.2, 1.9))
    if kind == "glass":
        return scenes.material(specular=(1, 1, 1), ior=ior, opaque=0.0)
    return scenes.material(diffuse=tuple(rng.uniform(0.1, 0.6, 3)), specular=(1, 1, 1), ior=ior,
                           opaque=float(rng.uniform(0.2, 0.8)))


def random_scene(seed, per_triangle_albedo=False):
    """A seeded random room (see the module docstring).  per_triangle_albedo:
    a heightfield floor with per-triangle albedo (not representable in the
    reference's one-material-per-model scenes)."""
    rng = np.random.default_rng(1000 + seed)
    hf = int(rng.choice([9, 17])) if per_triangle_albedo else 0
    base = scenes.cornell(sphere_level=int(rng.integers(1, 4)), heightfield_n=hf, seed=seed,
                          light_offset=(float(rng.uniform(-0.2, 0.2)), 0.0, float(rng.uniform(-0.2, 0.2))),
                          glass_radius=float(rng.uniform(0.1, 0.4)), mirror_radius=float(rng.uniform(0.1, 0.4)))
    pos = [base.tri_pos.astype(np.float64)]
    nrm = [base.tri_nrm.astype(np.float64)]
    model = [base.tri_model]
    mats = [base.materials]
    alb = [base.tri_diffuse] if base.tri_diffuse is not None else None
    m = base.nmodel
    for b in range(int(rng.integers(2, 6))):
        p, n = _blob(rng, int(rng.integers(4, 24)), degenerate=bool(b % 2 == 0))
        mat = _material(rng)
        pos.append(p)
        nrm.append(n)
        model.append(np.full(p.shape[0], m, np.int32))
        mats.append(mat[None, :])
        if alb is not None:
            alb.append(np.tile(mat[0:3], (p.shape[0], 1)))
        m += 1
    return scenes.Scene(np.concatenate(pos).astype(np.float32), np.concatenate(nrm).astype(np.float32),
                        np.concatenate(model).astype(np.int32), np.concatenate(mats).astype(np.float32),
                        light_model=base.light_model, light_intensity=base.light_intensity,
                        default_ior=base.default_ior,
                        tri_diffuse=None if alb is None else np.concatenate(alb).astype(np.float32))
