"""FP64 oracle of the global-map radiance estimate and the per-pixel resolve
(test infrastructure only: the checker of the plain and learned renders).

Follows the reference's CPU path in double precision on given eye-path hits:
  * neighbours: the k nearest photons with distance <= r
    (CudaPhotonMapping/PhotonGrid.cu:222-284, PhotonMaxHeap.cuh:43-127), by
    scipy's cKDTree;
  * estimate: r_k = the largest selected distance, sum over photons with
    dot(n, -dir) > 0 of power * alpha (1 - (1 - e^(-beta d^2 / (2 r_k^2))) /
    (1 - e^(-beta))), alpha = 1.818, beta = 1.953, times 1 / (pi r_k^2)
    (CudaPhotonMapping/Raytracer.cuh:110-138);
  * resolve: per hit, emission + 4 albedo opaque estimate, clamped to <= 1 per
    channel, times the path weight, summed over the pixel's hits
    (CudaPhotonMapping/Raytracer.cuh:187-211).
The hits (eye-path requests) come from the product's eye pass, whose own
parity with the reference is tested elsewhere; caustic estimates are not
restated here (the workloads that use this FP64 render build no caustic map).
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

ALPHA, BETA = 1.818, 1.953


class PhotonMap64:
    def __init__(self, pos, direction, power):
        self.pos = np.asarray(pos, np.float64).reshape(-1, 3)
        self.dir = np.asarray(direction, np.float64).reshape(-1, 3)
        self.pow = np.asarray(power, np.float64).reshape(-1, 3)
        self.tree = cKDTree(self.pos, leafsize=32, balanced_tree=False, compact_nodes=False)

    def estimate(self, qpos, qnrm, k, r):
        qpos = np.asarray(qpos, np.float64).reshape(-1, 3)
        qnrm = np.asarray(qnrm, np.float64).reshape(-1, 3)
        out = np.zeros((qpos.shape[0], 3))
        if qpos.shape[0] == 0:
            return out
        d, idx = self.tree.query(qpos, k=k, distance_upper_bound=r * (1 + 1e-12), workers=-1)
        d = d.reshape(qpos.shape[0], -1)
        idx = idx.reshape(qpos.shape[0], -1)
        valid = np.isfinite(d)
        safe = np.where(valid, idx, 0)
        rk = np.where(valid, d, 0.0).max(axis=1)
        cos = -np.einsum("qkc,qc->qk", self.dir[safe], qnrm)
        use = valid & (cos > 0)
        fr = np.where(rk > 0, rk * rk, 1.0)[:, None]
        filt = ALPHA * (1 - (1 - np.exp(-BETA * d * d / (2 * fr))) / (1 - np.exp(-BETA)))
        filt = np.where(use, filt, 0.0)
        acc = np.einsum("qk,qkc->qc", filt, self.pow[safe])
        norm = np.where(rk > 0, 1.0 / (np.pi * rk * rk), 0.0)
        return acc * norm[:, None]


def estimate_ids(pos, direction, power, qpos, qnrm, ids, cnt):
    """FP64 estimate of get_color_from_photon_grid (CudaPhotonMapping/Raytracer.cuh:110-138)
    over given neighbour sets: ids[i, :cnt[i]] index the photon arrays (the
    oracle's kNN selection); r_k is the largest neighbour distance, in FP64."""
    qpos = np.asarray(qpos, np.float64).reshape(-1, 3)
    qnrm = np.asarray(qnrm, np.float64).reshape(-1, 3)
    ids = np.asarray(ids)
    k = ids.shape[1]
    valid = np.arange(k)[None, :] < np.asarray(cnt)[:, None]
    safe = np.where(valid, ids, 0).astype(np.int64)
    p = np.asarray(pos, np.float32)[safe].astype(np.float64)
    d = np.sqrt(((p - qpos[:, None, :]) ** 2).sum(-1))
    d = np.where(valid, d, 0.0)
    rk = d.max(axis=1)
    cos = -np.einsum("qkc,qc->qk", np.asarray(direction, np.float32)[safe].astype(np.float64), qnrm)
    use = valid & (cos > 0)
    fr = np.where(rk > 0, rk * rk, 1.0)[:, None]
    filt = ALPHA * (1 - (1 - np.exp(-BETA * d * d / (2 * fr))) / (1 - np.exp(-BETA)))
    filt = np.where(use, filt, 0.0)
    acc = np.einsum("qk,qkc->qc", filt, np.asarray(power, np.float32)[safe].astype(np.float64))
    norm = np.where(rk > 0, 1.0 / (np.pi * rk * rk), 0.0)
    return acc * norm[:, None]


def resolve_hits(hits, tables, est_global):
    """FP64 radiance per pixel from its eye-path hits (records a, b, c and
    counts per pixel, as Oracle scene eye_hits returns them); est_global(hit
    indices) -> (m, 3) FP64 estimates of those hits."""
    counts = np.asarray(hits["counts"], np.int64)
    base = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32)
    req = dict(a=hits["a"], b=hits["b"], c=hits["c"], px_base=base, px_count=counts.astype(np.int32))
    return resolve64(req, np.arange(counts.size), tables, est_global)


def scene_tables(scene):
    """Per-triangle albedo, opaque and emission arrays of a photonmap.scenes.Scene."""
    mats = np.asarray(scene.materials, np.float64)
    tm = np.asarray(scene.tri_model)
    alb = (np.asarray(scene.tri_diffuse, np.float64) if scene.tri_diffuse is not None else mats[tm, 0:3])
    return alb, mats[tm, 10], mats[tm, 6:9]


def resolve64(req, pixels, tables, est_global):
    """FP64 radiance of the given pixels from their requests.

    req: dict of numpy arrays a, b, c (n, 4) float32, px_base, px_count (npx,) int32.
    est_global(q_indices) -> (m, 3) float64 estimates of those requests.
    """
    alb, opq, emi = tables
    pixels = np.asarray(pixels, np.int64)
    base = req["px_base"][pixels].astype(np.int64)
    cnt = req["px_count"][pixels].astype(np.int64)
    owner = np.repeat(np.arange(pixels.size), cnt)
    q = np.repeat(base, cnt) + (np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    a, b, c = req["a"][q], req["b"][q], req["c"][q]
    tri = a[:, 3].copy().view(np.int32).astype(np.int64)
    flags = b[:, 3].copy().view(np.uint32)
    color = emi[tri].copy()
    g = (flags & 1) != 0
    if g.any():
        est = est_global(q[g])
        color[g] += 4.0 * alb[tri[g]] * opq[tri[g], None] * est
    color = np.minimum(color, 1.0)
    contrib = color * c[:, 0:3].astype(np.float64)
    out = np.zeros((pixels.size, 3))
    np.add.at(out, owner, contrib)
    return out
