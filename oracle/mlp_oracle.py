"""CPU oracle of the learned radiance cache (test infrastructure only).

This module is the checker for the cache kernels in
cuda-photon-mapping_b200/csrc/pm_mlp.cu; nothing in the product imports it.
The reference has no learned component: the network approximates the
global-map estimate of Raytracer::get_color_from_photon_grid
(CudaPhotonMapping/Raytracer.cuh:110-138).  The restatement follows the
kernels' arithmetic contract:

  * encoding: u = (p - lo) * inv per axis; octahedral normal
    (x, y) / (|x| + |y| + |z|), folded for z < 0, mapped by 0.5 v + 0.5; each
    of the 5 values s gives sin(pi F 2^f s), cos(pi F 2^f s), f = 0..5, F = 2^octave0, in that
    order (feature 12 j + 2 f, 12 j + 2 f + 1); 4 zero features follow;
  * BF16 (round to nearest even) at the same points as the kernels: the
    encoded features, the weights, every ReLU output, the output gradient and
    every back-propagated gradient; products accumulate in FP32 (float64 here
    when ``exact`` is set);
  * layer l: h = x W_l^T, ReLU for l < 4; y = the first 3 outputs of layer 4;
    loss = sum w (y - t / out_scale)^2; d loss / d y is scaled by grad_scale.
"""
from __future__ import annotations

import numpy as np

LAYERS = 5
DIM = 64
OUT = 16
PARAMS = LAYERS * DIM * DIM


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def octahedral(n: np.ndarray) -> np.ndarray:
    n = np.asarray(n, np.float32)
    a = (np.abs(n[:, 0]) + np.abs(n[:, 1]) + np.abs(n[:, 2])).astype(np.float32)
    a = np.where(a > 0, a, np.float32(1.0)).astype(np.float32)
    ox = (n[:, 0] / a).astype(np.float32)
    oy = (n[:, 1] / a).astype(np.float32)
    sx = np.where(ox >= 0, np.float32(1.0), np.float32(-1.0))
    sy = np.where(oy >= 0, np.float32(1.0), np.float32(-1.0))
    tx = ((np.float32(1.0) - np.abs(oy)) * sx).astype(np.float32)
    ty = ((np.float32(1.0) - np.abs(ox)) * sy).astype(np.float32)
    neg = n[:, 2] < 0
    ox = np.where(neg, tx, ox)
    oy = np.where(neg, ty, oy)
    return np.stack([np.float32(0.5) * ox + np.float32(0.5), np.float32(0.5) * oy + np.float32(0.5)], 1).astype(np.float32)


def encode(pos: np.ndarray, nrm: np.ndarray, lo, inv, octave0: int = 0) -> np.ndarray:
    """(n, 64) float32 features before BF16 rounding (frequencies pi 2^(octave0 + f))."""
    pos = np.asarray(pos, np.float32)
    lo = np.asarray(lo, np.float32)
    inv = np.asarray(inv, np.float32)
    u = ((pos - lo) * inv).astype(np.float32)
    s = np.concatenate([u, octahedral(nrm)], 1)          # (n, 5)
    feats = np.zeros((pos.shape[0], DIM), np.float32)
    for j in range(5):
        for f in range(6):
            x = (s[:, j] * (np.float32(1 << octave0) * np.float32(1 << f))).astype(np.float32).astype(np.float64)
            feats[:, 12 * j + 2 * f] = np.sin(np.pi * x).astype(np.float32)
            feats[:, 12 * j + 2 * f + 1] = np.cos(np.pi * x).astype(np.float32)
    return feats


def layer_weights(params: np.ndarray):
    w = np.asarray(params)
    w = (w if w.dtype == np.float64 else w.astype(np.float32)).reshape(LAYERS, DIM, DIM)
    return [w[l, : (OUT if l == LAYERS - 1 else DIM), :] for l in range(LAYERS)]


def forward_backward(params, pos, nrm, target, weight, lo, inv, out_scale, grad_scale, exact=False):
    """Returns (y (n, 3), loss sum, grad (PARAMS,)).  exact: no BF16 rounding, float64."""
    rnd = (lambda x: np.asarray(x, np.float64)) if exact else bf16
    dt = np.float64 if exact else np.float32
    W = [rnd(w).astype(dt) for w in layer_weights(params)]
    n = pos.shape[0]
    wt = np.ones(n, dt) if weight is None else np.asarray(weight, dt)
    X = [rnd(encode(pos, nrm, lo, inv)).astype(dt)]
    for l in range(LAYERS - 1):
        h = X[l] @ W[l].T
        X.append(rnd(np.maximum(h, 0)).astype(dt))
    y = (X[-1] @ W[-1].T)[:, :3]
    d = y - np.asarray(target, dt) / dt(out_scale)
    loss = float(np.sum(wt[:, None] * d * d))
    g = dt(grad_scale) * wt
    dY = np.zeros((n, OUT), dt)
    dY[:, :3] = rnd((g[:, None] * d).astype(dt)).astype(dt)
    grads = np.zeros((LAYERS, DIM, DIM), np.float64)
    for l in range(LAYERS - 1, -1, -1):
        out = dY.shape[1]
        grads[l, :out, :] = dY.T.astype(np.float64) @ X[l].astype(np.float64)
        if l > 0:
            dX = dY @ W[l]
            dY = rnd((dX * (X[l] > 0)).astype(dt)).astype(dt)
    return y, loss, grads.reshape(-1)


def infer(params, pos, nrm, lo, inv, out_scale):
    y, _, _ = forward_backward(params, pos, nrm, np.zeros((pos.shape[0], 3), np.float32), None, lo, inv,
                               out_scale, 0.0)
    return y * np.float32(out_scale)


def init_params(seed: int) -> np.ndarray:
    """Random parameters for tests (He-uniform, padding zero); not the library's initialisation."""
    rng = np.random.default_rng(seed)
    w = np.zeros((LAYERS, DIM, DIM), np.float32)
    for l in range(LAYERS):
        fan_in = 60 if l == 0 else DIM
        outs = 3 if l == LAYERS - 1 else DIM
        b = np.sqrt(6.0 / fan_in)
        w[l, :outs, :fan_in] = rng.uniform(-b, b, (outs, fan_in))
    return w.reshape(-1)
