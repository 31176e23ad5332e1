"""Learned radiance cache: the CPU oracle against finite differences, and the
tensor-core kernels (forward, backward, Adam) against the oracle."""
import numpy as np
import pytest

import mlp_oracle as mo

BOX = np.array([-1, -1, -1, 1, 1, 1], np.float32)


@pytest.fixture(scope="module")
def ctx():
    import torch
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return photonmap.Context(0)

LO = BOX[:3]
INV = np.float32(1.0) / (BOX[3:] - BOX[:3])


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    nrm = rng.standard_normal((n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    tgt = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    return pos, nrm, tgt


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e38, 1e-40], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                  # tie: to even
    assert r[2] == np.float32(1.015625)  # tie: to even (upwards)
    assert r[3] == -2.5
    assert np.isfinite(r[4])


def test_oracle_gradient_matches_finite_differences():
    pos, nrm, tgt = _samples(6, 1)
    w = mo.init_params(3).astype(np.float64)
    wt = np.linspace(0.5, 1.5, 6)
    _, loss, g = mo.forward_backward(w, pos, nrm, tgt, wt, LO, INV, 1.0, 2.0, exact=True)
    rng = np.random.default_rng(7)
    live = np.flatnonzero(g != 0)
    for idx in rng.choice(live, 24, replace=False):
        h = 1e-6
        wp = w.copy(); wp[idx] += h
        wm = w.copy(); wm[idx] -= h
        lp = mo.forward_backward(wp, pos, nrm, tgt, wt, LO, INV, 1.0, 2.0, exact=True)[1]
        lm = mo.forward_backward(wm, pos, nrm, tgt, wt, LO, INV, 1.0, 2.0, exact=True)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * max(1.0, abs(g[idx])), (idx, fd, g[idx])


def test_encoding_range():
    pos, nrm, _ = _samples(1000, 2)
    f = mo.encode(pos, nrm, LO, INV)
    assert f.shape == (1000, 64)
    assert np.all(np.abs(f[:, :60]) <= 1.0) and np.all(f[:, 60:] == 0)
    o = mo.octahedral(nrm)
    assert np.all((o >= 0) & (o <= 1))


@pytest.mark.gpu
def test_cache_gradient_matches_oracle(ctx):
    n = 40000                                   # ragged, several tiles per CTA (TMEM accumulation)
    pos, nrm, tgt = _samples(n, 11)
    wt = np.random.default_rng(5).uniform(0, 2, n).astype(np.float32)
    params = mo.init_params(21)
    ctx.cache_init(seed=1, out_scale=2.0, aabb=BOX)
    ctx.cache_set_params(params)
    g_gpu, loss_gpu = ctx.cache_gradient(pos, nrm, tgt, wt)
    _, loss_cpu, g_cpu = mo.forward_backward(params, pos, nrm, tgt, wt, LO, INV, 2.0, 2.0 / (3 * n))
    assert abs(loss_gpu - loss_cpu / (3 * n)) <= 1e-2 * (loss_cpu / (3 * n))
    g_gpu = g_gpu.reshape(5, 64, 64)
    g_cpu = g_cpu.reshape(5, 64, 64)
    for l in range(5):
        err = np.linalg.norm(g_gpu[l] - g_cpu[l]) / np.linalg.norm(g_cpu[l])
        assert err < 2e-2, (l, err)
    # padding stays untouched: layer 0 inputs 60..63 and layer 4 outputs 3..15
    assert np.all(g_gpu[0][:, 60:] == 0) and np.all(g_gpu[4][3:, :] == 0)


@pytest.mark.gpu
def test_cache_infer_matches_oracle(ctx):
    pos, nrm, _ = _samples(5000, 12)
    params = mo.init_params(22)
    ctx.cache_init(seed=1, out_scale=3.0, aabb=BOX)
    ctx.cache_set_params(params)
    y = ctx.cache_infer(pos, nrm).cpu().numpy()
    ref = mo.infer(params, pos, nrm, LO, INV, 3.0)
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err < 1e-2, err


@pytest.mark.gpu
def test_cache_training_reduces_loss(ctx):
    # a smooth radiance-like field over the box: the network must fit it
    rng = np.random.default_rng(3)

    def field(p, n):
        return np.stack([0.5 + 0.3 * np.sin(3 * p[:, 0]) * np.cos(2 * p[:, 2]),
                         0.4 + 0.2 * p[:, 1] + 0.1 * n[:, 1],
                         0.3 + 0.25 * np.cos(4 * p[:, 0] * p[:, 1])], 1).astype(np.float32)

    ctx.cache_init(seed=4, lr=5e-3, out_scale=1.0, aabb=BOX)
    first = None
    for it in range(300):
        pos, nrm, _ = _samples(16384, 100 + it)
        loss = ctx.cache_train_step(pos, nrm, field(pos, nrm))
        if first is None:
            first = loss
    pos, nrm, _ = _samples(20000, 999)
    pred = ctx.cache_infer(pos, nrm).cpu().numpy()
    mse = float(np.mean((pred - field(pos, nrm)) ** 2))
    assert mse < 0.05 * first, (first, mse)
    # the trained weights are what the library reports
    w = ctx.cache_params()
    assert np.isfinite(w).all() and np.abs(w).max() > 0


@pytest.mark.gpu
def test_train_steps_match_single_steps(ctx):
    # the multi-step entry point walks the pool like repeated single steps (wrapping at the end)
    n, b, steps = 50000, 16384, 5
    pos, nrm, tgt = _samples(n, 31)
    ctx.cache_init(seed=2, lr=1e-3, out_scale=1.0, aabb=BOX)
    off = 0
    for _ in range(steps):
        if off + b > n:
            off = 0
        ctx.cache_train_step(pos[off:off + b], nrm[off:off + b], tgt[off:off + b])
        off += b
    w_single = ctx.cache_params()
    ctx.cache_init(seed=2, lr=1e-3, out_scale=1.0, aabb=BOX)
    loss, off2 = ctx.cache_train_steps(pos, nrm, tgt, steps, b, 0, want_loss=False)
    w_multi = ctx.cache_params()
    assert off2 == off and np.isnan(loss)
    # gradient sums are atomics in arbitrary order: equal up to FP32 reassociation
    np.testing.assert_allclose(w_multi, w_single, rtol=0, atol=2e-5)
    loss, _ = ctx.cache_train_steps(pos, nrm, tgt, 1, b, off2)
    assert np.isfinite(loss) and loss > 0
