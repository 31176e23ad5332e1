"""Learned render: the radiance cache in the frame, with the per-tile exact-gather fallback."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def setup():
    import photonmap
    from photonmap import scenes
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = photonmap.Context(0)
    sc, cs, w = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    ctx.trace_photons(w["seed"], w["max_bounces"], w["photons"])
    ctx.build_grid(photonmap.PM_MAP_GLOBAL)
    cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
    return ctx, cam, w


def _train(ctx, cam, w, steps, seed=1):
    from photonmap import learned
    pool = learned.training_pool(ctx, cam, w["k"], w["radius"], n=1 << 18, seed=seed)
    ctx.cache_init(seed=0, lr=3e-3, out_scale=pool.scale)
    learned.cache_fit(ctx, pool, steps, batch=16384)


@pytest.mark.gpu
def test_sample_points_are_primary_hits(setup):
    ctx, cam, w = setup
    pos, nrm, wt = ctx.cache_sample_points(cam, 4096, seed=3)
    p, n, v = pos.cpu().numpy(), nrm.cpu().numpy(), wt.cpu().numpy()
    assert set(np.unique(v)) <= {0.0, 1.0} and v.mean() > 0.5
    hit = v > 0
    assert np.all(np.abs(p[hit]) <= 1.0 + 1e-3)                 # inside the room
    assert np.allclose(np.linalg.norm(n[hit], axis=1), 1.0, atol=1e-3)
    again = ctx.cache_sample_points(cam, 4096, seed=3)[0]
    assert torch.equal(again, pos)                              # seeded


@pytest.mark.gpu
def test_learned_render_exact_mode_is_the_plain_render(setup):
    ctx, cam, w = setup
    rgb_p, rad_p = ctx.render(cam, w["k"], w["radius"], w["max_depth"])
    ctx.cache_init(seed=0, out_scale=1.0)
    rgb_e, rad_e, st = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], max_rel_err=-1.0)
    assert st["fallback_tiles"] == st["tiles"]
    assert torch.equal(rgb_e, rgb_p)
    assert torch.equal(rad_e, rad_p)


@pytest.mark.gpu
def test_trained_cache_replaces_most_gathers(setup):
    ctx, cam, w = setup
    _, rad_p = ctx.render(cam, w["k"], w["radius"], w["max_depth"])
    ctx.cache_init(seed=0, out_scale=1.0)
    _, _, st0 = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], max_rel_err=0.1)
    _train(ctx, cam, w, 600)
    _, rad_l, st1 = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], max_rel_err=0.1)
    # what the trained network gains: most requests no longer need the exact gather
    assert st1["fallback_requests"] < 0.5 * st0["fallback_requests"], (st0, st1)
    # and the image stays close to the plain render
    a, b = rad_l.cpu().numpy(), rad_p.cpu().numpy()
    rel = np.abs(a - b).mean() / np.abs(b).mean()
    assert rel < 0.1, (rel, st1)


@pytest.mark.gpu
def test_noise_aware_check_still_rejects_a_wrong_cache(setup):
    """The measured frame's check (bias above 5 % by two standard errors) still
    sends the tiles of an untrained or a mis-scaled cache to the exact gather."""
    from photonmap import learned
    ctx, cam, w = setup
    S = learned.FRAME_SETTINGS
    ctx.cache_init(seed=0, out_scale=1.0)
    _, _, st0 = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
    assert st0["fallback_tiles"] > 0.5 * st0["tiles"], st0
    _train(ctx, cam, w, 600)
    _, _, st1 = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
    assert st1["fallback_tiles"] < 0.2 * st1["tiles"], st1
    # the trained network with its output doubled: a systematic 2x error everywhere lit
    params = ctx.cache_params()
    params4 = params.reshape(5, 64, 64).copy()
    params4[4] *= 2.0
    ctx.cache_set_params(params4.reshape(-1))
    _, _, st2 = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
    assert st2["fallback_tiles"] > 0.5 * st2["tiles"], st2


def _rms(x):
    return float(np.sqrt(np.mean(np.square(x))))


@pytest.mark.gpu
def test_rmse_against_fp64_oracle():
    """Plain render = the FP64 oracle's estimator (fidelity); learned vs plain
    against an FP64 reference averaged over independent photon maps."""
    import photonmap
    from photonmap import scenes
    import render64
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = photonmap.Context(0)
    sc, cs, w = scenes.workload("cornell_hf_1080p")
    W, H, photons, k, r, depth = 480, 270, 2_000_000, w["k"], w["radius"], w["max_depth"]
    cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, W, H)
    ctx.set_scene(sc)
    tables = render64.scene_tables(sc)

    def trace(seed):
        ctx.trace_photons(seed, w["max_bounces"], photons)
        ctx.build_grid(photonmap.PM_MAP_GLOBAL)
        ph = ctx.photons(photonmap.PM_MAP_GLOBAL, sorted_=False)
        return render64.PhotonMap64(ph["list_pos"].cpu().numpy(), ph["list_dir"].cpu().numpy(),
                                    ph["list_power"].cpu().numpy())

    m0 = trace(0)
    _, rad_p = ctx.render(cam, k, r, depth)
    req = {key: v.cpu().numpy() for key, v in ctx.requests().items()}
    pixels = np.arange(0, W * H, 5)

    def fp64(m):
        return render64.resolve64(req, pixels, tables,
                                  lambda q: m.estimate(req["a"][q, :3], req["b"][q, :3], k, r))

    plain = rad_p.cpu().numpy()[pixels]
    same = fp64(m0)
    fidelity = _rms(plain - same) / _rms(same)
    assert fidelity < 1e-3, fidelity
    ref = np.mean([fp64(trace(s)) for s in range(1, 5)], axis=0)
    # the learned render, its cache trained on map 0's estimates: with the
    # plain 5 % threshold and with the settings the learned frame is timed with
    from photonmap import learned as lrn
    trace(0)
    _train(ctx, cam, w, 3000)
    rmse_plain = _rms(plain - ref) / _rms(ref)
    for settings in (dict(max_rel_err=0.05), lrn.FRAME_SETTINGS):
        _, rad_l, st = ctx.render_learned(cam, k, r, depth, **settings)
        learned = rad_l.cpu().numpy()[pixels]
        rmse_learned = _rms(learned - ref) / _rms(ref)
        print(f"\nrelative RMSE vs FP64 4-map reference: plain {rmse_plain:.4f} learned {rmse_learned:.4f} "
              f"({settings}); fidelity of plain to the FP64 same-map oracle {fidelity:.2e}; fallback {st}")
        assert rmse_learned <= rmse_plain, (settings, rmse_plain, rmse_learned, st)


@pytest.mark.gpu
def test_learned_graph_render_equals_learned_render(setup):
    """The captured frame without training is pm_render_learned bit for bit."""
    from photonmap import learned
    ctx, cam, w = setup
    _train(ctx, cam, w, 300)
    S = learned.FRAME_SETTINGS
    rgb, rad, st = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
    g = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=None, steps=0, radiance=True, **S)
    try:
        for _ in range(2):                      # replays are identical
            rgb_g, rad_g, st_g = g.run(stats=True)
            assert st_g == st
            assert torch.equal(rgb_g, rgb)
            assert torch.equal(rad_g, rad)
    finally:
        g.close()


@pytest.mark.gpu
def test_learned_graph_training_follows_eager_training(setup):
    """Frames of the graph train like cache_train_steps + render_learned: the
    same pool slices, the same weights up to the order of the gradient sums."""
    from photonmap import learned
    ctx, cam, w = setup
    pool = learned.training_pool(ctx, cam, w["k"], w["radius"], n=1 << 16, seed=2)
    S = learned.FRAME_SETTINGS
    frames, steps, batch = 3, 2, 16384
    ctx.cache_init(seed=3, lr=1e-3, out_scale=pool.scale)
    w0 = ctx.cache_params()
    g = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=pool, steps=steps, batch=batch, offset=5000,
                          radiance=True, **S)
    try:
        assert np.array_equal(ctx.cache_params(), w0)   # creating the graph leaves the cache as it was
        for _ in range(frames):
            _, rad_g, _ = g.run()
        off_g = g.offset()
        w_g = ctx.cache_params()
        rad_g = rad_g.clone()
    finally:
        g.close()
    ctx.cache_init(seed=3, lr=1e-3, out_scale=pool.scale)
    assert np.array_equal(ctx.cache_params(), w0)
    off = 5000
    for _ in range(frames):
        _, off = learned.cache_fit(ctx, pool, steps, batch=batch, offset=off, want_loss=False)
        _, rad_e, _ = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
    assert off_g == off
    np.testing.assert_allclose(w_g, ctx.cache_params(), rtol=0, atol=5e-5)
    a, b = rad_g.cpu().numpy(), rad_e.cpu().numpy()
    assert np.abs(a - b).mean() <= 1e-3 * np.abs(b).mean()


@pytest.mark.gpu
def test_learned_graph_refuses_after_rebuild(setup):
    """A graph holds the scene's, the map's and the cache's device addresses and
    the grid's dimensions in its launches: after the grid is rebuilt it refuses
    to run (PM_ERR_INVALID) instead of reading replaced buffers."""
    import photonmap
    from photonmap import learned
    ctx, cam, w = setup
    S = learned.FRAME_SETTINGS
    g = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=None, steps=0, **S)
    try:
        g.run()
        ctx.build_grid(photonmap.PM_MAP_GLOBAL)
        with pytest.raises(photonmap.PMError) as e:
            g.run()
        assert e.value.code == -1   # PM_ERR_INVALID
        assert ctx.status() == 0
    finally:
        g.close()
    g = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=None, steps=0, **S)   # made again: runs
    try:
        g.run()
    finally:
        g.close()


@pytest.mark.gpu
def test_learned_graph_overlapped_training(setup):
    """overlap_training: a frame renders with the cache as the previous frames
    trained it while its own training runs beside it, i.e. render_learned, then
    cache_train_steps: the same pool slices and weights, images as the eager
    sequence's."""
    from photonmap import learned
    ctx, cam, w = setup
    pool = learned.training_pool(ctx, cam, w["k"], w["radius"], n=1 << 16, seed=4)
    S = learned.FRAME_SETTINGS
    frames, steps, batch = 3, 2, 16384
    ctx.cache_init(seed=5, lr=1e-3, out_scale=pool.scale)
    w0 = ctx.cache_params()
    g = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=pool, steps=steps, batch=batch, offset=0,
                          radiance=True, overlap_training=True, **S)
    try:
        rads = []
        for _ in range(frames):
            _, rad_g, _ = g.run()
            rads.append(rad_g.clone())
        w_g = ctx.cache_params()
        off_g = g.offset()
    finally:
        g.close()
    ctx.cache_init(seed=5, lr=1e-3, out_scale=pool.scale)   # the same start: weights, Adam state, step
    assert np.array_equal(ctx.cache_params(), w0)
    off = 0
    for f in range(frames):
        _, rad_e, _ = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **S)
        a, b = rads[f].cpu().numpy(), rad_e.cpu().numpy()
        assert np.abs(a - b).mean() <= 1e-3 * np.abs(b).mean(), f
        _, off = learned.cache_fit(ctx, pool, steps, batch=batch, offset=off, want_loss=False)
    assert off_g == off
    np.testing.assert_allclose(w_g, ctx.cache_params(), rtol=0, atol=5e-5)
