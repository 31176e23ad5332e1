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
    pos, nrm, wt = ctx.cache_sample_points(cam, 1 << 18, seed=seed)
    lab, _, _ = ctx.gather(pos, nrm, w["k"], w["radius"])
    scale = float(lab[wt > 0].mean())
    ctx.cache_init(seed=0, lr=3e-3, out_scale=scale)
    b = 16384
    for it in range(steps):
        s = (it * b) % pos.shape[0]
        ctx.cache_train_step(pos[s:s + b], nrm[s:s + b], lab[s:s + b], wt[s:s + b])


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
