"""Batched form: many instances per frame through one work queue per stage,
replayed from a CUDA graph, against single-instance renders of each instance."""
import pytest

torch = pytest.importorskip("torch")


def _instances(n, seed, **kw):
    import photonmap
    from photonmap import scenes
    out = []
    for d in scenes.batch_instances(n=n, seed=seed, **kw):
        cs = d.pop("camera_spec")
        d["camera"] = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
        out.append(d)
    return out


def _single(inst, frame=0):
    import photonmap
    ctx = photonmap.Context(0)
    ctx.set_scene(inst["scene"])
    ctx.trace_photons(inst["seed"] + frame, inst["max_bounces"], inst["photons"])
    ctx.build_grid(photonmap.PM_MAP_GLOBAL)
    rgb, _ = ctx.render(inst["camera"], inst["k"], inst["radius"], inst["max_depth"], radiance=False)
    c = inst["camera"]
    return rgb.reshape(c.height, c.width, 3)


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_batch_equals_single_instance_renders(gpu):
    import photonmap
    insts = _instances(5, seed=7, photons_range=(10_000, 120_000), res_range=(64, 160))
    b = photonmap.Batch(insts, autotune=False, use_graph=True)
    b.frame(0)
    info = b.info()
    assert info["graph"] == 1 and info["underfilled"] == 0 and info["instances"] == 5
    assert info["photons_last_frame"] == sum(i["photons"] for i in insts)
    imgs = [b.image(i) for i in range(5)]
    for i, inst in enumerate(insts):
        assert torch.equal(imgs[i], _single(inst)), i
    # replaying the graph reproduces the frame
    b.frame(0)
    for i in range(5):
        assert torch.equal(b.image(i), imgs[i])
    b.close()


@pytest.mark.gpu
def test_batch_graph_equals_eager_on_new_frames(gpu):
    import photonmap
    insts = _instances(4, seed=11, photons_range=(10_000, 60_000), res_range=(48, 96), ks=(32, 128))
    g = photonmap.Batch(insts, autotune=False, use_graph=True)
    e = photonmap.Batch(insts, autotune=False, use_graph=False)
    assert g.info()["graph"] == 1 and e.info()["graph"] == 0
    for f in (1, 2):
        g.frame(f)
        e.frame(f)
        for i in range(4):
            assert torch.equal(g.image(i), e.image(i)), (f, i)
    # frame f traces the streams seeded with seed + f, as a single-instance render does
    for i, inst in enumerate(insts):
        assert torch.equal(g.image(i), _single(inst, frame=2)), i
    g.close()
    e.close()


@pytest.mark.gpu
def test_batch_autotuned(gpu):
    import photonmap
    insts = _instances(4, seed=3, photons_range=(20_000, 100_000), res_range=(64, 128))
    b = photonmap.Batch(insts, autotune=True, use_graph=True)
    info = b.info()
    assert info["desired_per_cell"] in (125, 250, 500, 1000, 2000)
    assert info["subcell_khint"] in (0.0, 0.25, 1.0, 4.0)
    assert info["gather_warps"] in (4, 8) and info["trace_refill"] in (4, 8, 16)
    assert info["gather_guess"] in (0.0, 1.5, 2.0, 3.0)
    b.frame(0)
    for i, inst in enumerate(insts):
        a = b.image(i).to(torch.int32)
        ref = _single(inst).to(torch.int32)
        # another cell size changes only the float summation order of the estimates
        assert int((a - ref).abs().max()) <= 1, i
        assert float((a != ref).float().mean()) < 0.01, i
    b.close()


@pytest.mark.gpu
def test_batch_instances_against_the_oracle(gpu, orc):
    """Two batch instances (jittered light, random sphere radii) against the
    oracle's own photon pass, grid and render of them: the photon lists bit
    for bit, 8-bit pixels at most one level apart (the estimates differ only
    by CUDA's expf / powf)."""
    import numpy as np
    import photonmap
    from photonmap import scenes
    insts = _instances(2, seed=21, photons_range=(20_000, 60_000), res_range=(64, 96))
    b = photonmap.Batch(insts, autotune=False, use_graph=True)
    b.frame(3)
    for i, inst in enumerate(insts):
        s = orc.scene(inst["scene"])
        tr = s.trace_photons(inst["seed"] + 3, inst["max_bounces"], inst["photons"])
        ph = {k: v.cpu().numpy() for k, v in b.photons(i).items()}
        assert ph["pos"].shape[0] == inst["photons"] == tr["g_pos"].shape[0]
        for k, o in (("pos", "g_pos"), ("power", "g_pow"), ("dir", "g_dir")):
            assert np.array_equal(ph[k].view(np.uint32), np.ascontiguousarray(tr[o], np.float32).view(np.uint32)), (i, k)
        g = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], s.aabb())
        c = inst["camera"]
        cs = scenes.default_camera(c.width, c.height)
        out = s.render(orc.camera(cs), c.width, c.height, g, inst["k"], inst["radius"], inst["max_depth"])
        img = b.image(i).cpu().numpy().reshape(-1, 3).astype(int)
        d = np.abs(img - out["rgb8"].astype(int))
        assert d.max() <= 1, i
        assert (d != 0).mean() < 0.01, i
        assert img.max() > 0
    b.close()
