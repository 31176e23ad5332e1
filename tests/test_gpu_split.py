"""The frame split over ranks with the CUDA library (photonmap/distributed.py):
two ranks reproduce the one-call frame of one context bit for bit (photon
lists, grids, image).

Both ranks run on the one GPU this test has, as two processes exchanging
through gloo (host memory): their kernels never wait on one another, the
collectives are host calls between the ranks' launches."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
S = dict(seed=11, bounces=10, gcap=400_000, ccap=20_000, W=160, H=90, k=64, r=0.1, depth=4, kc=32, rc=0.1,
         chunk=60_000)


def _camera(w):
    import photonmap
    from photonmap import scenes
    cs = scenes.default_camera(S["W"], S["H"])
    return photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)


def _scene():
    from photonmap import scenes
    return scenes.cornell(sphere_level=3, heightfield_n=64, seed=3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (os.path.join(ROOT, "cuda-photon-mapping_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import datetime
    import photonmap
    from photonmap import distributed
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ctx = photonmap.Context(0)
        ctx.set_scene(_scene())
        sf = distributed.SplitFrame(ctx, chunk=S["chunk"])
        sf.trace(S["seed"], S["bounces"], S["gcap"], S["ccap"])
        rgb, rad = sf.render(_camera(None), S["k"], S["r"], S["depth"], k_caustic=S["kc"], r_caustic=S["rc"])
        g = ctx.photons(0, sorted_=False)
        c = ctx.photons(1, sorted_=False)
        out[rank] = (g["list_pos"].cpu().numpy().tobytes(), c["list_pos"].cpu().numpy().tobytes(),
                     rgb.numpy().tobytes(), rad.numpy().tobytes(), ctx.status())
        torch.cuda.synchronize()
        ctx.close()
    finally:
        dist.destroy_process_group()


def test_split_frame_on_two_ranks_equals_one_context():
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = photonmap.Context(0)
    ctx.set_scene(_scene())
    ctx.trace_photons(S["seed"], S["bounces"], S["gcap"], S["ccap"])
    ctx.build_grid(0)
    ctx.build_grid(1)
    rgb1, rad1 = ctx.render(_camera(None), S["k"], S["r"], S["depth"], k_caustic=S["kc"], r_caustic=S["rc"])
    g1 = ctx.photons(0, sorted_=False)["list_pos"].cpu().numpy().tobytes()
    c1 = ctx.photons(1, sorted_=False)["list_pos"].cpu().numpy().tobytes()
    rgb1, rad1 = rgb1.cpu().numpy().tobytes(), rad1.cpu().numpy().tobytes()
    # the band render alone: its rows are the full frame's
    y0, y1 = 30, 61
    rgb_b, rad_b = ctx.render_rows(_camera(None), S["k"], S["r"], S["depth"], y0, y1, k_caustic=S["kc"],
                                   r_caustic=S["rc"])
    W = S["W"]
    full = np.frombuffer(rad1, np.float32).reshape(-1, 3)
    assert np.array_equal(rad_b.cpu().numpy()[y0 * W:y1 * W], full[y0 * W:y1 * W])
    ctx.close()
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        g, c, _, _, status = out[r]
        assert g == g1 and c == c1 and status == 0
    _, _, rgb, rad, _ = out[0]
    assert rgb == rgb1 and rad == rad1
