"""The frame split over ranks (photonmap/distributed.py) reproduces the
one-rank frame bit for bit: the photon lists (path shards, all-gathered and cut
at capacity in canonical order), the grids and the image (pixel-row bands).

On the CPU the ranks are gloo processes and each rank's renderer is the
oracle (tests only: it stands in for the CUDA library, so that what is tested
here is the split's host logic: path ranges per round, the exchanges, the
capacity cut, the bands).  tests/test_gpu_split.py runs the same split with
the CUDA library."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SETUP = dict(seed=7, bounces=8, gcap=20_000, ccap=1_500, W=48, H=36, k=40, r=0.15, depth=4, kc=16, rc=0.2,
             chunk=3_000)


class OracleEngine:
    """The per-rank renderer of the split, on the oracle (CPU)."""

    def __init__(self, sc):
        from oracle import Oracle
        self.orc = Oracle()
        self.s = self.orc.scene(sc)
        self.light_intensity = np.asarray(sc.light_intensity, np.float32)
        self.lists, self.grids = {}, {}

    def trace_paths(self, seed, max_bounces, power_capacity, p0, p1, tag=0):
        return self.s.trace_paths(seed, max_bounces, power_capacity, p0, p1, tag=tag)

    def set_photons(self, map_id, pos, power, direction):
        self.lists[map_id] = tuple(np.ascontiguousarray(np.asarray(a), np.float32) for a in (pos, power, direction))

    def build_grid(self, map_id):
        pos, pw, dr = self.lists[map_id]
        self.grids[map_id] = self.orc.grid_build(pos, pw, dr, self.s.aabb())

    def render_rows(self, cam, k, r, max_depth, y0, y1, k_caustic=0, r_caustic=0.2):
        W, H = cam.width, cam.height
        c = self.grids.get(1) if k_caustic > 0 else None
        out = self.s.render(self.orc.camera(cam), W, H, self.grids[0], k, r, max_depth, y0=y0, y1=y1, c=c,
                            k_c=k_caustic, r_c=r_caustic)
        rgb = np.zeros((H * W, 3), np.uint8)
        rad = np.zeros((H * W, 3), np.float32)
        rgb[y0 * W:y1 * W] = out["rgb8"]
        rad[y0 * W:y1 * W] = out["radiance"]
        return rgb.reshape(-1), rad


def _frame(engine, S):
    from photonmap import distributed, scenes
    sf = distributed.SplitFrame(engine, chunk=S["chunk"])
    paths = sf.trace(S["seed"], S["bounces"], S["gcap"], S["ccap"])
    cam = scenes.default_camera(S["W"], S["H"])
    rgb, rad = sf.render(cam, S["k"], S["r"], S["depth"], k_caustic=S["kc"], r_caustic=S["rc"])
    lists = {m: engine.lists[m] for m in engine.lists}
    return paths, lists, np.asarray(rgb), np.asarray(rad)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (os.path.join(ROOT, "cuda-photon-mapping_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import datetime
    from photonmap import scenes
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sc, _, _ = scenes.workload("cornell_small")
        paths, lists, rgb, rad = _frame(OracleEngine(sc), SETUP)
        out[rank] = (paths, {m: tuple(a.tobytes() for a in v) for m, v in lists.items()}, rgb.tobytes(),
                     rad.tobytes())
    finally:
        dist.destroy_process_group()


def test_split_frame_two_ranks_equals_one_rank(orc):
    from photonmap import scenes
    sc, _, _ = scenes.workload("cornell_small")
    # one rank (no process group): the reference result
    paths1, lists1, rgb1, rad1 = _frame(OracleEngine(sc), SETUP)
    # its photon lists are the oracle's own one-call photon pass
    tr = orc.scene(sc).trace_photons(SETUP["seed"], SETUP["bounces"], SETUP["gcap"], SETUP["ccap"])
    assert np.array_equal(lists1[0][0], tr["g_pos"]) and np.array_equal(lists1[0][2], tr["g_dir"])
    assert np.array_equal(lists1[0][1], tr["g_pow"])
    assert np.array_equal(lists1[1][0], tr["c_pos"]) and np.array_equal(lists1[1][1], tr["c_pow"])
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        paths, lists, rgb, rad = out[r]
        for m in (0, 1):   # every rank holds the one-rank photon lists
            assert lists[m] == tuple(a.tobytes() for a in lists1[m])
    _, _, rgb, rad = out[0]  # the gathered frame on rank 0
    assert rgb == rgb1.tobytes() and rad == rad1.tobytes()
    assert rgb1.reshape(-1, 3).max() > 0


def test_bands_cover_the_frame_once():
    from photonmap.distributed import band
    for H in (1, 7, 36, 1080):
        for world in (1, 2, 3, 8):
            rows = [band(H, r, world) for r in range(world)]
            assert rows[0][0] == 0 and rows[-1][1] == H
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
            assert max(y1 - y0 for y0, y1 in rows) - min(y1 - y0 for y0, y1 in rows) <= 1
