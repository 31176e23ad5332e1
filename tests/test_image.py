"""Headless frame output (pm_write_ppm / pm_write_pfm), the replacement of the
reference's GL pixel-buffer display (Drawer.cu:22-41, Window.cuh:88-126).

The canvas's row 0 is the bottom row (Camera.cuh:67-81), so the PPM, which
stores the top row first, holds the canvas rows in reverse; the PFM stores rows
bottom to top, in canvas order.  Host buffers are written on the CPU; device
buffers (a rendered frame) on the GPU.
"""
import numpy as np
import pytest

import photonmap
from photonmap import PMError, scenes


def _read_ppm(path):
    data = open(path, "rb").read()
    head = b"P6\n"
    assert data.startswith(head)
    dims, rest = data[len(head):].split(b"\n", 1)
    w, h = (int(v) for v in dims.split())
    maxval, body = rest.split(b"\n", 1)
    assert maxval == b"255"
    return w, h, np.frombuffer(body, np.uint8).reshape(h, w, 3)


def _read_pfm(path):
    data = open(path, "rb").read()
    head = b"PF\n"
    assert data.startswith(head)
    dims, rest = data[len(head):].split(b"\n", 1)
    w, h = (int(v) for v in dims.split())
    scale, body = rest.split(b"\n", 1)
    assert float(scale) < 0   # little-endian
    return w, h, np.frombuffer(body, "<f4").reshape(h, w, 3)


def test_ppm_rows_top_first(tmp_path):
    W, H = 5, 3
    canvas = np.arange(W * H * 3, dtype=np.uint8).reshape(H, W, 3)   # row 0 = bottom
    p = tmp_path / "f.ppm"
    photonmap.write_ppm(p, canvas, W, H)
    w, h, img = _read_ppm(p)
    assert (w, h) == (W, H)
    assert np.array_equal(img, canvas[::-1])


def test_pfm_rows_bottom_first(tmp_path):
    W, H = 4, 6
    rad = np.random.default_rng(3).random((H, W, 3), dtype=np.float32)
    p = tmp_path / "f.pfm"
    photonmap.write_pfm(p, rad, W, H)
    w, h, img = _read_pfm(p)
    assert (w, h) == (W, H)
    assert np.array_equal(img, rad)


def test_host_torch_tensors(tmp_path):
    torch = pytest.importorskip("torch")
    W, H = 3, 2
    canvas = torch.arange(W * H * 3, dtype=torch.uint8)
    photonmap.write_ppm(tmp_path / "t.ppm", canvas, W, H)
    _, _, img = _read_ppm(tmp_path / "t.ppm")
    assert np.array_equal(img, canvas.numpy().reshape(H, W, 3)[::-1])
    rad = torch.linspace(0, 1, W * H * 3, dtype=torch.float32).reshape(W * H, 3)
    photonmap.write_pfm(tmp_path / "t.pfm", rad, W, H)
    _, _, fimg = _read_pfm(tmp_path / "t.pfm")
    assert np.array_equal(fimg, rad.numpy().reshape(H, W, 3))
    with pytest.raises(PMError):
        photonmap.write_ppm(tmp_path / "t.ppm", canvas[::2], W, H)   # not contiguous


def test_errors(tmp_path):
    canvas = np.zeros(4 * 2 * 3, np.uint8)
    with pytest.raises(PMError):
        photonmap.write_ppm(tmp_path / "a.ppm", canvas, 0, 2)          # non-positive size
    with pytest.raises(PMError):
        photonmap.write_ppm(tmp_path / "a.ppm", canvas, 4, 3)          # buffer too small for 4 x 3
    with pytest.raises(PMError) as e:
        photonmap.write_ppm(tmp_path / "missing" / "a.ppm", canvas, 4, 2)   # directory does not exist
    assert e.value.code == -6
    assert photonmap.library().pm_write_ppm(b"x.ppm", None, 4, 2) == -1


@pytest.mark.gpu
def test_device_frame_round_trip(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = photonmap.Context(0)
    try:
        sc, cs, w = scenes.workload("cornell_small")
        ctx.set_scene(sc)
        W, H = 96, 64
        cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, W, H)
        ctx.trace_photons(5, 8, 40_000)
        ctx.build_grid(0)
        rgb, rad = ctx.render(cam, 32, 0.1, 4)
        torch.cuda.synchronize()
        photonmap.write_ppm(tmp_path / "d.ppm", rgb, W, H)
        photonmap.write_pfm(tmp_path / "d.pfm", rad, W, H)
        canvas = rgb.cpu().numpy().reshape(H, W, 3)
        _, _, img = _read_ppm(tmp_path / "d.ppm")
        assert np.array_equal(img, canvas[::-1])
        _, _, fimg = _read_pfm(tmp_path / "d.pfm")
        assert np.array_equal(fimg, rad.cpu().numpy().reshape(H, W, 3))
        assert canvas.any()   # the frame is not blank
    finally:
        ctx.close()
