"""Failure handling on the device and at the C boundary, with no GPU fault.

The reference ends the process on any CUDA error (check_cuda -> exit(99),
CudaPhotonMapping/CudaUtils.cu:6-14) and its grid scan waits on a spin barrier
with no limit (CudaPhotonMapping/CudaGridSynchronizer.cuh:13-27).  Here every
device wait is bounded and every failure is a status code:
  * a look-back wait that runs out (a predecessor tile that never publishes,
    made by the pm_debug_scan_stall test hook) ends the kernel normally and the
    call returns PM_ERR_TIMEOUT; the context stays usable;
  * an allocation the device cannot hold returns PM_ERR_OOM and leaves no half
    built map behind; the context stays usable.
Bad photon files are covered in tests/test_photon_file.py.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PM_ERR_TIMEOUT, PM_ERR_OOM = -4, -3


@pytest.fixture(scope="module")
def ctx():
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return photonmap.Context(0)


def _check_scan_works(ctx, n=100_003):
    a = np.random.default_rng(n).integers(0, 1000, n).astype(np.int32)
    out = ctx.scan_u32(torch.from_numpy(a), True).cpu().numpy().astype(np.uint32)
    assert np.array_equal(out, np.cumsum(a.astype(np.uint64)).astype(np.uint32))


def test_scan_wait_times_out_and_the_context_recovers(ctx):
    import photonmap
    x = torch.ones(3 * 4096, dtype=torch.int32)
    # no silent tile: the hook is the plain inclusive scan
    assert torch.equal(ctx.debug_scan_stall(x, 1 << 22, -1).cpu(), torch.cumsum(x, 0).to(torch.int32))
    for silent, limit in ((0, 1024), (1, 1024), (0, 1)):
        with pytest.raises(photonmap.PMError) as e:
            ctx.debug_scan_stall(x, limit, silent)
        assert e.value.code == PM_ERR_TIMEOUT
        assert ctx.status() == 0          # the status word was read and cleared
        _check_scan_works(ctx)            # kernels still run on this context


def test_allocation_failure_is_an_error_and_the_context_recovers(ctx):
    import photonmap
    from photonmap import scenes
    sc, cs, w = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    ctx.trace_photons(1, w["max_bounces"], 20_000)
    ctx.build_grid(0)
    # 2^34 photons need 3 x 206 GB of list buffers: more than the device holds
    with pytest.raises(photonmap.PMError) as e:
        ctx.trace_photons(1, w["max_bounces"], 1 << 34)
    assert e.value.code == PM_ERR_OOM
    assert ctx.photons(0, sorted_=False)["count"] == 0    # no map claims the released buffers
    with pytest.raises(photonmap.PMError):
        ctx.build_grid(0)                                  # PM_ERR_INVALID: the map is empty
    ctx.trace_photons(1, w["max_bounces"], 20_000)
    ctx.build_grid(0)
    cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, 64, 48)
    rgb, rad = ctx.render(cam, w["k"], w["radius"], w["max_depth"])
    assert rad.abs().sum().item() > 0
    assert ctx.status() == 0
