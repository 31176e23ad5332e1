"""The allocation-free scan entry point (pm_scan_u32_noalloc).

It exists for callers that may not allocate device memory themselves -- hosts
that hand the whole device to their own pool, or frame loops that must not call
cudaMalloc / cudaFree while work is in flight.  Its workspace is a fixed array
inside the library.  The test calls it through the C ABI twice in a row and
compares each result with the allocating scan (pm_scan_u32) bit for bit.  This
file is collected last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _noalloc():
    from photonmap import core
    fn = core.library().pm_scan_u32_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_scan_matches_allocating_scan_on_consecutive_calls():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import photonmap
    fn = _noalloc()
    ctx = photonmap.Context(0)
    rng = np.random.default_rng(2024)
    # two calls in a row per size; the second reuses the array the first left behind
    for n in (1_000_003, 4097, 4096 * 4096):
        a = rng.integers(0, 200, n).astype(np.int32)
        x = torch.from_numpy(a).cuda()
        for inclusive in (1, 0):
            ref = ctx.scan_u32(x, inclusive)
            for _ in range(2):
                out = torch.full_like(x, -1)
                torch.cuda.synchronize()
                assert fn(x.data_ptr(), out.data_ptr(), n, inclusive, None) == 0
                assert torch.equal(out, ref)
    want = np.cumsum(a.astype(np.uint64)).astype(np.uint32)
    assert np.array_equal(out.cpu().numpy().astype(np.uint32)[1:], want[:-1])
    ctx.close()


def test_noalloc_scan_rejects_sizes_beyond_its_array():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fn = _noalloc()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    # the size is checked before anything touches the buffers
    assert fn(x.data_ptr(), x.data_ptr(), 4096 * 4096 + 1, 1, None) == -1
    assert fn(x.data_ptr(), x.data_ptr(), -1, 1, None) == -1
    assert fn(x.data_ptr(), x.data_ptr(), 0, 1, None) == 0
