// pm_scan.cuh -- single-pass prefix sum with decoupled look-back.
//
// Replaces the reference's grid scan (CudaPhotonMapping/PrefixScanSum.cuh:12-279:
// a fixed 44 x 512 launch, Blelloch sweeps per block, a hand-rolled spin grid
// barrier and a serial re-scan of block sums).  Here: Merrill & Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back" (2016).  Tiles of
// 4096 elements take dynamic tile ids (so every predecessor of a running tile
// has started), publish (flag, value) in one 64-bit word, and look back a warp
// of predecessors at a time.  Every wait is bounded: after SCAN_SPIN_LIMIT polls
// the kernel records ST_TIMEOUT in the status word and finishes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pm {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr long long SCAN_SPIN_LIMIT = 1ll << 22;

// workspace bytes for a scan of n elements
inline size_t scan_workspace_bytes(int64_t n) {
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    return (size_t)(tiles + 1) * 8 + 64;
}

// exclusive (inclusive = 0) or inclusive scan of n u32 values; *total (device,
// may be null) receives the sum of all n values.  ws: scan_workspace_bytes(n).
// spin_limit: polls of one look-back wait before it gives up (ST_TIMEOUT);
// silent_tile >= 0 (test hook only) makes that tile publish nothing, so every
// later tile's look-back runs into the limit.
cudaError_t scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, uint32_t* total, void* ws,
                     unsigned* status, cudaStream_t st, long long spin_limit = SCAN_SPIN_LIMIT,
                     int silent_tile = -1);

}  // namespace pm
