// pm_scan.cu -- decoupled look-back scan (see pm_scan.cuh).
#include <mutex>
#include "../../include/pm_api.h"
#include "pm_scan.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr unsigned long long FLAG_AGG = 1ull << 32;      // tile aggregate available
constexpr unsigned long long FLAG_PREFIX = 2ull << 32;   // inclusive prefix available
constexpr int PAD_SHIFT = 5;                              // one pad word per 32 (bank conflicts)

__device__ __forceinline__ int padded(int i) { return i + (i >> PAD_SHIFT); }

__device__ __forceinline__ void publish(unsigned long long* st, unsigned long long flag, uint32_t v) {
    *((volatile unsigned long long*)st) = flag | (unsigned long long)v;
}
__device__ __forceinline__ unsigned long long poll(const unsigned long long* st) {
    return *((volatile const unsigned long long*)st);
}

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_u32(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t n, int inclusive,
           unsigned long long* tile_state, unsigned* tile_counter, uint32_t* total, unsigned* status,
           long long spin_limit, int silent_tile) {
    __shared__ uint32_t s_items[SCAN_TILE + SCAN_TILE / 32];
    __shared__ uint32_t s_warp[SCAN_THREADS / 32];
    __shared__ uint32_t s_prefix;
    __shared__ int s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = (int)atomicAdd(tile_counter, 1u);
    __syncthreads();
    const int tile = s_tile;
    const int64_t base = (int64_t)tile * SCAN_TILE;

#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int li = i * SCAN_THREADS + tid;
        int64_t gi = base + li;
        s_items[padded(li)] = gi < n ? in[gi] : 0u;
    }
    __syncthreads();
    uint32_t v[SCAN_ITEMS];
    uint32_t tsum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = s_items[padded(tid * SCAN_ITEMS + i)];
        tsum += v[i];
    }
    // block-wide exclusive scan of the per-thread sums
    uint32_t x = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t warp_off = 0, block_total = 0;
#pragma unroll
    for (int w = 0; w < SCAN_THREADS / 32; w++) {
        uint32_t s = s_warp[w];
        if (w < warp) warp_off += s;
        block_total += s;
    }
    uint32_t thread_excl = warp_off + x - tsum;

    // decoupled look-back (warp 0)
    if (warp == 0) {
        uint32_t exclusive = 0;
        const bool speaks = tile != silent_tile;   // silent_tile: the test hook's tile that publishes nothing
        if (tile == 0) {
            if (lane == 0 && speaks) publish(tile_state + tile, FLAG_PREFIX, block_total);
        } else {
            if (lane == 0 && speaks) publish(tile_state + tile, FLAG_AGG, block_total);
            int pred = tile - 1;
            long long spins = 0;
            bool timed_out = false;
            while (true) {
                int p = pred - lane;
                unsigned long long s = FLAG_PREFIX;   // lanes before tile 0 see an empty prefix
                if (p >= 0) {
                    s = poll(tile_state + p);
                    while ((s >> 32) == 0ull) {
                        if (++spins > spin_limit) { timed_out = true; break; }
                        s = poll(tile_state + p);
                    }
                }
                if (__any_sync(0xffffffffu, timed_out)) {
                    if (lane == 0) raise_status(status, ST_TIMEOUT);
                    break;
                }
                unsigned prefix_mask = __ballot_sync(0xffffffffu, (s >> 32) == 2ull);
                uint32_t val = (uint32_t)s;
                int stop = prefix_mask ? __ffs(prefix_mask) - 1 : 31;
                uint32_t contrib = lane <= stop ? val : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
                exclusive += contrib;
                if (prefix_mask) break;
                pred -= 32;
            }
            if (lane == 0 && speaks) publish(tile_state + tile, FLAG_PREFIX, exclusive + block_total);
        }
        if (lane == 0) s_prefix = exclusive;
    }
    __syncthreads();
    const uint32_t prefix = s_prefix;
    uint32_t run = prefix + thread_excl;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        uint32_t e = v[i];
        s_items[padded(tid * SCAN_ITEMS + i)] = inclusive ? run + e : run;
        run += e;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int li = i * SCAN_THREADS + tid;
        int64_t gi = base + li;
        if (gi < n) out[gi] = s_items[padded(li)];
    }
    if (total && tid == 0 && base + SCAN_TILE >= n) *total = prefix + block_total;
}

}  // namespace

cudaError_t scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, uint32_t* total, void* ws,
                     unsigned* status, cudaStream_t st, long long spin_limit, int silent_tile) {
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, 4, st);
        return cudaSuccess;
    }
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long* state = (unsigned long long*)ws;
    unsigned* counter = (unsigned*)(state + tiles);
    cudaError_t e = cudaMemsetAsync(ws, 0, (size_t)tiles * 8 + 8, st);
    if (e != cudaSuccess) return e;
    k_scan_u32<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, inclusive, state, counter, total, status,
                                                           spin_limit, silent_tile);
    return cudaGetLastError();
}

}  // namespace pm

// ---------------------------------------------------------------------------
// Allocation-free variant of the scan (pm_scan_u32_noalloc in pm_api.h).
//
// Some callers may not allocate device memory at all: an engine that reserves
// the whole device for its own pool before loading this library, or a render
// loop that must not call cudaMalloc / cudaFree while frames are in flight
// (those calls can synchronise the device and stall other streams).  For
// them this entry point takes only the caller's input and output buffers; the
// look-back workspace (tile states, tile counter, status word) lives in a
// fixed array in the library's own device memory, which every GPU that loads
// the library holds until the process exits.
//
// Limit: n <= PM_NOALLOC_SCAN_MAX (4096 tiles of 4096 = 16,777,216 values),
// i.e. 4096 tile-state words + 2 control words = 32,784 bytes per device.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, once per device, that device current); make that
// first call before capturing a stream.  All calls share the array, which
// keeps the last call's contents, so calls whose work overlaps on the GPU (two
// streams, two host threads) race; serialise them.  Each call clears the part
// it uses (tile states, counter, status word) before launching.
namespace {

constexpr int NOALLOC_TILES = 4096;
static __device__ __align__(256) unsigned long long g_noalloc_scan_ws[NOALLOC_TILES + 2];

std::once_flag g_noalloc_once[64];
void* g_noalloc_ptr[64] = {};
cudaError_t g_noalloc_err[64] = {};

}  // namespace

extern "C" int pm_scan_u32_noalloc(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, void* stream) {
    using namespace pm;
    static_assert((int64_t)NOALLOC_TILES * SCAN_TILE == PM_NOALLOC_SCAN_MAX, "limit mismatch");
    if (n < 0 || (n > 0 && (!in || !out))) return PM_ERR_INVALID;
    if (n > PM_NOALLOC_SCAN_MAX) return PM_ERR_INVALID;                     // beyond the fixed workspace
    if (n == 0) return PM_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PM_ERR_CUDA;
    // once per device, with that device current: the device address of the array
    std::call_once(g_noalloc_once[dev], [dev]() {
        void* p = nullptr;
        g_noalloc_err[dev] = cudaGetSymbolAddress(&p, g_noalloc_scan_ws);
        g_noalloc_ptr[dev] = p;
    });
    if (g_noalloc_err[dev] != cudaSuccess || !g_noalloc_ptr[dev]) return PM_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long* state = (unsigned long long*)g_noalloc_ptr[dev];
    unsigned* counter = (unsigned*)(state + NOALLOC_TILES);
    unsigned* status = counter + 2;
    // tile states, the tile counter and the status word must start at zero
    if (cudaMemsetAsync(state, 0, (size_t)tiles * 8, st) != cudaSuccess) return PM_ERR_CUDA;
    if (cudaMemsetAsync(counter, 0, 16, st) != cudaSuccess) return PM_ERR_CUDA;
    k_scan_u32<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, inclusive, state, counter, nullptr, status,
                                                           SCAN_SPIN_LIMIT, -1);
    if (cudaGetLastError() != cudaSuccess) return PM_ERR_CUDA;
    unsigned bits = 0;
    if (cudaMemcpyAsync(&bits, status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PM_ERR_CUDA;
    return (bits & ST_TIMEOUT) ? PM_ERR_TIMEOUT : PM_OK;
}
