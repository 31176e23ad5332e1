// pm_scan.cu -- decoupled look-back scan (see pm_scan.cuh).
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
           unsigned long long* tile_state, unsigned* tile_counter, uint32_t* total, unsigned* status) {
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
        if (tile == 0) {
            if (lane == 0) publish(tile_state + tile, FLAG_PREFIX, block_total);
        } else {
            if (lane == 0) publish(tile_state + tile, FLAG_AGG, block_total);
            int pred = tile - 1;
            long long spins = 0;
            bool timed_out = false;
            while (true) {
                int p = pred - lane;
                unsigned long long s = FLAG_PREFIX;   // lanes before tile 0 see an empty prefix
                if (p >= 0) {
                    s = poll(tile_state + p);
                    while ((s >> 32) == 0ull) {
                        if (++spins > SCAN_SPIN_LIMIT) { timed_out = true; break; }
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
            if (lane == 0) publish(tile_state + tile, FLAG_PREFIX, exclusive + block_total);
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
                     unsigned* status, cudaStream_t st) {
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, 4, st);
        return cudaSuccess;
    }
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long* state = (unsigned long long*)ws;
    unsigned* counter = (unsigned*)(state + tiles);
    cudaError_t e = cudaMemsetAsync(ws, 0, (size_t)tiles * 8 + 8, st);
    if (e != cudaSuccess) return e;
    k_scan_u32<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, inclusive, state, counter, total, status);
    return cudaGetLastError();
}

}  // namespace pm
