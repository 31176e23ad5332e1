// pm_grid.cu -- photon grid build.
//
// Reference: CudaPhotonMapping/PhotonGrid.cu:41-218 (analyze_density,
// count_photons_per_cell, prescan_per_cell_counts, assign_photons_to_cells).
// The reference scatters with an atomic per-cell offset, so the order inside a
// cell changes from run to run.  Here the order inside a cell is defined: by
// sub-cell (each cell split S x S x S, S chosen for the gather) and then by
// trace order, which makes the sorted arrays a pure function of the photon
// list; cell_starts / cell_sizes are the reference's exactly.  Pipeline (one stream, no host round trip except the
// re-grid decision the reference also takes on the host):
//   k_cell_count   cell id per photon (stored) + per-cell counts (atomics)
//   k_max          the largest cell count -> host decides on the re-grid
//   k_key_count    (sub-cell split S > 1) key = cell * S^3 + sub-cell + counts
//   scan_u32       exclusive scan of key counts (decoupled look-back) ->
//                  key_starts; cell_starts / cell_sizes follow exactly
//   LSD radix sort of the keys, 8 bits per pass, carrying the photon index:
//     k_radix_upsweep    per-tile digit histogram, digit-major
//     scan_u32           offsets of every (digit, tile)
//     k_radix_downsweep  stable in-tile ranks (warp match) + scatter
//   k_grid_gather  sorted photon index -> (pos, id), dir, power in slot order
#include <cmath>
#include <algorithm>
#include "pm_grid.cuh"
#include "pm_scan.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr int RADIX_THREADS = 256;
constexpr int RADIX_ITEMS = 16;
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ITEMS;
constexpr int RADIX_WARPS = RADIX_THREADS / 32;

struct GridGeom {
    float mnx, mny, mnz;
    int gx, gy, gz;
    float cell;
};

__device__ __forceinline__ uint32_t cell_of(const GridGeom& g, float px, float py, float pz) {
    int x = (int)((px - g.mnx) / g.cell);
    int y = (int)((py - g.mny) / g.cell);
    int z = (int)((pz - g.mnz) / g.cell);
    x = min(max(x, 0), g.gx - 1);
    y = min(max(y, 0), g.gy - 1);
    z = min(max(z, 0), g.gz - 1);
    return (uint32_t)(x + y * g.gx + z * g.gx * g.gy);
}

__global__ void k_cell_count(const float* __restrict__ pos, int64_t n, GridGeom g, uint32_t* __restrict__ cid,
                             uint32_t* __restrict__ counts) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = pos + 3 * i;
    uint32_t c = cell_of(g, p[0], p[1], p[2]);
    cid[i] = c;
    atomicAdd(counts + c, 1u);
}

// sub-cell key: cell * S^3 + sub-cell, the sub-cell taken from the fractional
// part of the same (p - min) / cell quotient that selects the cell
__device__ __forceinline__ int sub_of(float u, int c, int S) {
    float f = u - (float)c;
    int s = (int)(f * (float)S);
    return min(max(s, 0), S - 1);
}

__global__ void k_key_count(const float* __restrict__ pos, int64_t n, GridGeom g, int S, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ counts) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = pos + 3 * i;
    float ux = (p[0] - g.mnx) / g.cell, uy = (p[1] - g.mny) / g.cell, uz = (p[2] - g.mnz) / g.cell;
    int x = min(max((int)ux, 0), g.gx - 1);
    int y = min(max((int)uy, 0), g.gy - 1);
    int z = min(max((int)uz, 0), g.gz - 1);
    uint32_t c = (uint32_t)(x + y * g.gx + z * g.gx * g.gy);
    uint32_t sk = (uint32_t)(sub_of(ux, x, S) + S * (sub_of(uy, y, S) + S * sub_of(uz, z, S)));
    uint32_t k = c * (uint32_t)(S * S * S) + sk;
    key[i] = k;
    atomicAdd(counts + k, 1u);
}

__global__ void k_cells_from_keys(const uint32_t* __restrict__ key_starts, int64_t cells, int S3,
                                  uint32_t* __restrict__ starts, uint32_t* __restrict__ sizes) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    uint32_t a = key_starts[c * S3], b = key_starts[(c + 1) * S3];
    starts[c] = a;
    sizes[c] = b - a;
}

__global__ void k_max(const uint32_t* __restrict__ a, int64_t n, uint32_t* out) {
    uint32_t m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void __launch_bounds__(RADIX_THREADS)
k_radix_upsweep(const uint32_t* __restrict__ keys, int64_t n, int shift, uint32_t* __restrict__ hist, int tiles) {
    __shared__ uint32_t h[256];
    const int tid = threadIdx.x;
    h[tid] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RADIX_TILE;
#pragma unroll 4
    for (int i = 0; i < RADIX_ITEMS; i++) {
        int64_t gi = base + i * RADIX_THREADS + tid;
        if (gi < n) atomicAdd(&h[(keys[gi] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(int64_t)tid * tiles + blockIdx.x] = h[tid];
}

// Stable scatter of one radix pass.  A warp owns 512 consecutive keys and walks
// them 32 at a time in order; equal digits inside a step are ranked by lane with
// __match_any_sync, across steps by a per-warp running count, across warps by a
// prefix over the warps' counts.  vals_in == null means vals = index.
__global__ void __launch_bounds__(RADIX_THREADS)
k_radix_downsweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int64_t n, int shift,
                  const uint32_t* __restrict__ offsets, int tiles, uint32_t* __restrict__ keys_out,
                  uint32_t* __restrict__ vals_out) {
    __shared__ uint32_t wh[RADIX_WARPS][256];
    __shared__ uint32_t dbase[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < RADIX_WARPS * 256; i += RADIX_THREADS) (&wh[0][0])[i] = 0u;
    dbase[tid] = offsets[(int64_t)tid * tiles + blockIdx.x];
    __syncthreads();
    const int64_t wbase = (int64_t)blockIdx.x * RADIX_TILE + (int64_t)warp * (32 * RADIX_ITEMS);
    uint32_t k[RADIX_ITEMS], v[RADIX_ITEMS], r[RADIX_ITEMS];
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        int64_t gi = wbase + j * 32 + lane;
        bool valid = gi < n;
        unsigned vm = __ballot_sync(0xffffffffu, valid);
        k[j] = valid ? keys_in[gi] : 0u;
        v[j] = valid ? (vals_in ? vals_in[gi] : (uint32_t)gi) : 0u;
        r[j] = 0u;
        if (valid) {
            uint32_t d = (k[j] >> shift) & 255u;
            unsigned peers = __match_any_sync(vm, d);
            int leader = __ffs(peers) - 1;
            uint32_t old = 0u;
            if (lane == leader) {
                old = wh[warp][d];
                wh[warp][d] = old + (uint32_t)__popc(peers);
            }
            old = __shfl_sync(peers, old, leader);
            r[j] = old + (uint32_t)__popc(peers & lanemask_lt());
        }
        __syncwarp();
    }
    __syncthreads();
    {   // exclusive prefix over warps for digit tid
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RADIX_WARPS; w++) {
            uint32_t c = wh[w][tid];
            wh[w][tid] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        int64_t gi = wbase + j * 32 + lane;
        if (gi < n) {
            uint32_t d = (k[j] >> shift) & 255u;
            uint32_t p = dbase[d] + wh[warp][d] + r[j];
            if (keys_out) keys_out[p] = k[j];
            vals_out[p] = v[j];
        }
    }
}

__global__ void k_grid_gather(const uint32_t* __restrict__ order, int64_t n, const float* __restrict__ pos,
                              const float* __restrict__ dir, const float* __restrict__ pw, float4* __restrict__ gpos,
                              float* __restrict__ gdir, float* __restrict__ gpow, unsigned* status) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t s = order[j];
    if ((int64_t)s >= n) { raise_status(status, ST_BAD_INPUT); return; }
    const float* p = pos + 3 * (int64_t)s;
    gpos[j] = make_float4(p[0], p[1], p[2], __uint_as_float(s));
    const float* d = dir + 3 * (int64_t)s;
    gdir[3 * j] = d[0]; gdir[3 * j + 1] = d[1]; gdir[3 * j + 2] = d[2];
    const float* w = pw + 3 * (int64_t)s;
    gpow[3 * j] = w[0]; gpow[3 * j + 1] = w[1]; gpow[3 * j + 2] = w[2];
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void grid_dims(const float aabb[6], int64_t n, int desired, int dims[3], float* cell) {
    float sx = std::fabs(aabb[3] - aabb[0]);
    float sy = std::fabs(aabb[4] - aabb[1]);
    float sz = std::fabs(aabb[5] - aabb[2]);
    int N = (int)((n + desired - 1) / desired);
    float volume = sx * sy * sz;
    float c = std::cbrt(volume / N);
    dims[0] = (int)std::ceil(sx / c);
    dims[1] = (int)std::ceil(sy / c);
    dims[2] = (int)std::ceil(sz / c);
    *cell = c;
}

void grid_scratch_sizes(int64_t n, int64_t max_keys, size_t* hist_elems, size_t* scan_ws_bytes) {
    int64_t tiles = std::max<int64_t>(1, (n + RADIX_TILE - 1) / RADIX_TILE);
    *hist_elems = (size_t)256 * tiles;
    *scan_ws_bytes = std::max(scan_workspace_bytes((int64_t)256 * tiles), scan_workspace_bytes(max_keys + 1));
}

int grid_auto_subdiv(uint32_t max_count, int k_hint) {
    double per = (double)max_count / (2.0 * std::max(k_hint, 1));
    int S = 1;
    while (S < 8 && (double)(2 * S) * (2 * S) <= per) S *= 2;
    return S;
}

cudaError_t grid_count(GridBuffers& B, const float aabb[6], int desired, int regrid_mult, int regrid_div,
                       GridPlan* plan, cudaStream_t st) {
    cudaError_t e;
    const int64_t n = B.n;
    GridGeom g;
    g.mnx = aabb[0]; g.mny = aabb[1]; g.mnz = aabb[2];
    for (int pass = 0; pass < 2; pass++) {
        int want = pass == 0 ? desired : std::max(desired / regrid_div, 1);
        grid_dims(aabb, n, want, plan->dims, &plan->cell);
        g.gx = plan->dims[0]; g.gy = plan->dims[1]; g.gz = plan->dims[2]; g.cell = plan->cell;
        plan->cells = (int64_t)g.gx * g.gy * g.gz;
        if ((e = cudaMemsetAsync(B.cell_sizes, 0, (size_t)plan->cells * 4, st)) != cudaSuccess) return e;
        if (n > 0) {
            k_cell_count<<<blocks_for(n, 256), 256, 0, st>>>(B.pos, n, g, B.cid, B.cell_sizes);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if ((e = cudaMemsetAsync(B.small, 0, 4, st)) != cudaSuccess) return e;
        k_max<<<std::min<int64_t>(blocks_for(plan->cells, 256), 1184), 256, 0, st>>>(B.cell_sizes, plan->cells, B.small);
        uint32_t mx = 0;
        if ((e = cudaMemcpyAsync(&mx, B.small, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        plan->max_count = mx;
        if (pass == 0 && !(mx > (uint32_t)(regrid_mult * desired))) break;
    }
    return cudaSuccess;
}

cudaError_t grid_sort(GridBuffers& B, const float aabb[6], const GridPlan& plan, int S, cudaStream_t st) {
    cudaError_t e;
    const int64_t n = B.n;
    const int64_t cells = plan.cells;
    const int S3 = S * S * S;
    const int64_t keys = cells * S3;
    GridGeom g;
    g.mnx = aabb[0]; g.mny = aabb[1]; g.mnz = aabb[2];
    g.gx = plan.dims[0]; g.gy = plan.dims[1]; g.gz = plan.dims[2]; g.cell = plan.cell;
    if (S == 1) {
        // keys are the cell ids already in B.cid; counts are cell_sizes
        if ((e = scan_u32(B.cell_sizes, B.key_starts, cells, 0, B.key_starts + cells, B.scan_ws, B.status, st)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(B.cell_starts, B.key_starts, (size_t)cells * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    } else {
        if ((e = cudaMemsetAsync(B.key_counts, 0, (size_t)keys * 4, st)) != cudaSuccess) return e;
        if (n > 0) {
            k_key_count<<<blocks_for(n, 256), 256, 0, st>>>(B.pos, n, g, S, B.cid, B.key_counts);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if ((e = scan_u32(B.key_counts, B.key_starts, keys, 0, B.key_starts + keys, B.scan_ws, B.status, st)) != cudaSuccess) return e;
        k_cells_from_keys<<<blocks_for(cells, 256), 256, 0, st>>>(B.key_starts, cells, S3, B.cell_starts, B.cell_sizes);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (n == 0) return cudaSuccess;

    // LSD radix sort of the keys (stable), carrying the photon index
    int bits = 1;
    while (bits < 32 && ((uint64_t)1 << bits) < (uint64_t)keys) bits++;
    const int passes = (bits + 7) / 8;
    const int tiles = (int)((n + RADIX_TILE - 1) / RADIX_TILE);
    const uint32_t* kin = B.cid;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        const bool last = p == passes - 1;
        uint32_t* kout = last ? nullptr : B.keys[p & 1];
        uint32_t* vout = B.vals[p & 1];
        k_radix_upsweep<<<tiles, RADIX_THREADS, 0, st>>>(kin, n, shift, B.hist, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = scan_u32(B.hist, B.hist, (int64_t)256 * tiles, 0, nullptr, B.scan_ws, B.status, st)) != cudaSuccess) return e;
        k_radix_downsweep<<<tiles, RADIX_THREADS, 0, st>>>(kin, vin, n, shift, B.hist, tiles, kout, vout);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        kin = kout;
        vin = vout;
    }
    k_grid_gather<<<blocks_for(n, 256), 256, 0, st>>>(vin, n, B.pos, B.dir, B.pow, B.gpos, B.gdir, B.gpow, B.status);
    return cudaGetLastError();
}

}  // namespace pm
