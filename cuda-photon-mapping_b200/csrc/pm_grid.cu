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
//   k_count_cells  per-cell counts of both candidate grids (the desired
//                  resolution and the re-grid one) and their largest counts
//                  (shared-memory counters + k_count_max when both grids fit)
//                  -> host decides on the re-grid and on S
//   k_key_count    key = cell * S^3 + sub-cell per photon + key counts
//   scan_u32       exclusive scan of key counts (decoupled look-back) ->
//                  key_starts; cell_starts / cell_sizes follow exactly
//   LSD radix sort of the keys, <= 9 bits per pass, carrying the photon index:
//     k_radix_upsweep    per-tile digit histogram, digit-major
//     scan_u32           offsets of every (digit, tile)
//     k_radix_downsweep  stable in-tile ranks (per-bit ballots) + scatter
//   k_grid_gather  sorted photon index -> (pos, id), dir, power in slot order
#include <cmath>
#include <algorithm>
#include "pm_grid.cuh"
#include "pm_scan.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

// 512 threads of 8 keys per tile (3 blocks, 48 warps per SM): grid build
// 1.10 -> 1.03 ms per 10M photons against 256 x 16 (4 blocks, 32 warps) and
// 256 x 8 (5 or 6 blocks, 1.07 ms); the ranking and staging phases are
// latency bound, so more resident warps per SM pay.  RADIX_THREADS <=
// RADIX_MAX_BINS (each thread owns whole bins in the downsweep's prefix).
constexpr int RADIX_THREADS = 512;
constexpr int RADIX_ITEMS = 8;
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ITEMS;
constexpr int RADIX_WARPS = RADIX_THREADS / 32;
constexpr int RADIX_MAX_BITS = 9;
constexpr int RADIX_MAX_BINS = 1 << RADIX_MAX_BITS;

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

// Shared-memory variant of k_count_cells for grids whose cells fit in shared
// memory as 16-bit counters (two per 32-bit word; a block counts at most
// COUNT_CHUNK <= 65535 photons, so a half-word never carries into its
// neighbour).  Photons land on a few thousand hot surface cells, so global
// atomics on the cell counters contend; here each block adds into its own
// copy and flushes its non-zero counters once.
constexpr int COUNT_THREADS = 1024;
constexpr int COUNT_CHUNK = 65535;
constexpr int COUNT_SMEM_WORDS = 56 * 1024;   // 224 KB: 114,688 16-bit counters

// Photons [blockIdx.x * chunk, ... + chunk) (chunk <= COUNT_CHUNK, so no
// 16-bit counter can overflow).
__global__ void __launch_bounds__(COUNT_THREADS)
k_count_cells_smem(const float* __restrict__ pos, int64_t n, int64_t chunk, GridGeom ga, GridGeom gb, int two,
                   int cells_a, int cells_b, uint32_t* __restrict__ ca, uint32_t* __restrict__ cb) {
    extern __shared__ uint32_t h16[];
    const int words_a = (cells_a + 1) >> 1, words = words_a + (two ? (cells_b + 1) >> 1 : 0);
    for (int i = threadIdx.x; i < words; i += COUNT_THREADS) h16[i] = 0u;
    __syncthreads();
    const int64_t first = (int64_t)blockIdx.x * chunk;
    const int64_t last = min(first + chunk, n);
    for (int64_t i = first + threadIdx.x; i < last; i += COUNT_THREADS) {
        const float* p = pos + 3 * i;
        const float x = p[0], y = p[1], z = p[2];
        const uint32_t c = cell_of(ga, x, y, z);
        atomicAdd(&h16[c >> 1], 1u << (16 * (c & 1u)));
        if (two) {
            const uint32_t c2 = cell_of(gb, x, y, z);
            atomicAdd(&h16[words_a + (c2 >> 1)], 1u << (16 * (c2 & 1u)));
        }
    }
    __syncthreads();
    for (int w = threadIdx.x; w < words; w += COUNT_THREADS) {
        const uint32_t v = h16[w];
        if (!v) continue;
        const bool in_a = w < words_a;
        uint32_t* dst = in_a ? ca : cb;
        const int cell = 2 * (in_a ? w : w - words_a);
        if (v & 0xffffu) atomicAdd(dst + cell, v & 0xffffu);
        if (v >> 16) atomicAdd(dst + cell + 1, v >> 16);
    }
}

// largest counts of the two count arrays: mx[0] (a), mx[1] (b)
__global__ void k_count_max(const uint32_t* __restrict__ ca, int64_t na, const uint32_t* __restrict__ cb, int64_t nb,
                            uint32_t* mx) {
    uint32_t ma = 0u, mb = 0u;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += stride) ma = max(ma, ca[i]);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += stride) mb = max(mb, cb[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ma = max(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (ma) atomicMax(mx, ma);
        if (mb) atomicMax(mx + 1, mb);
    }
}

// photon counts of grid a and (when two) grid b; mx[0], mx[1] = largest counts
__global__ void k_count_cells(const float* __restrict__ pos, int64_t n, GridGeom ga, GridGeom gb, int two,
                              uint32_t* __restrict__ ca, uint32_t* __restrict__ cb, uint32_t* mx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t ma = 0u, mb = 0u;
    if (i < n) {
        const float* p = pos + 3 * i;
        const float x = p[0], y = p[1], z = p[2];
        ma = atomicAdd(ca + cell_of(ga, x, y, z), 1u) + 1u;
        if (two) mb = atomicAdd(cb + cell_of(gb, x, y, z), 1u) + 1u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ma = max(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (ma) atomicMax(mx, ma);
        if (mb) atomicMax(mx + 1, mb);
    }
}

// sub-cell key: cell * S^3 + sub-cell, the sub-cell taken from the fractional
// part of the same (p - min) / cell quotient that selects the cell
__device__ __forceinline__ int sub_of(float u, int c, int S) {
    float f = u - (float)c;
    int s = (int)(f * (float)S);
    return min(max(s, 0), S - 1);
}

__device__ __forceinline__ uint32_t sub_cell_key(const GridGeom& g, int S, const float* p) {
    float ux = (p[0] - g.mnx) / g.cell, uy = (p[1] - g.mny) / g.cell, uz = (p[2] - g.mnz) / g.cell;
    int x = min(max((int)ux, 0), g.gx - 1);
    int y = min(max((int)uy, 0), g.gy - 1);
    int z = min(max((int)uz, 0), g.gz - 1);
    uint32_t c = (uint32_t)(x + y * g.gx + z * g.gx * g.gy);
    uint32_t sk = (uint32_t)(sub_of(ux, x, S) + S * (sub_of(uy, y, S) + S * sub_of(uz, z, S)));
    return c * (uint32_t)(S * S * S) + sk;
}

__global__ void k_key_count(const float* __restrict__ pos, int64_t n, GridGeom g, int S, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ counts) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = sub_cell_key(g, S, pos + 3 * i);
    key[i] = k;
    atomicAdd(counts + k, 1u);
}

__device__ __forceinline__ int find_range(const int64_t* __restrict__ off, int n, int64_t v) {
    int lo = 0, hi = n - 1;   // last i with off[i] <= v
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Several instances in one key space: photon p of instance i's region (the
// first min(cap, filled) of its slots are photons) gets key key0 + its
// sub-cell key in the instance's grid; other slots get `sentinel`.
__global__ void k_key_count_multi(const float* __restrict__ pos, int64_t n, const GridInstDev* __restrict__ tab,
                                  const int64_t* __restrict__ ph_off, int ninst, const int64_t* __restrict__ filled,
                                  uint32_t sentinel, uint32_t* __restrict__ key, uint32_t* __restrict__ counts) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int i = find_range(ph_off, ninst, p);
    const GridInstDev t = tab[i];
    const int64_t local = p - t.ph0;
    uint32_t k = sentinel;
    if (local < min(t.cap, filled[i])) {
        GridGeom g;
        g.mnx = t.mn[0]; g.mny = t.mn[1]; g.mnz = t.mn[2];
        g.gx = t.gx; g.gy = t.gy; g.gz = t.gz; g.cell = t.cell;
        k = (uint32_t)t.key0 + sub_cell_key(g, t.S, pos + 3 * p);
    }
    key[p] = k;
    atomicAdd(counts + k, 1u);
}

// per global cell: the instance-relative start and size of its photons
__global__ void k_cells_multi(int64_t cells, const GridInstDev* __restrict__ tab, const int64_t* __restrict__ cell_off,
                              int ninst, const uint32_t* __restrict__ key_starts, uint32_t* __restrict__ starts,
                              uint32_t* __restrict__ sizes) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    const int i = find_range(cell_off, ninst, c);
    const GridInstDev t = tab[i];
    const int64_t S3 = (int64_t)t.S * t.S * t.S;
    const int64_t lc = c - t.cell0;
    const uint32_t base = key_starts[t.key0];
    const uint32_t a = key_starts[t.key0 + lc * S3], b = key_starts[t.key0 + (lc + 1) * S3];
    starts[c] = a - base;
    sizes[c] = b - a;
}

__global__ void k_cells_from_keys(const uint32_t* __restrict__ key_starts, int64_t cells, int S3,
                                  uint32_t* __restrict__ starts, uint32_t* __restrict__ sizes) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    uint32_t a = key_starts[c * S3], b = key_starts[(c + 1) * S3];
    starts[c] = a;
    sizes[c] = b - a;
}

__global__ void __launch_bounds__(RADIX_THREADS)
k_radix_upsweep(const uint32_t* __restrict__ keys, int64_t n, int shift, int bits, uint32_t* __restrict__ hist,
                int tiles) {
    __shared__ uint32_t h[RADIX_MAX_BINS];
    const int tid = threadIdx.x, bins = 1 << bits;
    const uint32_t dm = (uint32_t)bins - 1u;
    for (int b = tid; b < bins; b += RADIX_THREADS) h[b] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RADIX_TILE;
#pragma unroll 4
    for (int i = 0; i < RADIX_ITEMS; i++) {
        int64_t gi = base + i * RADIX_THREADS + tid;
        if (gi < n) atomicAdd(&h[(keys[gi] >> shift) & dm], 1u);
    }
    __syncthreads();
    for (int b = tid; b < bins; b += RADIX_THREADS) hist[(int64_t)b * tiles + blockIdx.x] = h[b];
}

// Stable scatter of one radix pass.  A warp owns 256 consecutive keys and walks
// them 32 at a time in order; equal digits inside a step are ranked by lane
// (the lanes of a digit found by one ballot per digit bit: grid build 1.14 ->
// 1.10 ms against __match_any_sync), across steps by a per-warp running
// count, across warps by a
// prefix over the warps' counts.  The tile is then staged in shared memory in
// digit order, so that consecutive threads write consecutive slots of each
// digit's output run (coalesced) instead of one scattered word per key.
// vals_in == null means vals = index.
struct RadixSmem {
    uint32_t wh[RADIX_WARPS][RADIX_MAX_BINS];   // per-warp digit counts, then warp offsets
    uint32_t dbase[RADIX_MAX_BINS];             // global start of the tile's run of each digit
    uint32_t lbase[RADIX_MAX_BINS];             // start of each digit inside the staged tile
    uint32_t wsum[RADIX_WARPS];
    uint32_t key[RADIX_TILE];
    uint32_t val[RADIX_TILE];
};

__global__ void __launch_bounds__(RADIX_THREADS, 3)   // 3 blocks per SM: the shared-memory limit
k_radix_downsweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int64_t n, int shift,
                  int bits, const uint32_t* __restrict__ offsets, int tiles, uint32_t* __restrict__ keys_out,
                  uint32_t* __restrict__ vals_out) {
    extern __shared__ __align__(16) unsigned char radix_smem[];
    RadixSmem& R = *reinterpret_cast<RadixSmem*>(radix_smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, bins = 1 << bits;
    const uint32_t dm = (uint32_t)bins - 1u;
    for (int i = tid; i < RADIX_WARPS * RADIX_MAX_BINS; i += RADIX_THREADS) (&R.wh[0][0])[i] = 0u;
    for (int b = tid; b < bins; b += RADIX_THREADS) R.dbase[b] = offsets[(int64_t)b * tiles + blockIdx.x];
    __syncthreads();
    const int64_t tbase = (int64_t)blockIdx.x * RADIX_TILE;
    const int64_t wbase = tbase + (int64_t)warp * (32 * RADIX_ITEMS);
    const int tcount = (int)min((int64_t)RADIX_TILE, n - tbase);
    uint32_t k[RADIX_ITEMS], v[RADIX_ITEMS], r[RADIX_ITEMS];
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        int64_t gi = wbase + j * 32 + lane;
        bool valid = gi < n;
        unsigned vm = __ballot_sync(0xffffffffu, valid);
        k[j] = valid ? keys_in[gi] : 0u;
        v[j] = valid ? (vals_in ? vals_in[gi] : (uint32_t)gi) : 0u;
        r[j] = 0u;
        // lanes holding the same digit: one ballot per digit bit (independent
        // instructions, where a match has one long latency)
        const uint32_t d = (k[j] >> shift) & dm;
        unsigned peers = vm;
#pragma unroll
        for (int b = 0; b < RADIX_MAX_BITS; b++) {
            if (b < bits) {
                const unsigned on = __ballot_sync(0xffffffffu, (d >> b) & 1u);
                peers &= ((d >> b) & 1u) ? on : ~on;
            }
        }
        if (valid) {
            int leader = __ffs(peers) - 1;
            uint32_t old = 0u;
            if (lane == leader) {
                old = R.wh[warp][d];
                R.wh[warp][d] = old + (uint32_t)__popc(peers);
            }
            old = __shfl_sync(peers, old, leader);
            r[j] = old + (uint32_t)__popc(peers & lanemask_lt());
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps; the tile's count of the digit
    constexpr int BPT = RADIX_MAX_BINS / RADIX_THREADS;   // bins per thread
    static_assert(BPT >= 1, "a thread owns at least one bin");
    uint32_t tot[BPT], part = 0;
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = tid * BPT + q;
        uint32_t run = 0;
        if (b < bins) {
#pragma unroll
            for (int w = 0; w < RADIX_WARPS; w++) {
                uint32_t c = R.wh[w][b];
                R.wh[w][b] = run;
                run += c;
            }
        }
        tot[q] = run;
        part += run;
    }
    // block-wide exclusive scan of the per-thread digit totals -> lbase
    uint32_t incl = part;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) R.wsum[warp] = incl;
    __syncthreads();
    uint32_t off = incl - part;
    for (int w = 0; w < warp; w++) off += R.wsum[w];
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = tid * BPT + q;
        if (b < bins) R.lbase[b] = off;
        off += tot[q];
    }
    __syncthreads();
    // stage the tile in digit order
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        int64_t gi = wbase + j * 32 + lane;
        if (gi < n) {
            const uint32_t d = (k[j] >> shift) & dm;
            const uint32_t lp = R.lbase[d] + R.wh[warp][d] + r[j];
            R.key[lp] = k[j];
            R.val[lp] = v[j];
        }
    }
    __syncthreads();
    // write out: slot i of the staged tile goes to dbase[d] + (i - lbase[d])
    for (int i = tid; i < tcount; i += RADIX_THREADS) {
        const uint32_t kk = R.key[i];
        const uint32_t d = (kk >> shift) & dm;
        const uint32_t p = R.dbase[d] + ((uint32_t)i - R.lbase[d]);
        if (keys_out) keys_out[p] = kk;
        vals_out[p] = R.val[i];
    }
}

// pw == nullptr: every photon has power pw0 (a traced map), so the power is
// written without a random read of the source list (gpow == nullptr: not
// written at all).  rec != nullptr: the
// photon's position and direction are read as one 32-byte record (one DRAM
// sector) instead of two 12-byte pieces of the position and direction arrays.
__global__ void k_grid_gather(const uint32_t* __restrict__ order, int64_t n, const float* __restrict__ pos,
                              const float* __restrict__ dir, const float4* __restrict__ rec,
                              const float* __restrict__ pw, float3 pw0, float4* __restrict__ gpos,
                              float* __restrict__ gdir, float* __restrict__ gpow, unsigned* status) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t s = order[j];
    if ((int64_t)s >= n) { raise_status(status, ST_BAD_INPUT); return; }
    float3 pp, dd;
    if (rec) {
        const float4 a = __ldg(rec + 2 * (int64_t)s), b = __ldg(rec + 2 * (int64_t)s + 1);
        pp = make_float3(a.x, a.y, a.z);
        dd = make_float3(b.x, b.y, b.z);
    } else {
        const float* p = pos + 3 * (int64_t)s;
        const float* d = dir + 3 * (int64_t)s;
        pp = make_float3(p[0], p[1], p[2]);
        dd = make_float3(d[0], d[1], d[2]);
    }
    gpos[j] = make_float4(pp.x, pp.y, pp.z, __uint_as_float(s));
    gdir[3 * j] = dd.x; gdir[3 * j + 1] = dd.y; gdir[3 * j + 2] = dd.z;
    if (!gpow) return;
    float3 w = pw0;
    if (pw) {
        const float* q = pw + 3 * (int64_t)s;
        w = make_float3(q[0], q[1], q[2]);
    }
    gpow[3 * j] = w.x; gpow[3 * j + 1] = w.y; gpow[3 * j + 2] = w.z;
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
    *hist_elems = (size_t)RADIX_MAX_BINS * tiles;
    *scan_ws_bytes = std::max(scan_workspace_bytes((int64_t)RADIX_MAX_BINS * tiles), scan_workspace_bytes(max_keys + 1));
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
    GridPlan pa{}, pb{};
    grid_dims(aabb, n, desired, pa.dims, &pa.cell);
    pa.cells = (int64_t)pa.dims[0] * pa.dims[1] * pa.dims[2];
    const int want_b = std::max(desired / regrid_div, 1);
    const bool two = want_b != desired;
    grid_dims(aabb, n, want_b, pb.dims, &pb.cell);
    pb.cells = (int64_t)pb.dims[0] * pb.dims[1] * pb.dims[2];
    auto geom = [&](const GridPlan& p) {
        GridGeom g;
        g.mnx = aabb[0]; g.mny = aabb[1]; g.mnz = aabb[2];
        g.gx = p.dims[0]; g.gy = p.dims[1]; g.gz = p.dims[2]; g.cell = p.cell;
        return g;
    };
    if ((e = cudaMemsetAsync(B.cell_sizes, 0, (size_t)pa.cells * 4, st)) != cudaSuccess) return e;
    if (two && (e = cudaMemsetAsync(B.counts2, 0, (size_t)pb.cells * 4, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(B.small, 0, 8, st)) != cudaSuccess) return e;
    int launches = 0;
    const int64_t smem_words = (pa.cells + 1) / 2 + (two ? (pb.cells + 1) / 2 : 0);
    if (n > 0 && smem_words <= COUNT_SMEM_WORDS) {
        const int smem = (int)smem_words * 4;
        if ((e = cudaFuncSetAttribute(k_count_cells_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
            return e;
        // one block per SM at this shared-memory size: whole waves of equal chunks
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int64_t least = blocks_for(n, COUNT_CHUNK);
        const int64_t nblk = (least + sms - 1) / sms * sms;
        const int64_t chunk = (n + nblk - 1) / nblk;
        k_count_cells_smem<<<(unsigned)blocks_for(n, (int)chunk), COUNT_THREADS, smem, st>>>(
            B.pos, n, chunk, geom(pa), geom(pb), two ? 1 : 0, (int)pa.cells, (int)pb.cells, B.cell_sizes, B.counts2);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_count_max<<<std::min<int64_t>(blocks_for(std::max(pa.cells, pb.cells), 256), 296), 256, 0, st>>>(
            B.cell_sizes, pa.cells, B.counts2, two ? pb.cells : 0, B.small);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        launches = 2;
    } else if (n > 0) {
        k_count_cells<<<blocks_for(n, 256), 256, 0, st>>>(B.pos, n, geom(pa), geom(pb), two ? 1 : 0, B.cell_sizes,
                                                            B.counts2, B.small);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        launches = 1;
    }
    uint32_t stack_mx[2] = {0u, 0u};
    uint32_t* mx = B.host_words ? B.host_words : stack_mx;
    if ((e = cudaMemcpyAsync(mx, B.small, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    pa.max_count = mx[0];
    pb.max_count = two ? mx[1] : mx[0];
    // the reference rebuilds at the finer resolution when a cell is overfull
    *plan = (mx[0] > (uint32_t)(regrid_mult * desired)) ? pb : pa;
    plan->launches = launches;
    return cudaSuccess;
}

cudaError_t grid_sort(GridBuffers& B, const float aabb[6], GridPlan& plan, int S, cudaStream_t st) {
    cudaError_t e;
    const int64_t n = B.n;
    const int64_t cells = plan.cells;
    const int S3 = S * S * S;
    const int64_t keys = cells * S3;
    GridGeom g;
    g.mnx = aabb[0]; g.mny = aabb[1]; g.mnz = aabb[2];
    g.gx = plan.dims[0]; g.gy = plan.dims[1]; g.gz = plan.dims[2]; g.cell = plan.cell;
    if ((e = cudaMemsetAsync(B.key_counts, 0, (size_t)keys * 4, st)) != cudaSuccess) return e;
    if (n > 0) {
        k_key_count<<<blocks_for(n, 256), 256, 0, st>>>(B.pos, n, g, S, B.cid, B.key_counts);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        plan.launches++;
    }
    if ((e = scan_u32(B.key_counts, B.key_starts, keys, 0, B.key_starts + keys, B.scan_ws, B.status, st)) != cudaSuccess) return e;
    k_cells_from_keys<<<blocks_for(cells, 256), 256, 0, st>>>(B.key_starts, cells, S3, B.cell_starts, B.cell_sizes);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    plan.launches += 2;
    if (n == 0) return cudaSuccess;

    int launches = 0;
    e = radix_and_gather(B, n, keys, &launches, st);
    plan.launches += launches;
    return e;
}

size_t radix_hist_elems(int64_t n) {
    return (size_t)RADIX_MAX_BINS * (size_t)std::max<int64_t>(1, (n + RADIX_TILE - 1) / RADIX_TILE);
}

// Stable LSD radix sort of n keys below 2^key_bits, digits of equal width <= 9 bits.
cudaError_t radix_sort_u32(const RadixBuffers& B, const uint32_t* keys_in, const uint32_t* vals_in, int64_t n,
                           int key_bits, bool want_keys, const uint32_t** keys_sorted, const uint32_t** vals_sorted,
                           int* launches, cudaStream_t st) {
    cudaError_t e;
    const int bits = std::min(std::max(key_bits, 1), 32);
    const int passes = (bits + RADIX_MAX_BITS - 1) / RADIX_MAX_BITS;
    const int width = (bits + passes - 1) / passes;
    const int tiles = (int)((n + RADIX_TILE - 1) / RADIX_TILE);
    const int64_t hist_n = ((int64_t)1 << width) * tiles;
    const uint32_t* kin = keys_in;
    const uint32_t* vin = vals_in;
    if ((e = cudaFuncSetAttribute(k_radix_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RadixSmem))) !=
        cudaSuccess)
        return e;
    for (int p = 0; p < passes; p++) {
        const int shift = width * p;
        const bool last = p == passes - 1;
        uint32_t* kout = (last && !want_keys) ? nullptr : B.keys[p & 1];
        uint32_t* vout = B.vals[p & 1];
        k_radix_upsweep<<<tiles, RADIX_THREADS, 0, st>>>(kin, n, shift, width, B.hist, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = scan_u32(B.hist, B.hist, hist_n, 0, nullptr, B.scan_ws, B.status, st)) != cudaSuccess) return e;
        k_radix_downsweep<<<tiles, RADIX_THREADS, sizeof(RadixSmem), st>>>(kin, vin, n, shift, width, B.hist, tiles,
                                                                           kout, vout);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        kin = kout;
        vin = vout;
    }
    if (keys_sorted) *keys_sorted = kin;
    if (vals_sorted) *vals_sorted = vin;
    *launches += 3 * passes;
    return cudaSuccess;
}

// LSD radix sort of B.cid (keys < key_space, stable), carrying the photon
// index; then the sorted records.
cudaError_t radix_and_gather(GridBuffers& B, int64_t n, int64_t key_space, int* launches, cudaStream_t st) {
    int bits = 1;
    while (bits < 32 && ((uint64_t)1 << bits) < (uint64_t)key_space) bits++;
    RadixBuffers RB{{B.keys[0], B.keys[1]}, {B.vals[0], B.vals[1]}, B.hist, B.scan_ws, B.status};
    const uint32_t* order = nullptr;
    cudaError_t e = radix_sort_u32(RB, B.cid, nullptr, n, bits, false, nullptr, &order, launches, st);
    if (e != cudaSuccess) return e;
    k_grid_gather<<<blocks_for(n, 256), 256, 0, st>>>(
        order, n, B.pos, B.dir, B.rec, B.uniform_pow ? nullptr : B.pow,
        make_float3(B.pow_value[0], B.pow_value[1], B.pow_value[2]), B.gpos, B.gdir,
        B.uniform_pow && B.defer_pow ? nullptr : B.gpow, B.status);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t grid_multi(GridBuffers& B, const GridMulti& M, int* launches, cudaStream_t st) {
    cudaError_t e;
    const int64_t n = B.n;
    const int64_t key_space = M.total_keys + 1;           // + the sentinel of empty slots
    if ((e = cudaMemsetAsync(B.key_counts, 0, (size_t)key_space * 4, st)) != cudaSuccess) return e;
    if (n > 0) {
        k_key_count_multi<<<blocks_for(n, 256), 256, 0, st>>>(B.pos, n, M.tab, M.ph_off, M.ninst, M.filled,
                                                             (uint32_t)M.total_keys, B.cid, B.key_counts);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *launches += 1;
    }
    if ((e = scan_u32(B.key_counts, B.key_starts, key_space, 0, B.key_starts + key_space, B.scan_ws, B.status, st)) !=
        cudaSuccess)
        return e;
    k_cells_multi<<<blocks_for(M.total_cells, 256), 256, 0, st>>>(M.total_cells, M.tab, M.cell_off, M.ninst,
                                                                  B.key_starts, B.cell_starts, B.cell_sizes);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *launches += 2;
    if (n == 0) return cudaSuccess;
    return radix_and_gather(B, n, key_space, launches, st);
}

}  // namespace pm
