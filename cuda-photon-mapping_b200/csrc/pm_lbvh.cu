// pm_lbvh.cu -- device BVH builder: a linear BVH over Morton codes
// (T. Karras, "Maximizing parallelism in the construction of BVHs, octrees,
// and k-d trees", HPG 2012), emitted in the node format the traversal of
// pm_scene.cuh reads.
//
// The reference has no acceleration structure (it tests every triangle of
// every model whose box a ray meets, CudaPhotonMapping/Model.cuh:366-446; its
// kd-tree code only reduces a model to an AABB, KdTree.cu:395-464).  The
// closest-hit answer of the traversal does not depend on the tree's shape
// (smallest (t, triangle index) with conservatively padded boxes), so this
// builder and the host SAH builder give bit-identical photon maps; the SAH
// tree traces faster, this one builds in about a millisecond.
//
//   k_lbvh_bounds     centroid bounds (ordered-integer atomics)
//   k_lbvh_morton     30-bit Morton code of each centroid in those bounds
//   radix_sort_u32    stable sort of the codes carrying the triangle index
//                     (stable: equal codes stay in triangle order)
//   k_lbvh_hierarchy  one thread per interior node: its range of sorted
//                     triangles and split from the common-prefix lengths of
//                     the keys (code, sorted position)
//   k_lbvh_boxes      bottom-up from each triangle: the second thread to reach
//                     an interior node unions its children's boxes, computes
//                     the subtree's SAH cost and writes the node; a child of
//                     <= 4 triangles becomes a leaf when testing them costs
//                     no more than its best split (the host builder's cost
//                     model: 1 per interior visit, 1.2 per triangle test)
#include <algorithm>
#include "pm_lbvh.cuh"
#include "pm_grid.cuh"
#include "pm_scan.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr int LEAF_MAX = 4;
constexpr float SAH_CT = 1.0f;   // cost of an interior visit (one node, two slab tests) ...
constexpr float SAH_CI = 1.2f;   // ... and of one triangle test
constexpr int MAX_CLIMB = 256;   // levels a bottom-up thread may climb (tree depth is < 70)

// float <-> unsigned with the same order (for atomicMin / atomicMax)
__device__ __forceinline__ uint32_t ford(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funord(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

struct Box6 { float lo[3], hi[3]; };

__device__ __forceinline__ Box6 tri_box(const float* __restrict__ tp, int t) {
    const float* p = tp + 9 * (size_t)t;
    Box6 b;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        b.lo[a] = fminf(fminf(p[a], p[3 + a]), p[6 + a]);
        b.hi[a] = fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]);
    }
    return b;
}

__global__ void k_lbvh_bounds(const float* __restrict__ tp, int n, uint32_t* __restrict__ cb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float mn[3] = {3.0e38f, 3.0e38f, 3.0e38f}, mx[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    if (t < n) {
        const Box6 b = tri_box(tp, t);
#pragma unroll
        for (int a = 0; a < 3; a++) mn[a] = mx[a] = 0.5f * (b.lo[a] + b.hi[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            atomicMin(cb + a, ford(mn[a]));
            atomicMax(cb + 3 + a, ford(mx[a]));
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {   // 10 bits -> every third bit
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_lbvh_morton(const float* __restrict__ tp, int n, const uint32_t* __restrict__ cb,
                              uint32_t* __restrict__ codes) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const Box6 b = tri_box(tp, t);
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float c = 0.5f * (b.lo[a] + b.hi[a]);
        const float lo = funord(cb[a]), hi = funord(cb[3 + a]);
        const float ext = hi - lo;
        const float u = ext > 0.f ? (c - lo) / ext : 0.f;
        q[a] = (uint32_t)min(max((int)(u * 1024.f), 0), 1023);
    }
    codes[t] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
}

// common-prefix length of the keys (code, position) at sorted positions i, j; -1 outside
__device__ __forceinline__ int lbvh_delta(const uint32_t* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = k[i], b = k[j];
    return a == b ? 32 + __clz(i ^ j) : __clz(a ^ b);
}

// children: >= 0 interior node, < 0 ~(sorted position) of a single triangle
__global__ void k_lbvh_hierarchy(const uint32_t* __restrict__ k, int n, int* __restrict__ child,
                                 int* __restrict__ range, int* __restrict__ parent_int, int* __restrict__ parent_leaf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = lbvh_delta(k, n, i, i + 1) - lbvh_delta(k, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = lbvh_delta(k, n, i, i - d);
    int lmax = 2;
    while (lbvh_delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (lbvh_delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = lbvh_delta(k, n, i, j);
    int s = 0;
    for (int div = 2;; div <<= 1) {
        const int t = (l + div - 1) / div;
        if (lbvh_delta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const int c0 = lo == gamma ? ~gamma : gamma;
    const int c1 = hi == gamma + 1 ? ~(gamma + 1) : gamma + 1;
    child[2 * i] = c0;
    child[2 * i + 1] = c1;
    range[2 * i] = lo;
    range[2 * i + 1] = hi;
    if (c0 < 0) parent_leaf[gamma] = i; else parent_int[gamma] = i;
    if (c1 < 0) parent_leaf[gamma + 1] = i; else parent_int[gamma + 1] = i;
    if (i == 0) parent_int[0] = -1;
}

__device__ __forceinline__ Box6 load_box(const float* __restrict__ b, int i) {
    Box6 r;
#pragma unroll
    for (int a = 0; a < 3; a++) { r.lo[a] = __ldcg(b + 6 * i + a); r.hi[a] = __ldcg(b + 6 * i + 3 + a); }
    return r;
}
__device__ __forceinline__ void store_box(float* b, int i, const Box6& r) {
#pragma unroll
    for (int a = 0; a < 3; a++) { __stcg(b + 6 * i + a, r.lo[a]); __stcg(b + 6 * i + 3 + a, r.hi[a]); }
}

// one child's half of a node record: (lo - p, ref), (hi + p, 0), p = pad + 1e-5 max(|lo|, |hi|) per axis
__device__ __forceinline__ void put_child(float4* o, const Box6& b, int ref, float pad) {
    float lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float span = fmaxf(fabsf(b.lo[a]), fabsf(b.hi[a]));
        const float p = pad + span * 1e-5f;
        lo[a] = b.lo[a] - p;
        hi[a] = b.hi[a] + p;
    }
    o[0] = make_float4(lo[0], lo[1], lo[2], __int_as_float(ref));
    o[1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

// the traversal's ref of child c: interior node index, or a leaf ~(first << 8 | count)
// (a single triangle, or an interior node whose subtree is cheaper as a leaf)
__device__ __forceinline__ int child_ref(int c, const int* __restrict__ range, const int* isleaf) {
    if (c < 0) return ~(((~c) << 8) | 1);
    const int lo = range[2 * c], hi = range[2 * c + 1];
    if (__ldcg(isleaf + c)) return ~((lo << 8) | (hi - lo + 1));
    return c;
}

__device__ __forceinline__ float half_area(const Box6& b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_lbvh_boxes(const float* __restrict__ tp, int n, const uint32_t* __restrict__ order,
                             const int* __restrict__ child, const int* __restrict__ range,
                             const int* __restrict__ parent_int, const int* __restrict__ parent_leaf,
                             uint32_t* __restrict__ arrived, float* ibox, float* lbox, float* cost, int* isleaf,
                             float4* __restrict__ nodes, int* __restrict__ prim, float pad, unsigned* status) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int tri = (int)order[p];
    if (tri < 0 || tri >= n) { raise_status(status, ST_BAD_INPUT); return; }
    prim[p] = tri;
    store_box(lbox, p, tri_box(tp, tri));
    int x = parent_leaf[p];
    for (int climb = 0; x >= 0; climb++) {
        if (climb >= MAX_CLIMB || x >= n - 1) { raise_status(status, ST_BAD_INPUT); return; }
        __threadfence();
        if (atomicAdd(arrived + x, 1u) == 0u) return;   // the sibling's thread finishes this node
        __threadfence();
        const int c0 = child[2 * x], c1 = child[2 * x + 1];
        const Box6 b0 = c0 < 0 ? load_box(lbox, ~c0) : load_box(ibox, c0);
        const Box6 b1 = c1 < 0 ? load_box(lbox, ~c1) : load_box(ibox, c1);
        Box6 u;
#pragma unroll
        for (int a = 0; a < 3; a++) { u.lo[a] = fminf(b0.lo[a], b1.lo[a]); u.hi[a] = fmaxf(b0.hi[a], b1.hi[a]); }
        store_box(ibox, x, u);
        // SAH cost of the subtree: CT + (A0 C0 + A1 C1) / A as an interior node,
        // CI n as a leaf of n <= LEAF_MAX triangles; the cheaper one is kept
        const float C0 = c0 < 0 ? SAH_CI : __ldcg(cost + c0), C1 = c1 < 0 ? SAH_CI : __ldcg(cost + c1);
        const float A = half_area(u);
        const float split = SAH_CT + (A > 0.f ? (half_area(b0) * C0 + half_area(b1) * C1) / A : C0 + C1);
        const int cnt = range[2 * x + 1] - range[2 * x] + 1;
        const bool leaf = x != 0 && cnt <= LEAF_MAX && SAH_CI * (float)cnt <= split;
        __stcg(cost + x, leaf ? SAH_CI * (float)cnt : split);
        __stcg(isleaf + x, leaf ? 1 : 0);
        put_child(nodes + 4 * (size_t)x, b0, child_ref(c0, range, isleaf), pad);
        put_child(nodes + 4 * (size_t)x + 2, b1, child_ref(c1, range, isleaf), pad);
        x = parent_int[x];
    }
}

// one triangle: a root holding it as a leaf and an empty second child
__global__ void k_lbvh_single(const float* __restrict__ tp, float4* __restrict__ nodes, int* __restrict__ prim,
                              float pad) {
    prim[0] = 0;
    put_child(nodes, tri_box(tp, 0), ~((0 << 8) | 1), pad);
    nodes[2] = make_float4(3.0e38f, 3.0e38f, 3.0e38f, __int_as_float(~0));
    nodes[3] = make_float4(-3.0e38f, -3.0e38f, -3.0e38f, 0.f);
}

inline unsigned blocks_of(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// scratch carve-up (byte offsets, 256-aligned)
struct Layout {
    size_t cb, codes, keys0, keys1, vals0, vals1, hist, scan, child, range, pint, pleaf, arrived, ibox, lbox, cost,
        isleaf, total;
};
inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
Layout layout(int n) {
    Layout L{};
    const size_t N = (size_t)std::max(n, 2);
    const size_t hist = radix_hist_elems(n);
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = up256(o + bytes); return at; };
    L.cb = take(6 * 4);
    L.codes = take(N * 4);
    L.keys0 = take(N * 4);
    L.keys1 = take(N * 4);
    L.vals0 = take(N * 4);
    L.vals1 = take(N * 4);
    L.hist = take(hist * 4);
    L.scan = take(scan_workspace_bytes((int64_t)hist));
    L.child = take(2 * N * 4);
    L.range = take(2 * N * 4);
    L.pint = take(N * 4);
    L.pleaf = take(N * 4);
    L.arrived = take(N * 4);
    L.ibox = take(6 * N * 4);
    L.lbox = take(6 * N * 4);
    L.cost = take(N * 4);
    L.isleaf = take(N * 4);
    L.total = o;
    return L;
}

__global__ void k_leaf_records(const float4* __restrict__ tri, const int* __restrict__ prim, int n,
                               float4* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int t = prim[j];
    if (t < 0 || t >= n) return;
    const float4* src = tri + 5 * (size_t)t;
    float4* dst = out + 4 * (size_t)j;
    dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2];
    const float4 q4 = src[4];
    dst[3] = make_float4(q4.x, q4.y, q4.z, __int_as_float(t));
}

}  // namespace

cudaError_t bvh_leaf_records(const float4* tri, const int* prim, int ntri, float4* out, cudaStream_t st) {
    if (ntri <= 0) return cudaSuccess;
    k_leaf_records<<<blocks_of(ntri, 256), 256, 0, st>>>(tri, prim, ntri, out);
    return cudaGetLastError();
}

size_t lbvh_scratch_bytes(int ntri) { return layout(ntri).total; }

cudaError_t lbvh_build(const float* tri_pos, int ntri, float pad, float4* nodes, int* prim, void* scratch,
                       unsigned* status, int* launches, cudaStream_t st) {
    if (ntri <= 0 || ntri >= (1 << 23)) return cudaErrorInvalidValue;
    cudaError_t e;
    if (ntri == 1) {
        k_lbvh_single<<<1, 1, 0, st>>>(tri_pos, nodes, prim, pad);
        *launches += 1;
        return cudaGetLastError();
    }
    const int n = ntri;
    const Layout L = layout(n);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    uint32_t* cb = reinterpret_cast<uint32_t*>(base + L.cb);
    uint32_t* codes = reinterpret_cast<uint32_t*>(base + L.codes);
    int* child = reinterpret_cast<int*>(base + L.child);
    int* range = reinterpret_cast<int*>(base + L.range);
    int* pint = reinterpret_cast<int*>(base + L.pint);
    int* pleaf = reinterpret_cast<int*>(base + L.pleaf);
    uint32_t* arrived = reinterpret_cast<uint32_t*>(base + L.arrived);
    float* ibox = reinterpret_cast<float*>(base + L.ibox);
    float* lbox = reinterpret_cast<float*>(base + L.lbox);
    float* cost = reinterpret_cast<float*>(base + L.cost);
    int* isleaf = reinterpret_cast<int*>(base + L.isleaf);
    if ((e = cudaMemsetAsync(cb, 0xff, 12, st)) != cudaSuccess) return e;   // minima start at the largest key
    if ((e = cudaMemsetAsync(cb + 3, 0, 12, st)) != cudaSuccess) return e;  // maxima at the smallest
    if ((e = cudaMemsetAsync(arrived, 0, (size_t)n * 4, st)) != cudaSuccess) return e;
    k_lbvh_bounds<<<blocks_of(n, 256), 256, 0, st>>>(tri_pos, n, cb);
    k_lbvh_morton<<<blocks_of(n, 256), 256, 0, st>>>(tri_pos, n, cb, codes);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    RadixBuffers RB{{reinterpret_cast<uint32_t*>(base + L.keys0), reinterpret_cast<uint32_t*>(base + L.keys1)},
                    {reinterpret_cast<uint32_t*>(base + L.vals0), reinterpret_cast<uint32_t*>(base + L.vals1)},
                    reinterpret_cast<uint32_t*>(base + L.hist), base + L.scan, status};
    const uint32_t* skeys = nullptr;
    const uint32_t* order = nullptr;
    if ((e = radix_sort_u32(RB, codes, nullptr, n, 30, true, &skeys, &order, launches, st)) != cudaSuccess) return e;
    k_lbvh_hierarchy<<<blocks_of(n - 1, 256), 256, 0, st>>>(skeys, n, child, range, pint, pleaf);
    k_lbvh_boxes<<<blocks_of(n, 256), 256, 0, st>>>(tri_pos, n, order, child, range, pint, pleaf, arrived, ibox, lbox,
                                                    cost, isleaf, nodes, prim, pad, status);
    *launches += 4;
    return cudaGetLastError();
}

}  // namespace pm
