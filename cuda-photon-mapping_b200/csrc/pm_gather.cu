// pm_gather.cu -- kNN photon gather + radiance estimate.
//
// Reference: CudaPhotonMapping/PhotonGrid.cu:222-284 (cube of cells of half
// width ceil(r / cell) around the query's cell, distance test <= r),
// PhotonMaxHeap.cuh:43-127 (bounded max-heap of k), Raytracer.cuh:110-138
// (Gaussian-filtered density estimate over the selected photons).
//
// Selection rule: the k photons with the smallest (distance, source id) pairs
// among those with distance <= r.  This is the reference heap's set whenever no
// two candidates tie at the k-th distance; on ties it is deterministic (the
// reference's heap keeps whichever the sift order leaves).  Distances are the
// reference's length(p - q) in IEEE float, so the sets are bit-exact.
//
// One thread per query.  The candidate heap keeps 64-bit keys
// (float bits of the distance << 32 | source id): non-negative float bits order
// like the floats, so integer comparison is the lexicographic order.  Once k
// candidates are held, a cell whose box lies farther than the current k-th
// distance (with a relative margin far above float rounding) is skipped; that
// prunes most of the reference's 27-cell cube without changing the answer.
// The heap is finally sorted so the estimate sums in ascending order.
#include "pm_gather.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr int GATHER_THREADS = 128;

template <int KCAP>
struct TopK {
    unsigned long long key[KCAP];
    uint32_t slot[KCAP];
    int size;
    __device__ __forceinline__ void sift_down(int i, int n) {
        while (true) {
            int l = 2 * i + 1, r = l + 1, big = i;
            if (l < n && key[l] > key[big]) big = l;
            if (r < n && key[r] > key[big]) big = r;
            if (big == i) break;
            unsigned long long tk = key[i]; key[i] = key[big]; key[big] = tk;
            uint32_t ts = slot[i]; slot[i] = slot[big]; slot[big] = ts;
            i = big;
        }
    }
    __device__ __forceinline__ void push(unsigned long long k, uint32_t s, int kmax) {
        if (size < kmax) {
            int i = size++;
            key[i] = k; slot[i] = s;
            while (i > 0) {
                int p = (i - 1) >> 1;
                if (key[p] >= key[i]) break;
                unsigned long long tk = key[i]; key[i] = key[p]; key[p] = tk;
                uint32_t ts = slot[i]; slot[i] = slot[p]; slot[p] = ts;
                i = p;
            }
        } else if (k < key[0]) {
            key[0] = k; slot[0] = s;
            sift_down(0, size);
        }
    }
    __device__ __forceinline__ void sort_ascending() {
        for (int n = size; n > 1; n--) {
            unsigned long long tk = key[0]; key[0] = key[n - 1]; key[n - 1] = tk;
            uint32_t ts = slot[0]; slot[0] = slot[n - 1]; slot[n - 1] = ts;
            sift_down(0, n - 1);
        }
    }
};

__device__ __forceinline__ int cell_coord(float p, float mn, float cell, int g) {
    int c = (int)((p - mn) / cell);
    return min(max(c, 0), g - 1);
}

// squared distance from q to the box of cell (x, y, z); boxes of boundary cells
// are open towards the outside (photons there were clamped into them)
__device__ __forceinline__ float cell_dist2(const GatherGrid& G, V3 q, int x, int y, int z) {
    const float pad = G.cell * 1e-4f;
    float lo, hi, dx, dy, dz;
    lo = x == 0 ? -3.0e38f : G.mn[0] + (float)x * G.cell - pad;
    hi = x == G.gx - 1 ? 3.0e38f : G.mn[0] + (float)(x + 1) * G.cell + pad;
    dx = fmaxf(fmaxf(lo - q.x, q.x - hi), 0.f);
    lo = y == 0 ? -3.0e38f : G.mn[1] + (float)y * G.cell - pad;
    hi = y == G.gy - 1 ? 3.0e38f : G.mn[1] + (float)(y + 1) * G.cell + pad;
    dy = fmaxf(fmaxf(lo - q.y, q.y - hi), 0.f);
    lo = z == 0 ? -3.0e38f : G.mn[2] + (float)z * G.cell - pad;
    hi = z == G.gz - 1 ? 3.0e38f : G.mn[2] + (float)(z + 1) * G.cell + pad;
    dz = fmaxf(fmaxf(lo - q.z, q.z - hi), 0.f);
    return dx * dx + dy * dy + dz * dz;
}

template <int KCAP>
__global__ void __launch_bounds__(GATHER_THREADS)
k_gather(GatherGrid G, GatherQueries Q, float r, int k, int require_full, GatherOut O) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Q.n) return;
    V3 q, nrm;
    if (Q.pos3) {
        q = ld3(Q.pos3 + 3 * i);
        nrm = ld3(Q.nrm3 + 3 * i);
    } else {
        float4 a = Q.pos4[i], b = Q.nrm4[i];
        if ((__float_as_uint(b.w) & Q.flag_mask) == 0u) {
            st3(O.rad + 3 * i, v3(0.f, 0.f, 0.f));
            if (O.cnt) O.cnt[i] = 0;
            if (O.rk) O.rk[i] = 0.f;
            return;
        }
        q = xyz(a);
        nrm = xyz(b);
    }
    if (k <= 0) {
        st3(O.rad + 3 * i, v3(0.f, 0.f, 0.f));
        if (O.cnt) O.cnt[i] = 0;
        if (O.rk) O.rk[i] = 0.f;
        return;
    }
    TopK<KCAP> H;
    H.size = 0;
    const int hx = cell_coord(q.x, G.mn[0], G.cell, G.gx);
    const int hy = cell_coord(q.y, G.mn[1], G.cell, G.gy);
    const int hz = cell_coord(q.z, G.mn[2], G.cell, G.gz);
    const int rc = (int)ceilf(r / G.cell);
    const int x0 = max(0, hx - rc), y0 = max(0, hy - rc), z0 = max(0, hz - rc);
    const int x1 = min(G.gx - 1, hx + rc), y1 = min(G.gy - 1, hy + rc), z1 = min(G.gz - 1, hz + rc);
    const float r_lim = r * (1.f + 1e-5f);
    for (int it = -1; ; ) {
        int x, y, z;
        if (it < 0) { x = hx; y = hy; z = hz; }
        else {
            int nx = x1 - x0 + 1, ny = y1 - y0 + 1;
            int nz = z1 - z0 + 1;
            if (it >= nx * ny * nz) break;
            x = x0 + it % nx; y = y0 + (it / nx) % ny; z = z0 + it / (nx * ny);
            if (x == hx && y == hy && z == hz) { it++; continue; }
        }
        it++;
        float lim = r_lim;
        if (H.size == k) lim = fminf(lim, __uint_as_float((uint32_t)(H.key[0] >> 32)) * (1.f + 1e-5f));
        if (cell_dist2(G, q, x, y, z) > lim * lim) continue;
        const uint32_t c = (uint32_t)(x + y * G.gx + z * G.gx * G.gy);
        const uint32_t s0 = G.starts[c], sz = G.sizes[c];
        for (uint32_t j = 0; j < sz; j++) {
            float4 p = __ldg(G.gpos + s0 + j);
            V3 dv = vsub(xyz(p), q);
            float d = vlength(dv);
            if (d <= r) {
                unsigned long long key = ((unsigned long long)__float_as_uint(d) << 32) | __float_as_uint(p.w);
                if (H.size < k || key < H.key[0]) H.push(key, s0 + j, k);
            }
        }
    }
    H.sort_ascending();
    const int cnt = H.size;
    float rk = cnt ? __uint_as_float((uint32_t)(H.key[cnt - 1] >> 32)) : 0.f;
    if (O.ids) {
        for (int e = 0; e < k; e++)
            O.ids[i * k + e] = e < cnt ? (uint32_t)(H.key[e] & 0xffffffffull) : 0xffffffffu;
    }
    if (O.cnt) O.cnt[i] = cnt;
    if (O.rk) O.rk[i] = rk;
    V3 res = v3(0.f, 0.f, 0.f);
    if (cnt > 0 && !(require_full && cnt != k)) {
        const float alpha = 1.818f, beta = 1.953f;
        float fr = rk * rk;
        for (int e = 0; e < cnt; e++) {
            uint32_t s = H.slot[e];
            V3 pd = ld3(G.gdir + 3 * (size_t)s);
            float cs = vdot(nrm, vneg(pd));
            if (cs > 0) {
                float d = __uint_as_float((uint32_t)(H.key[e] >> 32));
                float filter = alpha * (1.f - (1.f - expf(-beta * d * d / (2 * fr))) / (1.f - expf(-beta)));
                res = vadd(res, vscale(ld3(G.gpow + 3 * (size_t)s), filter));
            }
        }
        float common = 1.f / (3.14159265358979f * (rk * rk) * 1);
        res = vscale(res, common);
    }
    st3(O.rad + 3 * i, res);
}

template <int KCAP>
cudaError_t launch(const GatherGrid& G, const GatherQueries& Q, float r, int k, int require_full, const GatherOut& O,
                   cudaStream_t st) {
    unsigned blocks = (unsigned)((Q.n + GATHER_THREADS - 1) / GATHER_THREADS);
    k_gather<KCAP><<<blocks, GATHER_THREADS, 0, st>>>(G, Q, r, k, require_full, O);
    return cudaGetLastError();
}

}  // namespace

cudaError_t gather(const GatherGrid& G, const GatherQueries& Q, float r, int k, int require_full,
                   const GatherOut& O, unsigned* status, cudaStream_t st) {
    (void)status;
    if (Q.n <= 0) return cudaSuccess;
    if (k <= 16) return launch<16>(G, Q, r, k, require_full, O, st);
    if (k <= 32) return launch<32>(G, Q, r, k, require_full, O, st);
    if (k <= 64) return launch<64>(G, Q, r, k, require_full, O, st);
    if (k <= 128) return launch<128>(G, Q, r, k, require_full, O, st);
    if (k <= 256) return launch<256>(G, Q, r, k, require_full, O, st);
    return cudaErrorInvalidValue;
}

}  // namespace pm
