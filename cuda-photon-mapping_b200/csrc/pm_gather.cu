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
// like the floats, so integer comparison is the lexicographic order.  Photons
// are stored by (cell, sub-cell); the walk starts with the query's sub-cell,
// and once k candidates are held, every (sub-)cell whose box lies farther than
// the current k-th distance (with a relative margin far above float rounding)
// is skipped.  A candidate is first tested on its squared distance against a
// bound slightly above the threshold's square, so the correctly rounded sqrt
// -- the reference's distance -- is only taken for candidates that can enter.
// The answer is the exhaustive walk's.  The heap is finally sorted so the
// estimate sums in ascending order.
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

// Cell / sub-cell of a point: the quotient (p - min) / cell selects the cell
// (clamped, CudaPhotonMapping/PhotonGrid.cu:10-23); its fractional part the sub-cell.
__device__ __forceinline__ void locate(float p, float mn, float cell, int g, int S, int& c, int& s) {
    float u = (p - mn) / cell;
    c = min(max((int)u, 0), g - 1);
    float f = u - (float)c;
    s = min(max((int)(f * (float)S), 0), S - 1);
}

// distance from q to the slab [lo, hi] along one axis; an open side (photons
// clamped into a boundary cell from outside the grid) is at infinity
__device__ __forceinline__ float axis_gap(float q, float lo, float hi, bool open_lo, bool open_hi) {
    float a = open_lo ? 0.f : lo - q;
    float b = open_hi ? 0.f : q - hi;
    return fmaxf(fmaxf(a, b), 0.f);
}

template <int KCAP>
struct Walk {
    const GatherGrid& G;
    V3 q;
    float r;
    int k;
    TopK<KCAP> H;
    float lim2;        // squared pre-filter: a candidate with s > lim2 cannot enter
    float lim;         // distance bound used for pruning cells / sub-cells
    __device__ Walk(const GatherGrid& g, V3 qq, float rr, int kk) : G(g), q(qq), r(rr), k(kk) {
        H.size = 0;
        lim = r;
        lim2 = r * r * 1.000001f;
    }
    __device__ __forceinline__ void tighten() {
        if (H.size == k) {
            float dk = __uint_as_float((uint32_t)(H.key[0] >> 32));
            lim = fminf(r, dk);
            lim2 = lim * lim * 1.000001f;
        }
    }
    // scan the photons of one sub-cell key
    __device__ __forceinline__ void scan(uint32_t key) {
        const uint32_t a = __ldg(G.key_starts + key), b = __ldg(G.key_starts + key + 1);
        for (uint32_t j = a; j < b; j++) {
            float4 p = __ldg(G.gpos + j);
            float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
            float s = dx * dx + dy * dy + dz * dz;
            if (s <= lim2) {
                float d = sqrtf(s);
                if (d <= r) {
                    unsigned long long kk = ((unsigned long long)__float_as_uint(d) << 32) | __float_as_uint(p.w);
                    if (H.size < k || kk < H.key[0]) {
                        H.push(kk, j, k);
                        tighten();
                    }
                }
            }
        }
    }
    // visit the sub-cells of cell (x, y, z) that lie within lim of q
    __device__ __forceinline__ void cell(int x, int y, int z, uint32_t skip_key) {
        const float c = G.cell, pad = c * 1e-4f;
        const float m = 1.f + 1e-5f;
        float lo_x = G.mn[0] + (float)x * c, lo_y = G.mn[1] + (float)y * c, lo_z = G.mn[2] + (float)z * c;
        const bool ox0 = x == 0, ox1 = x == G.gx - 1, oy0 = y == 0, oy1 = y == G.gy - 1, oz0 = z == 0, oz1 = z == G.gz - 1;
        float L = lim * m;
        float gx = axis_gap(q.x, lo_x - pad, lo_x + c + pad, ox0, ox1);
        float gy = axis_gap(q.y, lo_y - pad, lo_y + c + pad, oy0, oy1);
        float gz = axis_gap(q.z, lo_z - pad, lo_z + c + pad, oz0, oz1);
        if (gx * gx + gy * gy + gz * gz > L * L) return;
        const int S = G.S;
        const float sc = c / (float)S;
        const uint32_t base = (uint32_t)(x + y * G.gx + z * G.gx * G.gy) * (uint32_t)(S * S * S);
        // sub-cell index ranges along each axis that the sphere of radius lim can reach
        int sx0 = ox0 ? 0 : max(0, (int)floorf((q.x - L - pad - lo_x) / sc));
        int sx1 = ox1 ? S - 1 : min(S - 1, (int)floorf((q.x + L + pad - lo_x) / sc));
        int sy0 = oy0 ? 0 : max(0, (int)floorf((q.y - L - pad - lo_y) / sc));
        int sy1 = oy1 ? S - 1 : min(S - 1, (int)floorf((q.y + L + pad - lo_y) / sc));
        int sz0 = oz0 ? 0 : max(0, (int)floorf((q.z - L - pad - lo_z) / sc));
        int sz1 = oz1 ? S - 1 : min(S - 1, (int)floorf((q.z + L + pad - lo_z) / sc));
        for (int sz = sz0; sz <= sz1; sz++)
            for (int sy = sy0; sy <= sy1; sy++)
                for (int sx = sx0; sx <= sx1; sx++) {
                    const uint32_t key = base + (uint32_t)(sx + S * (sy + S * sz));
                    if (key == skip_key) continue;
                    L = lim * m;
                    float ax = axis_gap(q.x, lo_x + sx * sc - pad, lo_x + (sx + 1) * sc + pad, ox0 && sx == 0, ox1 && sx == S - 1);
                    float ay = axis_gap(q.y, lo_y + sy * sc - pad, lo_y + (sy + 1) * sc + pad, oy0 && sy == 0, oy1 && sy == S - 1);
                    float az = axis_gap(q.z, lo_z + sz * sc - pad, lo_z + (sz + 1) * sc + pad, oz0 && sz == 0, oz1 && sz == S - 1);
                    if (ax * ax + ay * ay + az * az > L * L) continue;
                    scan(key);
                }
    }
};

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
    Walk<KCAP> W(G, q, r, k);
    int hx, hy, hz, sx, sy, sz;
    locate(q.x, G.mn[0], G.cell, G.gx, G.S, hx, sx);
    locate(q.y, G.mn[1], G.cell, G.gy, G.S, hy, sy);
    locate(q.z, G.mn[2], G.cell, G.gz, G.S, hz, sz);
    const int S = G.S;
    const uint32_t home_key = (uint32_t)(hx + hy * G.gx + hz * G.gx * G.gy) * (uint32_t)(S * S * S) +
                              (uint32_t)(sx + S * (sy + S * sz));
    // the query's own sub-cell first, then the rest of its cell, then the cube
    // of cells of half width ceil(r / cell) (CudaPhotonMapping/PhotonGrid.cu:257-284)
    W.scan(home_key);
    W.cell(hx, hy, hz, home_key);
    const int rc = (int)ceilf(r / G.cell);
    const int x0 = max(0, hx - rc), y0 = max(0, hy - rc), z0 = max(0, hz - rc);
    const int x1 = min(G.gx - 1, hx + rc), y1 = min(G.gy - 1, hy + rc), z1 = min(G.gz - 1, hz + rc);
    for (int z = z0; z <= z1; z++)
        for (int y = y0; y <= y1; y++)
            for (int x = x0; x <= x1; x++) {
                if (x == hx && y == hy && z == hz) continue;
                W.cell(x, y, z, 0xffffffffu);
            }
    TopK<KCAP>& H = W.H;
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
