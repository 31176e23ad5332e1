// pm_learned.cu -- the learned render's tile check and fallback selection.
//
// The learned render answers every global-map request of the eye pass with the
// radiance cache, then checks the cache per screen tile: P probe requests per
// tile (the first request of the pixels at fixed positions inside the tile)
// are also answered by the exact kNN gather, and a tile whose relative bias
// over its probes exceeds a threshold takes the exact gather for all of its
// requests.  Probe slots are fixed per (tile, probe), so the result
// does not depend on scheduling.
#include <algorithm>
#include "pm_learned.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

// probe position k of P inside a tile of edge T: a ceil(sqrt(P)) grid of cell centres
// Each probe's request: the first request of its pixel, which the probe pass
// (probe_hits) traced from the camera with the eye pass's own device code;
// the two records must agree bit for bit, and a probe whose record differs
// from its request raises ST_BAD_INPUT (its request index is then dropped).
__global__ void k_probe_req(CameraDev cam, Requests R, int tile, int P, int tiles_x, int64_t ntiles,
                            const float4* __restrict__ ppos, const float4* __restrict__ pnrm,
                            uint32_t* __restrict__ preq, unsigned* status) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ntiles * P) return;
    const int64_t t = s / P;
    const int k = (int)(s % P);
    int dx, dy;
    probe_xy(k, P, tile, dx, dy);
    const int x = (int)(t % tiles_x) * tile + dx, y = (int)(t / tiles_x) * tile + dy;
    uint32_t q = 0xffffffffu;
    if (x < cam.W && y < cam.H) {
        const int64_t px = (int64_t)y * cam.W + x;
        if (R.px_count[px] > 0) {
            const uint32_t r = R.px_base[px];
            if (__float_as_uint(R.b[r].w) & 1u) q = r;
        }
    }
    const float4 pa = ppos[s], pb = pnrm[s];
    const bool probe = (__float_as_uint(pb.w) & 1u) != 0u;
    bool same = probe == (q != 0xffffffffu);
    if (same && probe) {
        const float4 ra = R.a[q], rb = R.b[q];
        same = __float_as_uint(pa.x) == __float_as_uint(ra.x) && __float_as_uint(pa.y) == __float_as_uint(ra.y) &&
               __float_as_uint(pa.z) == __float_as_uint(ra.z) && __float_as_uint(pa.w) == __float_as_uint(ra.w) &&
               __float_as_uint(pb.x) == __float_as_uint(rb.x) && __float_as_uint(pb.y) == __float_as_uint(rb.y) &&
               __float_as_uint(pb.z) == __float_as_uint(rb.z);
    }
    if (!same) {
        raise_status(status, ST_BAD_INPUT);
        q = 0xffffffffu;
    }
    preq[s] = q;
}

// Per tile: the cache's relative bias over its probes,
//   sum_c |sum_k (cache_kc - exact_kc)| / sum_c sum_k exact_kc,
// flagged when above the threshold (a negative threshold flags every tile:
// the exact render).  The exact probe estimates carry the kNN estimate's own
// noise (about 1 / sqrt(k) relative); summing signed differences over the
// probes averages it down, while a systematic cache error stays.  With
// noise_z > 0 the tile must exceed the threshold by noise_z standard errors of
// that sum as well (per channel sqrt(n) x the sample standard deviation of the
// n differences), so that probe noise alone does not flag it.
__global__ void k_tile_flags(int64_t ntiles, int P, const uint32_t* __restrict__ preq, const float* __restrict__ exact,
                             const float* __restrict__ cached, float max_rel_err, float noise_z,
                             uint8_t* __restrict__ flag, unsigned long long* __restrict__ nflag) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    V3 bias = v3(0.f, 0.f, 0.f), sq = v3(0.f, 0.f, 0.f), ref = v3(0.f, 0.f, 0.f);
    int cnt = 0;
    for (int k = 0; k < P; k++) {
        const int64_t s = t * P + k;
        const uint32_t q = preq[s];
        if (q == 0xffffffffu) continue;
        const V3 e = ld3(exact + 3 * s), c = ld3(cached + 3 * (size_t)q);
        const V3 d = vsub(c, e);
        bias = vadd(bias, d);
        sq = vadd(sq, vmul(d, d));
        ref = vadd(ref, e);
        cnt++;
    }
    const float num = fabsf(bias.x) + fabsf(bias.y) + fabsf(bias.z);
    const float den = fabsf(ref.x) + fabsf(ref.y) + fabsf(ref.z);
    float se = 0.f;
    if (noise_z > 0.f && cnt > 1) {
        const float n = (float)cnt, m = n / (n - 1.f);
        se = sqrtf(fmaxf(m * (sq.x - bias.x * bias.x / n), 0.f)) + sqrtf(fmaxf(m * (sq.y - bias.y * bias.y / n), 0.f)) +
             sqrtf(fmaxf(m * (sq.z - bias.z * bias.z / n), 0.f));
    }
    const bool f = max_rel_err < 0.f || (cnt > 0 && num > max_rel_err * den + noise_z * se);
    flag[t] = f ? 1 : 0;
    if (f) atomicAdd(nflag, 1ull);
}

// request q (of nreq): flag bit 2 and a list entry when its tile is flagged (all lanes of the warp call this)
__device__ __forceinline__ void mark_one(int64_t q, int64_t nreq, Requests& R, int W, int tile, int tiles_x,
                                         const uint8_t* __restrict__ flag, unsigned long long* __restrict__ nfb,
                                         uint32_t* __restrict__ list) {
    bool fb = false;
    if (q < nreq) {
        float4 b = R.b[q];
        uint32_t flags = __float_as_uint(b.w);
        const uint32_t px = __float_as_uint(R.c[q].w);
        const int x = (int)(px % (uint32_t)W), y = (int)(px / (uint32_t)W);
        flags &= ~LEARNED_FALLBACK;
        if ((flags & 1u) && flag[(int64_t)(y / tile) * tiles_x + x / tile]) {
            flags |= LEARNED_FALLBACK;
            fb = true;
        }
        b.w = __uint_as_float(flags);
        R.b[q] = b;
    }
    const unsigned m = __ballot_sync(0xffffffffu, fb);
    unsigned long long base = 0;
    if ((threadIdx.x & 31) == 0 && m) base = atomicAdd(nfb, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (fb) list[base + __popc(m & lanemask_lt())] = (uint32_t)q;
}

// requests of flagged tiles that need the global estimate get flag bit 2 and
// join the list of fallback requests (list order is immaterial: every answer
// is written at its request's index)
__global__ void k_mark_fallback(int64_t cap, const unsigned long long* __restrict__ n_dev, Requests R, int W, int tile,
                                int tiles_x, const uint8_t* __restrict__ flag, unsigned long long* __restrict__ nfb,
                                uint32_t* __restrict__ list) {
    const int64_t nreq = n_dev ? (int64_t)min(*n_dev, (unsigned long long)cap) : cap;
    for (int64_t b0 = (int64_t)blockIdx.x * blockDim.x; b0 < nreq; b0 += (int64_t)gridDim.x * blockDim.x)
        mark_one(b0 + threadIdx.x, nreq, R, W, tile, tiles_x, flag, nfb, list);
}

// est = exact for fallback requests, else the cache
__global__ void k_merge(int64_t cap, const unsigned long long* __restrict__ n_dev, Requests R,
                        const float* __restrict__ cached, const float* __restrict__ exact, float* __restrict__ est) {
    const int64_t nreq = n_dev ? (int64_t)min(*n_dev, (unsigned long long)cap) : cap;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nreq; q += (int64_t)gridDim.x * blockDim.x) {
        const bool fb = (__float_as_uint(R.b[q].w) & LEARNED_FALLBACK) != 0u;
        const float* src = fb ? exact : cached;
        est[3 * q] = src[3 * q];
        est[3 * q + 1] = src[3 * q + 1];
        est[3 * q + 2] = src[3 * q + 2];
    }
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// one thread per request when the count is known on the host, else a
// grid-stride launch of (at most) 8 blocks of 256 per SM over the capacity
inline unsigned req_blocks(int64_t cap, bool on_device, int sm_count) {
    const unsigned b = blocks(cap, 256);
    return on_device ? std::min<unsigned>(b, (unsigned)(8 * std::max(sm_count, 1))) : b;
}

}  // namespace

cudaError_t learned_probe_req(const CameraDev& cam, const Requests& R, int tile, int P, const float4* ppos,
                              const float4* pnrm, uint32_t* preq, unsigned* status, cudaStream_t st) {
    const int tx = (cam.W + tile - 1) / tile, ty = (cam.H + tile - 1) / tile;
    const int64_t ntiles = (int64_t)tx * ty;
    k_probe_req<<<blocks(ntiles * P, 256), 256, 0, st>>>(cam, R, tile, P, tx, ntiles, ppos, pnrm, preq, status);
    return cudaGetLastError();
}

cudaError_t learned_select(const CameraDev& cam, const Requests& R, int64_t nreq, const unsigned long long* nreq_dev,
                           int tile, int P, const uint32_t* preq, const float* probe_exact, const float* cached,
                           float max_rel_err, float noise_z, uint8_t* tile_flag, unsigned long long* counts,
                           uint32_t* fallback_list, int sm_count, cudaStream_t st) {
    const int tx = (cam.W + tile - 1) / tile, ty = (cam.H + tile - 1) / tile;
    const int64_t ntiles = (int64_t)tx * ty;
    k_tile_flags<<<blocks(ntiles, 256), 256, 0, st>>>(ntiles, P, preq, probe_exact, cached, max_rel_err, noise_z, tile_flag,
                                                      counts);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || nreq <= 0) return e;
    k_mark_fallback<<<req_blocks(nreq, nreq_dev != nullptr, sm_count), 256, 0, st>>>(nreq, nreq_dev, R, cam.W, tile, tx,
                                                                                    tile_flag, counts + 1, fallback_list);
    return cudaGetLastError();
}

cudaError_t learned_merge(const Requests& R, int64_t nreq, const unsigned long long* nreq_dev, const float* cached,
                          const float* exact, float* est, int sm_count, cudaStream_t st) {
    if (nreq <= 0) return cudaSuccess;
    k_merge<<<req_blocks(nreq, nreq_dev != nullptr, sm_count), 256, 0, st>>>(nreq, nreq_dev, R, cached, exact, est);
    return cudaGetLastError();
}

}  // namespace pm
