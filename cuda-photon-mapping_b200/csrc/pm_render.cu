// pm_render.cu -- eye pass and per-pixel resolve.
//
// Reference: CudaPhotonMapping/Raytracer.cuh:140-241 (render_trace),
// RaytracePlanner.cuh:30-69, MediumManager.cuh:17-79, MMInnerStack.cuh:131,
// MMOuterStack.cuh:269, RayPlanStack.cuh:13-88, Camera.cuh:67-81,
// Raytracer.cuh:95-107 (tone map), 277 (quantisation).
//
// The reference computes each pixel in one thread, interleaving ray steps and
// kNN gathers.  The ray steps never depend on gathered values, so the pass is
// split: k_eye follows every eye path (closest hits, refraction plans, mirror
// bounces) and records one gather request per hit; the gather kernel then
// estimates all requests in one launch; k_resolve combines each pixel's
// requests in hit order (clamp <= 1, path weight), tone-maps and quantises.
// The refraction planner and medium bookkeeping are restated with the
// reference's index arithmetic and per-pixel storage that starts zeroed
// (the reference's GPU path zeroes it once with cudaMemset and lets threads
// share slots across pixels; per-pixel zeroed storage is the deterministic
// reading of that).
#include "pm_render.cuh"

namespace pm {

namespace {

constexpr int EYE_THREADS = 128;
constexpr int MD = RENDER_MAX_DEPTH;
constexpr int DCMAX = (MD + 1) / 2;
constexpr int SLOTS = MD + 2;

struct Plan { Ray ray; int depth; V3 coef; int in_obj; };

struct MediumState {
    int D, DC;
    int outer_size;
    int cont[SLOTS];
    float dior[SLOTS * DCMAX];
    int did[SLOTS * DCMAX];
    int nplans;
    Plan plans[MD];
    bool overflow;
    bool zeroed;   // cont / dior / did hold their zeros (written on the first refraction)
    __device__ void init(int d) {
        D = d; DC = (d + 1) / 2; outer_size = 0; nplans = 0; overflow = false; zeroed = false;
    }
    // The storage starts zeroed; most eye paths never refract, so the zeros are
    // written only when a path first reads or writes it (plans are always
    // written before they are read).
    __device__ void touch() {
        if (zeroed) return;
        for (int i = 0; i < SLOTS; i++) cont[i] = 0;
        for (int i = 0; i < SLOTS * DCMAX; i++) { dior[i] = 0.f; did[i] = 0; }
        zeroed = true;
    }
    __device__ int idx(int slot, int depth) {
        if (slot < 0 || slot > D + 1 || depth < 0 || depth >= DC) { overflow = true; return -1; }
        return slot * DCMAX + depth;
    }
    __device__ float ior_at(int slot, int depth) { int k = idx(slot, depth); return k < 0 ? 0.f : dior[k]; }
    __device__ int id_at(int slot, int depth) { int k = idx(slot, depth); return k < 0 ? 0 : did[k]; }
    __device__ void set_at(int slot, int depth, float ior, int id) {
        int k = idx(slot, depth);
        if (k >= 0) { dior[k] = ior; did[k] = id; }
    }
};

struct Rgi { float n1, n2; bool in_obj; };

__device__ Rgi get_refractive_indices(MediumState& M, float def, int model_id, float ior) {
    int L = M.outer_size;
    if (L == 0) return Rgi{def, ior, true};
    M.touch();
    int s = M.cont[L - 1];
    if (s == 0) return Rgi{def, ior, true};
    if (M.id_at(L, s - 1) == model_id) {
        bool in_obj = s > 1;
        return Rgi{ior, in_obj ? M.ior_at(L, s - 2) : def, in_obj};
    }
    return Rgi{M.ior_at(L, s - 1), ior, true};
}
__device__ void increase_depth(MediumState& M, bool& max_level) {
    M.touch();
    int L = M.outer_size;
    if (L == 0) { M.outer_size = 1; L = 1; }
    if (L < M.D) {
        int count = (M.D + 1) / 2;
        int other = M.cont[L - 1];
        if (!(M.outer_size > M.D - 1)) {
            int to = max(other, 0);
            int from = max(to - count, 0);
            for (int i = from; i < to; i++) M.set_at(L, i, M.ior_at(L - 1, i), M.id_at(L - 1, i));
            M.cont[M.outer_size] = to - from;
            M.outer_size++;
        }
        max_level = false;
    } else {
        max_level = true;
    }
}
__device__ void reduce_depth(MediumState& M, bool& max_level) {
    if (!max_level && M.outer_size > 0) M.outer_size--;
    max_level = false;
}
__device__ void inform(MediumState& M, int model_id, float ior, bool max_level) {
    M.touch();
    int pos = M.outer_size - 1 - (max_level ? 0 : 1);
    if (pos < 0 || pos >= SLOTS) { M.overflow = true; return; }
    int s = M.cont[pos];
    if (s != 0) {
        if (M.id_at(s, s - 1) == model_id) M.cont[pos] = s - 1;
    } else if (!(M.DC == 0 || s > M.DC - 1)) {
        M.set_at(s, s, ior, model_id);
        M.cont[pos] = s + 1;
    }
}
__device__ void push_refraction(MediumState& M, bool& max_level, const Ray& r, int depth, V3 coef, int model_id,
                                float ior, float opaque, bool in_obj) {
    increase_depth(M, max_level);
    inform(M, model_id, ior, max_level);
    if (!(M.D == 0 || M.nplans > M.D - 1)) {
        Plan& p = M.plans[M.nplans++];
        p.ray = r; p.depth = depth + 1; p.coef = vscale(coef, 1.f - opaque); p.in_obj = in_obj;
    }
}
__device__ bool pop_refraction(MediumState& M, bool& max_level, Ray& r, int& depth, V3& coef, bool& in_obj) {
    reduce_depth(M, max_level);
    if (M.nplans == 0) return false;
    const Plan& p = M.plans[--M.nplans];
    r = p.ray; depth = p.depth; coef = p.coef; in_obj = p.in_obj != 0;
    return true;
}

__device__ __forceinline__ V3 camera_dir(const CameraDev& c, int x, int y) {
    float u = ((float)x + 0.5f) / (float)c.W;
    float v = ((float)y + 0.5f) / (float)c.H;
    V3 pos = ld3(c.pos);
    V3 hor = vscale(ld3(c.right), c.vw);
    V3 ver = vscale(ld3(c.up), c.vh);
    V3 llc = vsub(vsub(vscale(vadd(pos, ld3(c.fwd)), c.focal), vscale(hor, 0.5f)), vscale(ver, 0.5f));
    return vsub(vadd(vadd(llc, vscale(hor, u)), vscale(ver, v)), pos);
}

__device__ __forceinline__ V3 camera_dir_at(const CameraDev& c, float u, float v) {
    V3 pos = ld3(c.pos);
    V3 hor = vscale(ld3(c.right), c.vw);
    V3 ver = vscale(ld3(c.up), c.vh);
    V3 llc = vsub(vsub(vscale(vadd(pos, ld3(c.fwd)), c.focal), vscale(hor, 0.5f)), vscale(ver, 0.5f));
    return vsub(vadd(vadd(llc, vscale(hor, u)), vscale(ver, v)), pos);
}

constexpr uint32_t SAMPLE_TAG = 0x53414d50u;   // stream tag of the training-point sampler

__global__ void k_sample_hits(DevScene S, CameraDev cam, int64_t n, uint64_t seed, float* __restrict__ pos,
                              float* __restrict__ nrm, float* __restrict__ weight) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stream rs;
    rs.init(seed, (uint64_t)i, SAMPLE_TAG);
    // stratified: sample i lies in pixel floor(i * W * H / n) (row-major), so
    // consecutive samples are image neighbours (coherent for the gather)
    const int64_t npx = (int64_t)cam.W * cam.H;
    const int64_t px = (int64_t)(((unsigned __int128)i * (unsigned __int128)npx) / (unsigned __int128)n);
    const float ju = rs.next(), jv = rs.next();   // (0, 1]
    const float u = ((float)(px % cam.W) + 1.f - ju) / (float)cam.W;
    const float v = ((float)(px / cam.W) + 1.f - jv) / (float)cam.H;
    Ray ray;
    ray.o = ld3(cam.pos);
    ray.d = vnorm_div(camera_dir_at(cam, u, v));
    Hit h;
    V3 p = v3(0.f, 0.f, 0.f), nn = v3(0.f, 1.f, 0.f);
    float w = 0.f;
    if (intersect(S, ray.o, ray.d, h)) {
        const Material m = load_mat(S, hit_model(S, h.tri));
        nn = shading_normal(S, h);
        p = vadd(vscale(ray.d, h.t), ray.o);
        w = vnull(tri_albedo(S, h.tri, m)) ? 0.f : 1.f;
    }
    st3(pos + 3 * i, p);
    st3(nrm + 3 * i, nn);
    weight[i] = w;
}

// The record of one eye-path hit: (hit point, triangle), (shading normal,
// flags); the model and material of the hit for the path's next step.
__device__ __forceinline__ void hit_record(const DevScene& S, const Ray& ray, const Hit& h, bool in_obj, float4& a,
                                          float4& b, int& model, Material& m, V3& n, V3& ip) {
    model = hit_model(S, h.tri);
    m = load_mat(S, model);
    n = shading_normal(S, h);
    ip = vadd(vscale(ray.d, h.t), ray.o);
    if (in_obj && vdot(ray.d, n) > 0) n = vscale(n, -1.f);
    V3 mdiff = tri_albedo(S, h.tri, m);
    uint32_t flags = 2u | ((!in_obj && !vnull(mdiff)) ? 1u : 0u);
    a = make_float4(ip.x, ip.y, ip.z, __int_as_float(h.tri));
    b = make_float4(n.x, n.y, n.z, __uint_as_float(flags));
}

__device__ __forceinline__ Ray primary_ray(const CameraDev& cam, int x, int y) {
    Ray ray;
    ray.o = ld3(cam.pos);
    ray.d = vnorm_div(camera_dir(cam, x, y));
    return ray;
}

// the eye path of local pixel `li` (image of `cam`): its gather requests in hit
// order (c.w = pixel bits `px`); returns the number of hits
__device__ __forceinline__ int eye_hits(const DevScene& S, const CameraDev& cam, int D, int64_t li, uint32_t px,
                                        float4* ha, float4* hb, float4* hc, unsigned* status) {
    int nh = 0;
    const int64_t i = li;
    {
        const int x = (int)(i % cam.W), y = (int)(i / cam.W);
        Ray ray = primary_ray(cam, x, y);
        MediumState M;
        M.init(D);
        int new_depth = 0, cur = -1;
        V3 coef = v3(1.f, 1.f, 1.f);
        bool max_level = false, in_obj = false;
        while ((cur < D && cur != new_depth) || pop_refraction(M, max_level, ray, new_depth, coef, in_obj)) {
            cur = new_depth;
            Hit h;
            if (!intersect(S, ray.o, ray.d, h)) continue;
            int model;
            Material m;
            V3 n, ip;
            float4 ra, rb;
            hit_record(S, ray, h, in_obj, ra, rb, model, m, n, ip);
            if (nh < RENDER_MAX_HITS) {
                ha[nh] = ra;
                hb[nh] = rb;
                hc[nh] = make_float4(coef.x, coef.y, coef.z, __uint_as_float(px));
                nh++;
            } else {
                raise_status(status, ST_OVERFLOW);
            }
            if (m.opaque < 1.f && cur != D - 1) {
                Rgi ri = get_refractive_indices(M, S.default_ior, model, m.ior);
                Ray nr;
                if (ray_refract(ray, ip, n, ri.n1, ri.n2, nr))
                    push_refraction(M, max_level, nr, cur, coef, model, m.ior, m.opaque, ri.in_obj);
            }
            if (!in_obj && !vnull(m.specular) && cur != D - 1) {
                Ray nr = ray_reflect(ray, ip, n);
                float c = powf(fmaxf(vdot(nr.d, vneg(ray.d)), 0.0f), m.shininess);
                coef = vmul(coef, vscale(vscale(m.specular, m.opaque), c));
                ray = nr;
                new_depth = cur + 1;
            }
        }
        if (M.overflow) raise_status(status, ST_STACK);
    }
    return nh;
}

// reserve nh consecutive request slots (one atomic per warp) and write them;
// every lane of the warp calls this, `valid` lanes own pixel gi
__device__ __forceinline__ void eye_emit(Requests& R, bool valid, int64_t gi, int nh, const float4* ha,
                                         const float4* hb, const float4* hc, unsigned* status) {
    const int lane = threadIdx.x & 31;
    unsigned incl = (unsigned)nh;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    unsigned long long base = 0;
    unsigned wtotal = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 31 && wtotal) base = atomicAdd(R.counter, (unsigned long long)wtotal);
    base = __shfl_sync(0xffffffffu, base, 31) + (incl - (unsigned)nh);
    if (!valid) return;
    if ((int64_t)(base + nh) > R.cap) {
        raise_status(status, ST_OVERFLOW);
        R.px_base[gi] = 0;
        R.px_count[gi] = 0;
        return;
    }
    for (int k = 0; k < nh; k++) {
        R.a[base + k] = ha[k];
        R.b[base + k] = hb[k];
        R.c[base + k] = hc[k];
    }
    R.px_base[gi] = (uint32_t)base;
    R.px_count[gi] = (uint32_t)nh;
}

__global__ void __launch_bounds__(EYE_THREADS)
k_eye(DevScene S, CameraDev cam, int D, Requests R, unsigned* status, const int* __restrict__ order) {
    const int64_t npx = (int64_t)cam.W * cam.H;
    const int64_t blk = order ? (int64_t)order[blockIdx.x] : (int64_t)blockIdx.x;
    const int64_t i = blk * blockDim.x + threadIdx.x;
    const bool valid = i < npx;
    float4 ha[RENDER_MAX_HITS], hb[RENDER_MAX_HITS], hc[RENDER_MAX_HITS];
    const int nh = valid ? eye_hits(S, cam, D, i, (uint32_t)i, ha, hb, hc, status) : 0;
    eye_emit(R, valid, i, nh, ha, hb, hc, status);
}

__device__ __forceinline__ int find_pixel_instance(const int64_t* __restrict__ off, int ninst, int64_t g) {
    int lo = 0, hi = ninst - 1;   // last i with off[i] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// eye_emit with the requests of class cls (0 or 1) in their own range:
// class 0 at [0, split) from R.counter[0], class 1 at [split, R.cap) from
// R.counter[1]; one scan carries both classes' counts (class 1 in the high 16
// bits: at most 32 x RENDER_MAX_HITS per warp) and lane 31 reserves both
__device__ __forceinline__ void eye_emit_split(Requests& R, int64_t split, bool valid, int cls, int64_t gi, int nh,
                                               const float4* ha, const float4* hb, const float4* hc,
                                               unsigned* status) {
    static_assert(32 * RENDER_MAX_HITS < 65536, "per-class warp counts must fit 16 bits");
    const int lane = threadIdx.x & 31;
    const unsigned mine = (unsigned)nh << (cls ? 16 : 0);
    unsigned incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned wtotal = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long b0 = 0, b1 = 0;
    if (lane == 31) {
        if (wtotal & 0xffffu) b0 = atomicAdd(R.counter, (unsigned long long)(wtotal & 0xffffu));
        if (wtotal >> 16) b1 = atomicAdd(R.counter + 1, (unsigned long long)(wtotal >> 16));
    }
    b0 = __shfl_sync(0xffffffffu, b0, 31);
    b1 = __shfl_sync(0xffffffffu, b1, 31);
    if (!valid) return;
    const unsigned excl = incl - mine;
    const int64_t hi = cls ? R.cap : split;
    const int64_t base = cls ? split + (int64_t)(b1 + (excl >> 16)) : (int64_t)(b0 + (excl & 0xffffu));
    if (base + nh > hi) {
        raise_status(status, ST_OVERFLOW);
        R.px_base[gi] = 0;
        R.px_count[gi] = 0;
        return;
    }
    for (int k = 0; k < nh; k++) {
        R.a[base + k] = ha[k];
        R.b[base + k] = hb[k];
        R.c[base + k] = hc[k];
    }
    R.px_base[gi] = (uint32_t)base;
    R.px_count[gi] = (uint32_t)nh;
}

// all instances' pixels in one launch: global pixel g of instance i (off[i] <= g < off[i+1])
__global__ void __launch_bounds__(EYE_THREADS)
k_eye_multi(const RenderInstDev* __restrict__ tab, const int64_t* __restrict__ px_off, int ninst, int64_t npx,
            Requests R, int64_t split, unsigned* status) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g < npx;
    float4 ha[RENDER_MAX_HITS], hb[RENDER_MAX_HITS], hc[RENDER_MAX_HITS];
    int nh = 0, cls = 0;
    if (valid) {
        const int i = find_pixel_instance(px_off, ninst, g);
        const RenderInstDev& T = tab[i];
        cls = T.cls;
        nh = eye_hits(T.S, T.cam, T.max_depth, g - __ldg(px_off + i), (uint32_t)g, ha, hb, hc, status);
    }
    eye_emit_split(R, split, valid, cls, g, nh, ha, hb, hc, status);
}

// combine pixel gi's requests with the scene's materials, tone-map, quantise
__device__ __forceinline__ void resolve_pixel(const DevScene& S, int64_t gi, const Requests& R,
                                              const float* __restrict__ est_g, const float* __restrict__ est_c,
                                              float tone_t, uint8_t* __restrict__ rgb8, float* __restrict__ radiance) {
    const uint32_t base = R.px_base[gi], cnt = R.px_count[gi];
    V3 acc = v3(0.f, 0.f, 0.f);
    for (uint32_t r = 0; r < cnt; r++) {
        const size_t q = (size_t)base + r;
        float4 a = R.a[q], b = R.b[q], c = R.c[q];
        const int tri = __float_as_int(a.w);
        const int model = hit_model(S, tri);
        const Material m = load_mat(S, model);
        const uint32_t flags = __float_as_uint(b.w);
        V3 color = v3(0.f, 0.f, 0.f);
        if (flags & 1u) {
            V3 di_op = vscale(tri_albedo(S, tri, m), m.opaque);
            color = vadd(color, vscale(vmul(ld3(est_g + 3 * q), di_op), 4.f));
        }
        color = vadd(color, m.emission);
        if (est_c) color = vadd(color, vscale(ld3(est_c + 3 * q), m.opaque));
        color = vmin1(color, 1.f);
        acc = vadd(acc, vmul(color, xyz(c)));
    }
    if (radiance) st3(radiance + 3 * gi, acc);
    V3 e = v3(expf(-tone_t * acc.x), expf(-tone_t * acc.y), expf(-tone_t * acc.z));
    V3 mp = vsub(v3(1.f, 1.f, 1.f), e);
    const float rg = 1.0f / 2.2f;
    V3 l = vmin1(v3(powf(mp.x, rg), powf(mp.y, rg), powf(mp.z, rg)), 1.f);
    rgb8[3 * gi] = (uint8_t)(l.x * 255);
    rgb8[3 * gi + 1] = (uint8_t)(l.y * 255);
    rgb8[3 * gi + 2] = (uint8_t)(l.z * 255);
}

__global__ void k_resolve(DevScene S, int64_t npx, Requests R, const float* __restrict__ est_g,
                          const float* __restrict__ est_c, float tone_t, uint8_t* __restrict__ rgb8,
                          float* __restrict__ radiance) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npx) return;
    resolve_pixel(S, i, R, est_g, est_c, tone_t, rgb8, radiance);
}

__global__ void k_resolve_multi(const RenderInstDev* __restrict__ tab, const int64_t* __restrict__ px_off, int ninst,
                                int64_t npx, Requests R, const float* __restrict__ est_g, float tone_t,
                                uint8_t* __restrict__ rgb8, float* __restrict__ radiance) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npx) return;
    const int i = find_pixel_instance(px_off, ninst, g);
    resolve_pixel(tab[i].S, g, R, est_g, nullptr, tone_t, rgb8, radiance);
}

}  // namespace

namespace {
__device__ __forceinline__ uint32_t spread10r(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__global__ void k_request_keys(const float4* __restrict__ a, int64_t n, float lx, float ly, float lz, float sx,
                               float sy, float sz, uint32_t* __restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = a[i];
    const uint32_t x = (uint32_t)min(max((int)((p.x - lx) * sx), 0), 511);
    const uint32_t y = (uint32_t)min(max((int)((p.y - ly) * sy), 0), 511);
    const uint32_t z = (uint32_t)min(max((int)((p.z - lz) * sz), 0), 511);
    keys[i] = (spread10r(x) << 2) | (spread10r(y) << 1) | spread10r(z);
}
}  // namespace

cudaError_t request_keys(const float4* a, int64_t n, const float aabb[6], uint32_t* keys, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    float sc[3];
    for (int k = 0; k < 3; k++) {
        const float ext = aabb[3 + k] - aabb[k];
        sc[k] = ext > 0.f ? 512.f / ext : 0.f;
    }
    k_request_keys<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, n, aabb[0], aabb[1], aabb[2], sc[0], sc[1], sc[2],
                                                                 keys);
    return cudaGetLastError();
}

namespace {
__global__ void k_probe_hits(DevScene S, CameraDev cam, int tile, int P, int tiles_x, int64_t nprobe,
                             float4* __restrict__ ppos, float4* __restrict__ pnrm) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nprobe) return;
    const int64_t t = s / P;
    int dx, dy;
    probe_xy((int)(s % P), P, tile, dx, dy);
    const int x = (int)(t % tiles_x) * tile + dx, y = (int)(t / tiles_x) * tile + dy;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = make_float4(0.f, 0.f, 1.f, 0.f);
    if (x < cam.W && y < cam.H) {
        const Ray ray = primary_ray(cam, x, y);
        Hit h;
        if (intersect(S, ray.o, ray.d, h)) {
            int model;
            Material m;
            V3 n, ip;
            float4 ra, rb;
            hit_record(S, ray, h, false, ra, rb, model, m, n, ip);
            if (__float_as_uint(rb.w) & 1u) {
                a = ra;
                b = make_float4(rb.x, rb.y, rb.z, __uint_as_float(1u));
            }
        }
    }
    ppos[s] = a;
    pnrm[s] = b;
}
}  // namespace

cudaError_t probe_hits(const DevScene& S, const CameraDev& cam, int tile, int P, float4* ppos, float4* pnrm,
                       cudaStream_t st) {
    const int tx = (cam.W + tile - 1) / tile, ty = (cam.H + tile - 1) / tile;
    const int64_t n = (int64_t)tx * ty * P;
    if (n <= 0) return cudaSuccess;
    k_probe_hits<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, cam, tile, P, tx, n, ppos, pnrm);
    return cudaGetLastError();
}

int64_t eye_blocks(int64_t npx) { return (npx + EYE_THREADS - 1) / EYE_THREADS; }
int eye_threads() { return EYE_THREADS; }

cudaError_t eye_pass(const DevScene& S, const CameraDev& cam, int max_depth, Requests R, unsigned* status,
                     cudaStream_t st, const int* block_order, int64_t nblocks) {
    if (max_depth < 0 || max_depth > RENDER_MAX_DEPTH) return cudaErrorInvalidValue;
    const int64_t npx = (int64_t)cam.W * cam.H;
    const int64_t all = eye_blocks(npx);
    if (nblocks < 0) nblocks = all;
    if (nblocks > all || (nblocks < all && !block_order)) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(R.counter, 0, 8, st);
    if (e != cudaSuccess || nblocks == 0) return e;
    k_eye<<<(unsigned)nblocks, EYE_THREADS, 0, st>>>(S, cam, max_depth, R, status, block_order);
    return cudaGetLastError();
}

cudaError_t eye_pass_multi(const RenderInstDev* tab, const int64_t* px_off, int ninst, int64_t npx, Requests R,
                           int64_t split, unsigned* status, cudaStream_t st) {
    if (split < 0 || split > R.cap) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(R.counter, 0, 16, st);
    if (e != cudaSuccess || npx <= 0) return e;
    k_eye_multi<<<(unsigned)((npx + EYE_THREADS - 1) / EYE_THREADS), EYE_THREADS, 0, st>>>(tab, px_off, ninst, npx, R,
                                                                                          split, status);
    return cudaGetLastError();
}

cudaError_t resolve_multi(const RenderInstDev* tab, const int64_t* px_off, int ninst, int64_t npx, Requests R,
                          const float* est_g, float tone_t, uint8_t* rgb8, float* radiance, cudaStream_t st) {
    if (npx <= 0) return cudaSuccess;
    k_resolve_multi<<<(unsigned)((npx + 255) / 256), 256, 0, st>>>(tab, px_off, ninst, npx, R, est_g, tone_t, rgb8,
                                                                   radiance);
    return cudaGetLastError();
}

cudaError_t sample_primary_hits(const DevScene& S, const CameraDev& cam, int64_t n, uint64_t seed, float* pos,
                                float* nrm, float* weight, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_sample_hits<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, cam, n, seed, pos, nrm, weight);
    return cudaGetLastError();
}

cudaError_t resolve(const DevScene& S, const CameraDev& cam, Requests R, const float* est_g, const float* est_c,
                    float tone_t, uint8_t* rgb8, float* radiance, cudaStream_t st) {
    const int64_t npx = (int64_t)cam.W * cam.H;
    k_resolve<<<(unsigned)((npx + 255) / 256), 256, 0, st>>>(S, npx, R, est_g, est_c, tone_t, rgb8, radiance);
    return cudaGetLastError();
}

}  // namespace pm
