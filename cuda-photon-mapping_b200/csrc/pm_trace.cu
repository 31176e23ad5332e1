// pm_trace.cu -- photon tracing.
//
// Reference: CudaPhotonMapping/PhotonTracing.cu:127-375 (emit / trace / destiny),
// Model.cuh:202-243 (light point), Ray.cuh:16-96, PathOperator.cuh:7-42,
// PhotonTraceStack.cuh:40-116, PhotonArray.cuh:31-42.
//
// Layout and scheduling differ from the reference on purpose:
//  * every photon path p draws from its own counter-based stream (Philox,
//    counter = (draw, p, tag)), so a path's photons do not depend on which
//    thread traces it or when;
//  * a persistent grid traces the paths [p0, p0 + npaths) of one batch.  Lanes
//    whose path ended take the next path indices together (one atomic per
//    warp, ballot ranks), so SIMD lanes stay busy however long paths are;
//  * the k-th photon a path stores goes to stage slot [k][path], a 32-byte
//    record written as two 16-byte vector stores: (position, map flag) and
//    (direction, 0); one record fills one DRAM sector, so no sector is left
//    half written (a half-written sector costs a read of it from DRAM before
//    its write-back);
//  * k_compact writes the batch's photons into the global / caustic lists in
//    canonical order (path, then bounce) after exclusive scans of the per-path
//    counts, and cuts each list exactly at its capacity.
// A path that misses all geometry ends there and stores nothing (the reference
// returns an undefined value from trace() in that case); a refraction that
// yields no ray also ends the path.
#include <type_traits>
#include <vector>
#include "pm_trace.cuh"
#include "pm_scan.cuh"

namespace pm {

namespace {

constexpr int TRACE_THREADS = 128;
// 8 blocks of 128 per SM (64 registers, a few spilled): the traversal is
// bound by the latency of its node and triangle loads, and twice the resident
// warps hide more of it than the spills cost (10M photons: 5.77 -> 5.10 ms).
// 9 blocks (56 registers) measure within 0.5 % of 8; 10 blocks (48 registers,
// 300 B of spill stores) are 6 % slower.
constexpr int TRACE_MIN_BLOCKS = 8;
// top TRACE_SMEM_STACK entries of each lane's traversal stack in shared memory
// (8: 5.13 -> 4.92 ms per 10M photons; 16 and 32 entries take L1 from the
// node and triangle loads: 4.98 and 5.08 ms)
constexpr int TRACE_SMEM_STACK = 8;
using TraceStack = SplitStack<TRACE_SMEM_STACK, TRACE_THREADS>;
constexpr int MAX_STACK = 32;
constexpr int REJECT_LIMIT = 1 << 16;   // emission rejection loop bound (acceptance ~1/2 on valid lights)
constexpr int TRACE_REFILL = 8;          // default for KParams::refill (12 lanes measure the same)
// A traversal round ends once no more than TRACE_CUT lanes still descend
// (each keeps its traversal state for the next round): the few lanes whose
// ray crosses many nodes before its first leaf no longer hold the other
// lanes' hits back (10M photons: 3.85 -> 3.80 ms; 100M-photon stress scene
// -4 %; 2, 4, 8 and 12 lanes measure the same or slower).
constexpr int TRACE_CUT = 6;

enum { DIF = 0, SPEC = 1, ABSORB = 2, REFR = 3, NONE = 4 };

// The random stream of a photon path, two forms of the same Philox-4x32-10
// stream (pm_device.cuh's Stream: draw i is word (i & 3) of Philox(counter =
// (i >> 2, path_lo, path_hi, tag), key = seed)):
//  * ParamStream (k_trace): the launch's tag and the seed's ten round keys
//    (rk0 / rk1) are read from the kernel parameters, so a lane holds only
//    its path index, draw counter and the current block of four words, and
//    a Philox round takes no key additions (10M photons: 4.00 -> 3.85 ms);
//  * RegStream (k_trace_multi, whose lanes trace different instances, each
//    with its own seed): pm_device.cuh's Stream, keys in registers.
struct KParams;
struct ParamStream {
    uint32_t plo, phi, n;
    uint4 buf;
    __device__ __forceinline__ void init(const KParams&, uint64_t path) {
        plo = (uint32_t)path; phi = (uint32_t)(path >> 32); n = 0;
    }
    __device__ __forceinline__ float next(const KParams& P);
};
struct RegStream {
    Stream s;
    __device__ __forceinline__ void init(const KParams& P, uint64_t path);
    __device__ __forceinline__ float next(const KParams&) { return s.next(); }
};

template <class St>
struct Lane {
    St st;
    Ray ray;
    int bounce;
    int ng, nc;             // photons stored so far (global / caustic)
    int diffuse_surfs;
    int last;
    int sn;                 // medium stack size
};

struct KParams {
    DevScene S;
    uint64_t seed;
    uint32_t tag;
    int max_bounces;
    int64_t p0, npaths;
    V3 power;
    unsigned long long* counter;
    float4* stage;          // 2 float4 per slot
    uint32_t* cnt_g;
    uint32_t* cnt_c;
    unsigned* status;
    int refill;             // lanes with a finished query that end a warp's traversal loop
    unsigned long long* work;   // work-counting launch: rays, BVH node visits, triangle tests (else null)
    uint32_t rk0[10], rk1[10];  // Philox round keys of seed: low / high word + round x (0x9E3779B9, 0xBB67AE85)
};

__device__ __forceinline__ float ParamStream::next(const KParams& P) {
    if ((n & 3u) == 0u) {
        uint4 c = make_uint4(n >> 2, plo, phi, P.tag);
#pragma unroll
        for (int r = 0; r < 10; ++r) {   // philox10 of pm_device.cuh with the round keys precomputed
            const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
            const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
            c = make_uint4(hi1 ^ c.y ^ P.rk0[r], lo1, hi0 ^ c.w ^ P.rk1[r], lo0);
        }
        buf = c;
    }
    const uint32_t w = (n & 3u) == 0u ? buf.x : (n & 3u) == 1u ? buf.y : (n & 3u) == 2u ? buf.z : buf.w;
    ++n;
    return unit_from_u32(w);
}
__device__ __forceinline__ void RegStream::init(const KParams& P, uint64_t path) { s.init(P.seed, path, P.tag); }

// the round keys of KParams::seed (philox10's key schedule)
static void round_keys(KParams& P) {
    uint32_t k0 = (uint32_t)P.seed, k1 = (uint32_t)(P.seed >> 32);
    for (int r = 0; r < 10; r++) {
        P.rk0[r] = k0;
        P.rk1[r] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// light point + cosine-weighted direction by rejection (PhotonTracing.cu:345-369)
template <class LaneT>
__device__ __forceinline__ void start_path(const KParams& P, LaneT& L, int64_t path) {
    const DevScene& S = P.S;
    L.st.init(P, (uint64_t)path);
    int k = (int)roundf(0 + L.st.next(P) * (float)(S.light_count - 1));
    int tri = S.light_first + k;
    float bx = L.st.next(P);
    float by = 0.f + L.st.next(P) * ((1.f - bx) - 0.f);
    float bz = 1.f - bx - by;
    const float* tp = S.tri_pos + 9 * (size_t)tri;
    const float* tn = S.tri_nrm + 9 * (size_t)tri;
    V3 point = vadd(vadd(vscale(ld3(tp), bx), vscale(ld3(tp + 3), by)), vscale(ld3(tp + 6), bz));
    V3 lnorm = vadd(vadd(vscale(ld3(tn), bx), vscale(ld3(tn + 3), by)), vscale(ld3(tn + 6), bz));
    L.ray.o = vadd(point, vscale(lnorm, 0.0001f));
    float prob, dt;
    V3 d;
    int tries = 0;
    do {
        if (++tries > REJECT_LIMIT) {   // a light without a usable normal: end the path
            raise_status(P.status, ST_BAD_INPUT);
            L.ray.d = v3(0.f, 0.f, 0.f);
            break;
        }
        d.x = -1.f + L.st.next(P) * 2.f;
        d.y = -1.f + L.st.next(P) * 2.f;
        d.z = -1.f + L.st.next(P) * 2.f;
        d = vnorm_recip(d);
        prob = L.st.next(P);
        dt = vdot(d, lnorm);
        if (dt < 0) { dt = -dt; d = vscale(d, -1.f); }
    } while (prob > dt);
    if (tries <= REJECT_LIMIT) L.ray.d = d;
    L.bounce = 0;
    L.ng = L.nc = 0;
    L.diffuse_surfs = 0;
    L.last = NONE;
    L.sn = 0;
}

// Marsaglia disc, rejected into the hemisphere of n (Ray.cuh:16-56)
template <class St>
__device__ __forceinline__ Ray diffuse_bounce(V3 from, V3 n, St& st, const KParams& P) {
    V3 d;
    do {
        float x1, x2, s1, s2;
        do {
            x1 = -1.f + st.next(P) * 2.f;
            x2 = -1.f + st.next(P) * 2.f;
            s1 = x1 * x1;
            s2 = x2 * x2;
        } while (s1 + s2 >= 1);
        float f = sqrtf(1.f - s1 - s2);
        d = v3(2.f * x1 * f, 2.f * x2 * f, 1.f - 2.f * (s1 + s2));
    } while (vdot(d, n) < 0);
    Ray r;
    r.d = vnorm_div(d);
    r.o = vadd(from, vscale(r.d, 0.0001f));
    return r;
}

// Fresnel-Schlick with the integer powers written as products (PhotonTracing.cu:215-218)
__device__ __forceinline__ float schlick(float cosNL, float n1, float n2) {
    float q = (n1 - n2) / (n1 + n2);
    float f0 = q * q;
    float c = 1.f - cosNL;
    float c2 = c * c;
    float c5 = c2 * c2 * c;
    return f0 + (1.f - f0) * c5;
}

// the surface interaction of one bounce of lane L at hit h (PhotonTracing.cu:278-326);
// returns false when the path ends
template <class LaneT>
__device__ __forceinline__ bool shade(const KParams& P, LaneT& L, const Hit& h, float* sior, int* sid, int64_t j) {
    const DevScene& S = P.S;
    const int model = hit_model(S, h.tri);
    const Material m = load_mat(S, model);
    V3 n = shading_normal(S, h);
    V3 ip = vadd(vscale(L.ray.d, h.t), L.ray.o);
    if (vdot(L.ray.d, n) > 0) n = vscale(n, -1.f);
    float cosNL = vdot(vneg(L.ray.d), n);
    V3 mdiff = tri_albedo(S, h.tri, m);

    int dest;
    bool refr = false;
    if (m.opaque != 1.f) {
        float n1, n2;
        if (L.sn == 0) { n1 = S.default_ior; n2 = m.ior; }
        else if (sid[L.sn - 1] == model) { n1 = sior[L.sn - 1]; n2 = L.sn == 1 ? S.default_ior : sior[L.sn - 2]; }
        else { n1 = sior[L.sn - 1]; n2 = m.ior; }
        float cang;
        bool tir = critical_angle(S, n1, n2, cang) && cosNL <= cang;
        if (!tir) {
            float pr = 1.f - schlick(cosNL, n1, n2);
            float e = L.st.next(P);
            refr = !(e > pr);
        }
    }
    if (refr) {
        dest = REFR;
    } else {
        float max_lp = vmax3(P.power);
        float e = 0.f + L.st.next(P) * (2.f - 0.f);
        float pd = vmax3(vmul(mdiff, P.power)) / max_lp;
        if (e <= pd) dest = DIF;
        else {
            float ps = vmax3(vmul(m.specular, P.power)) / max_lp;
            dest = (e <= pd + ps) ? SPEC : ABSORB;
        }
    }

    Ray nr;
    nr.o = v3(0.f, 0.f, 0.f); nr.d = v3(0.f, 0.f, 0.f);
    bool alive = true;
    if (dest == REFR) {
        float n1, n2;
        if (L.sn != 0 && sid[L.sn - 1] == model) {
            n1 = sior[L.sn - 1];
            n2 = L.sn == 1 ? S.default_ior : sior[L.sn - 2];
            L.sn--;
        } else {
            bool was_empty = L.sn == 0;
            float top_ior = was_empty ? 0.f : sior[L.sn - 1];
            if (L.sn < P.max_bounces && L.sn < MAX_STACK) { sior[L.sn] = m.ior; sid[L.sn] = model; L.sn++; }
            else raise_status(P.status, ST_STACK);
            n1 = was_empty ? S.default_ior : top_ior;
            n2 = m.ior;
        }
        if (!ray_refract(L.ray, ip, n, n1, n2, nr)) alive = false;
    } else if (dest == DIF || (dest == ABSORB && !vnear(m.specular, v3(1.f, 1.f, 1.f)))) {
        bool caustic = (L.last == SPEC || L.last == REFR) && L.diffuse_surfs == 0;
        int slot = L.ng + L.nc;
        size_t o = (size_t)slot * (size_t)P.npaths + (size_t)j;
        P.stage[2 * o] = make_float4(ip.x, ip.y, ip.z, __int_as_float(caustic ? 2 : 1));
        P.stage[2 * o + 1] = make_float4(L.ray.d.x, L.ray.d.y, L.ray.d.z, 0.f);
        if (caustic) L.nc++; else L.ng++;
    } else if (dest == SPEC) {
        nr = ray_reflect(L.ray, ip, n);
    }
    if (dest == DIF) {
        nr = diffuse_bounce(ip, n, L.st, P);
        L.diffuse_surfs++;
    }
    L.last = dest;
    if (dest == ABSORB || !alive) return false;
    L.ray = nr;
    return true;
}

// Lane states of k_trace.
enum { L_IDLE = 0, L_RAY = 1, L_TRACE = 2, L_HIT = 3, L_DONE = 4 };

// Persistent photon tracer.  Each lane runs a small state machine:
//   IDLE  -> takes the next path of the batch (RAY) or finds none (DONE);
//   RAY   -> starts the traversal of its current ray (TRACE);
//   TRACE -> traversal rounds; a completed query moves it to HIT;
//   HIT   -> the second pass of the t == 0 rule (TRACE), or the surface
//            interaction: the next ray (RAY) or the end of the path (IDLE).
// A warp leaves its traversal loop as soon as P.refill of its lanes have
// finished their query, serves those lanes, and resumes: lanes whose ray is
// long (rays grazing the heightfield cross hundreds of leaves) keep their
// traversal state while the others get new rays, instead of holding the whole
// warp until the longest ray of a bounce is done.
// COUNT: the work-counting variant (the same photons; each thread adds its
// rays, node visits and triangle tests to P.work at the end).
template <bool COUNT>
__global__ void __launch_bounds__(TRACE_THREADS, TRACE_MIN_BLOCKS)
k_trace(KParams P) {
    const int lane = threadIdx.x & 31;
    Lane<ParamStream> L;
    Trav T;
    std::conditional_t<COUNT, Work, NoWork> work;
    unsigned rays = 0;
    __shared__ int stack_cols[TRACE_SMEM_STACK * TRACE_THREADS];
    TraceStack stack;
    stack.col = stack_cols + threadIdx.x;
    float sior[MAX_STACK];
    int sid[MAX_STACK];
    int64_t j = -1;          // batch-local path index of this lane
    int state = L_IDLE;
    while (true) {
        const bool need = state == L_IDLE;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(P.counter, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const unsigned long long mine = base + (unsigned long long)__popc(m & lanemask_lt());
                if ((int64_t)mine < P.npaths) {
                    j = (int64_t)mine;
                    start_path(P, L, P.p0 + j);
                    state = L_RAY;
                } else {
                    state = L_DONE;
                }
            }
        }
        if (__all_sync(0xffffffffu, state == L_DONE)) break;
        if (state == L_RAY) {
            trav_init(T, L.ray.o, L.ray.d, stack);
            if (COUNT) rays++;
            state = L_TRACE;
        }
        while (true) {
            const bool tr = state == L_TRACE;
            if (!__any_sync(0xffffffffu, tr)) break;
            if (__popc(__ballot_sync(0xffffffffu, state == L_HIT)) >= P.refill) break;
            if (tr && trav_step<TRACE_CUT>(P.S, T, L.ray.o, L.ray.d, stack, work)) state = L_HIT;
        }
        if (state == L_HIT) {
            Hit h;
            const int r = trav_resolve(P.S, T, h, stack);
            if (r == TRAV_AGAIN) {
                state = L_TRACE;
            } else {
                const bool alive = r == TRAV_HIT && shade(P, L, h, sior, sid, j);
                L.bounce++;
                if (!alive || L.bounce > P.max_bounces - 1) {
                    P.cnt_g[j] = (uint32_t)L.ng;
                    P.cnt_c[j] = (uint32_t)L.nc;
                    j = -1;
                    state = L_IDLE;
                } else {
                    state = L_RAY;
                }
            }
        }
    }
    if constexpr (COUNT) {
        unsigned long long v[3] = {rays, work.nodes, work.tri_tests};
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
            if (lane == 0) atomicAdd(P.work + c, v[c]);
        }
    }
}

// Several scene instances in one launch: one queue over the concatenated path
// ranges; a lane that takes global path g traces path g - off[i] (+ the
// instance's p0) of instance i, off[i] <= g < off[i+1], with that instance's
// parameters (tab[i]: scene, stream seed, power; stage and count arrays are
// shared, indexed by g with stride tab[i].npaths = the total).  The photons of
// each instance are those of a single-instance trace of it.
__device__ __forceinline__ int find_instance(const int64_t* __restrict__ off, int ninst, int64_t g) {
    int lo = 0, hi = ninst - 1;   // last i with off[i] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(TRACE_THREADS, TRACE_MIN_BLOCKS)
k_trace_multi(const KParams* __restrict__ tab, const int64_t* __restrict__ off, int ninst, int64_t total,
              unsigned long long* counter, int refill) {
    const int lane = threadIdx.x & 31;
    Lane<RegStream> L;
    Trav T;
    __shared__ int stack_cols[TRACE_SMEM_STACK * TRACE_THREADS];
    TraceStack stack;
    stack.col = stack_cols + threadIdx.x;
    float sior[MAX_STACK];
    int sid[MAX_STACK];
    int64_t j = -1;          // global path index of this lane
    int inst = 0;
    int state = L_IDLE;
    while (true) {
        const bool need = state == L_IDLE;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const unsigned long long mine = base + (unsigned long long)__popc(m & lanemask_lt());
                if ((int64_t)mine < total) {
                    j = (int64_t)mine;
                    inst = find_instance(off, ninst, j);
                    const KParams& P = tab[inst];
                    start_path(P, L, P.p0 + (j - __ldg(off + inst)));
                    state = L_RAY;
                } else {
                    state = L_DONE;
                }
            }
        }
        if (__all_sync(0xffffffffu, state == L_DONE)) break;
        const KParams& P = tab[inst];
        if (state == L_RAY) {
            trav_init(T, L.ray.o, L.ray.d, stack);
            state = L_TRACE;
        }
        while (true) {
            const bool tr = state == L_TRACE;
            if (!__any_sync(0xffffffffu, tr)) break;
            if (__popc(__ballot_sync(0xffffffffu, state == L_HIT)) >= refill) break;
            if (tr && trav_step<TRACE_CUT>(P.S, T, L.ray.o, L.ray.d, stack)) state = L_HIT;
        }
        if (state == L_HIT) {
            Hit h;
            const int r = trav_resolve(P.S, T, h, stack);
            if (r == TRAV_AGAIN) {
                state = L_TRACE;
            } else {
                const bool alive = r == TRAV_HIT && shade(P, L, h, sior, sid, j);
                L.bounce++;
                if (!alive || L.bounce > P.max_bounces - 1) {
                    P.cnt_g[j] = (uint32_t)L.ng;
                    P.cnt_c[j] = (uint32_t)L.nc;
                    j = -1;
                    state = L_IDLE;
                } else {
                    state = L_RAY;
                }
            }
        }
    }
}

// Canonical-order append of a multi-instance trace: instance i's global-map
// photons go to pos/dir/pow[ph0[i] + local offset], cut at cap[i];
// inst_total[i] = global photons the instance produced before the cut.  A
// batch builds no caustic map: caustic photons are dropped.
__global__ void k_compact_multi(int64_t total, const int64_t* __restrict__ off, int ninst,
                                const TraceInstOut* __restrict__ io, const float4* __restrict__ stage,
                                const uint32_t* __restrict__ cnt_g,
                                const uint32_t* __restrict__ cnt_c, const uint32_t* __restrict__ scan_g,
                                const uint32_t* __restrict__ grand_total, float* gpos, float* gdir, float* gpow,
                                int64_t* __restrict__ inst_total) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ninst) {
        const int64_t a = __ldg(off + g), b = __ldg(off + g + 1);
        const uint32_t sa = a < total ? scan_g[a] : *grand_total;
        const uint32_t sb = b < total ? scan_g[b] : *grand_total;
        inst_total[g] = (int64_t)(sb - sa);
    }
    if (g >= total) return;
    const int i = find_instance(off, ninst, g);
    const TraceInstOut o = io[i];
    int64_t og = (int64_t)(scan_g[g] - scan_g[__ldg(off + i)]);
    const int slots = (int)(cnt_g[g] + cnt_c[g]);
    for (int k = 0; k < slots && og < o.cap; k++) {
        const size_t sidx = (size_t)k * (size_t)total + (size_t)g;
        const float4 p = stage[2 * sidx];
        if (__float_as_int(p.w) == 2) continue;
        const float4 d = stage[2 * sidx + 1];
        const int64_t idx = o.ph0 + og++;
        gpos[3 * idx] = p.x; gpos[3 * idx + 1] = p.y; gpos[3 * idx + 2] = p.z;
        gdir[3 * idx] = d.x; gdir[3 * idx + 1] = d.y; gdir[3 * idx + 2] = d.z;
        gpow[3 * idx] = o.power[0]; gpow[3 * idx + 1] = o.power[1]; gpow[3 * idx + 2] = o.power[2];
    }
}

__global__ void k_lists_from_rec(const float4* __restrict__ rec, int64_t n, V3 pw, float* dir, float* pow) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (dir) {
        const float4 d = rec[2 * i + 1];
        dir[3 * i] = d.x; dir[3 * i + 1] = d.y; dir[3 * i + 2] = d.z;
    }
    pow[3 * i] = pw.x; pow[3 * i + 1] = pw.y; pow[3 * i + 2] = pw.z;
}

// canonical-order append of one batch into the two photon lists
// (rec lists, when set: each photon's position and direction also as one
// 32-byte record, which the grid build gathers with one sector read)
__global__ void k_compact(int64_t npaths, const float4* __restrict__ stage,
                          const uint32_t* __restrict__ cnt_g, const uint32_t* __restrict__ cnt_c,
                          const uint32_t* __restrict__ scan_g, const uint32_t* __restrict__ scan_c, V3 power,
                          float* gpos, float* gdir, float* gpow, int64_t gcap, int64_t gfilled, float4* grec,
                          bool glists, float* cpos, float* cdir, float* cpow, int64_t ccap, int64_t cfilled,
                          float4* crec, bool clists) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= npaths) return;
    int ng = (int)cnt_g[j], nc = (int)cnt_c[j];
    int64_t og = gfilled + scan_g[j], oc = ccap > 0 ? cfilled + scan_c[j] : 0;
    for (int k = 0; k < ng + nc; k++) {
        size_t o = (size_t)k * (size_t)npaths + (size_t)j;
        float4 p = stage[2 * o];
        float4 d = stage[2 * o + 1];
        bool caustic = __float_as_int(p.w) == 2;
        float *dp, *dd, *dw;
        float4* dr;
        bool lists;
        int64_t idx;
        if (caustic) {
            if (oc >= ccap) { oc++; continue; }
            idx = oc++; dp = cpos; dd = cdir; dw = cpow; dr = crec; lists = clists;
        } else {
            if (og >= gcap) { og++; continue; }
            idx = og++; dp = gpos; dd = gdir; dw = gpow; dr = grec; lists = glists;
        }
        dp[3 * idx] = p.x; dp[3 * idx + 1] = p.y; dp[3 * idx + 2] = p.z;
        if (lists) {   // else rec carries the direction and the power is the batch's
            dd[3 * idx] = d.x; dd[3 * idx + 1] = d.y; dd[3 * idx + 2] = d.z;
            dw[3 * idx] = power.x; dw[3 * idx + 1] = power.y; dw[3 * idx + 2] = power.z;
        }
        if (dr) {
            dr[2 * idx] = make_float4(p.x, p.y, p.z, 0.f);
            dr[2 * idx + 1] = make_float4(d.x, d.y, d.z, 0.f);
        }
    }
}

}  // namespace

size_t trace_multi_table_bytes(int ninst) { return (size_t)ninst * sizeof(KParams); }

cudaError_t trace_multi_tables(const TraceMulti& M, const TraceInst* insts, cudaStream_t st) {
    std::vector<KParams> tab((size_t)M.ninst);
    for (int i = 0; i < M.ninst; i++) {
        KParams& P = tab[(size_t)i];
        const TraceInst& I = insts[i];
        P.S = I.S; P.seed = I.seed; P.tag = I.tag; P.max_bounces = I.max_bounces;
        P.p0 = I.p0; P.npaths = M.total;
        P.power = v3(I.power[0], I.power[1], I.power[2]);
        P.counter = M.path_counter;
        P.stage = M.stage;
        P.cnt_g = M.cnt_g; P.cnt_c = M.cnt_c;
        P.status = M.status;
        P.refill = M.refill > 0 ? std::min(M.refill, 32) : TRACE_REFILL;
        P.work = nullptr;
        round_keys(P);
    }
    cudaError_t e = cudaMemcpyAsync(M.table, tab.data(), tab.size() * sizeof(KParams), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t trace_multi(const TraceMulti& M, cudaStream_t st) {
    cudaError_t e;
    if (M.total <= 0) return cudaSuccess;
    if ((e = cudaMemsetAsync(M.path_counter, 0, 8, st)) != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_multi, TRACE_THREADS, 0)) != cudaSuccess)
        return e;
    const int64_t want = (M.total + TRACE_THREADS - 1) / TRACE_THREADS;
    const int64_t grid = std::min<int64_t>(want, (int64_t)std::max(per_sm, 1) * M.sm_count);
    const int refill = M.refill > 0 ? std::min(M.refill, 32) : TRACE_REFILL;
    k_trace_multi<<<(unsigned)grid, TRACE_THREADS, 0, st>>>((const KParams*)M.table, M.path_off, M.ninst, M.total,
                                                            M.path_counter, refill);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = scan_u32(M.cnt_g, M.scan_g, M.total, 0, M.totals, M.scan_ws, M.status, st)) != cudaSuccess) return e;
    const int64_t n = std::max<int64_t>(M.total, M.ninst);
    k_compact_multi<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        M.total, M.path_off, M.ninst, M.outs, M.stage, M.cnt_g, M.cnt_c, M.scan_g, M.totals, M.pos,
        M.dir, M.pow, M.inst_total);
    return cudaGetLastError();
}

cudaError_t trace_batch(TraceBatch& B, PhotonList& G, PhotonList& C, cudaStream_t st) {
    cudaError_t e;
    if (B.npaths <= 0) return cudaSuccess;
    if ((e = cudaMemsetAsync(B.path_counter, 0, 8, st)) != cudaSuccess) return e;
    KParams P;
    P.S = B.S; P.seed = B.seed; P.tag = B.tag; P.max_bounces = B.max_bounces;
    P.p0 = B.p0; P.npaths = B.npaths;
    P.power = v3(B.power[0], B.power[1], B.power[2]);
    P.counter = B.path_counter;
    P.stage = B.stage;
    P.cnt_g = B.cnt_g; P.cnt_c = B.cnt_c;
    P.status = B.status;
    P.refill = B.refill > 0 ? std::min(B.refill, 32) : TRACE_REFILL;
    P.work = B.work;
    round_keys(P);
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<false>, TRACE_THREADS, 0)) != cudaSuccess)
        return e;
    int64_t want = (B.npaths + TRACE_THREADS - 1) / TRACE_THREADS;
    int64_t grid = std::min<int64_t>(want, (int64_t)std::max(per_sm, 1) * B.sm_count);
    if (B.k_begin && (e = cudaEventRecord(B.k_begin, st)) != cudaSuccess) return e;
    if (B.work) k_trace<true><<<(unsigned)grid, TRACE_THREADS, 0, st>>>(P);
    else k_trace<false><<<(unsigned)grid, TRACE_THREADS, 0, st>>>(P);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (B.k_end && (e = cudaEventRecord(B.k_end, st)) != cudaSuccess) return e;
    if ((e = scan_u32(B.cnt_g, B.scan_g, B.npaths, 0, B.totals, B.scan_ws, B.status, st)) != cudaSuccess) return e;
    // no caustic map: its counts still steer the loop below, its offsets are not needed
    if (C.cap > 0 && (e = scan_u32(B.cnt_c, B.scan_c, B.npaths, 0, B.totals + 1, B.scan_ws, B.status, st)) != cudaSuccess)
        return e;
    k_compact<<<(unsigned)((B.npaths + 255) / 256), 256, 0, st>>>(
        B.npaths, B.stage, B.cnt_g, B.cnt_c, B.scan_g, B.scan_c, P.power,
        G.pos, G.dir, G.pow, G.cap, G.filled, G.rec, G.lists || !G.rec, C.pos, C.dir, C.pow, C.cap, C.filled, C.rec,
        C.lists || !C.rec);
    return cudaGetLastError();
}

cudaError_t photon_lists_from_rec(const float4* rec, int64_t n, const float pw[3], float* dir, float* pow,
                                  cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_lists_from_rec<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rec, n, v3(pw[0], pw[1], pw[2]), dir, pow);
    return cudaGetLastError();
}

}  // namespace pm
