// pm_oracle.cpp -- CPU restatement of the reference photon-mapping hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is linked by
// the test-suite, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
// reference leg, and nowhere else.  The product (the CUDA library under
// cuda-photon-mapping_b200/) never calls into it.
//
// Every function restates one piece of Alator-ux/Cuda-Photon-Mapping
// (paths relative to that project, CPM = CudaPhotonMapping/):
//   Philox stream        : replaces curand (CPM/CudaRandom.cu:6-11) with an injected,
//                          counter-based stream per photon path (Salmon et al., SC'11).
//   light sampling       : CPM/Model.cuh:202-243, CPM/CudaRandom.cuh:9-15
//   emission direction   : CPM/PhotonTracing.cu:350-369
//   intersection         : CPM/Model.cuh:69-120, 366-446; CPM/AABB.cuh:103-111;
//                          CPM/PhotonTracing.cu:178-213; CPM/Raytracer.cuh:66-93
//   bounce logic         : CPM/PhotonTracing.cu:127-326, CPM/PathOperator.cuh:7-42
//   ray ops              : CPM/Ray.cuh:16-96
//   critical angles      : CPM/PhotonTracing.cu:71-125, CPM/HashMap.cuh:9-85
//   photon grid          : CPM/PhotonGrid.cu:10-218 (count, exclusive scan, scatter)
//   kNN + max-heap       : CPM/PhotonGrid.cu:222-284, CPM/PhotonMaxHeap.cuh:43-127
//   radiance estimate    : CPM/Raytracer.cuh:110-138
//   eye pass             : CPM/Raytracer.cuh:95-241, CPM/RaytracePlanner.cuh:30-69,
//                          CPM/MediumManager.cuh:17-79, CPM/MMInnerStack.cuh,
//                          CPM/MMOuterStack.cuh, CPM/RayPlanStack.cuh
//   camera               : CPM/Camera.cuh:43-81
//
// Arithmetic contract: IEEE binary32, round-to-nearest, no FMA contraction
// (built with -ffp-contract=off), every vec3 expression evaluated in the same
// order as the reference's host build (the non-__CUDA_ARCH__ branch of
// CPM/vec3.cuh).  Two integer powers are spelled out as products
// (Fresnel-Schlick, pm_pow5 below); both the oracle and the CUDA kernels use
// the same spelling so decisions taken on them agree bit for bit.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp -shared).

#include <cmath>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <utility>
#include <map>

#include "philox.h"

namespace {

// ---------------------------------------------------------------- vec3 ------
struct V3 { float x, y, z; };
static inline V3 v3(float a, float b, float c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
// float * vec3 and vec3 * float are both (t*v.x, t*v.y, t*v.z) on the host (CPM/vec3.cuh:365-389)
static inline V3 vscale(V3 a, float t) { return v3(t * a.x, t * a.y, t * a.z); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
// dot: x*x' + y*y' + z*z' left to right (CPM/vec3.cuh:272)
static inline float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b) {   // CPM/vec3.cuh:297-299
    return v3(a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x);
}
static inline float vlength(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline bool vnull(V3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
// member normalize(): *this /= length()  ->  u = 1/len; x *= u ... (CPM/vec3.cuh:156-169, 211-224)
static inline V3 vnormalize_member(V3 a) {
    if (vnull(a)) return a;
    float u = 1.0f / vlength(a);
    return v3(a.x * u, a.y * u, a.z * u);
}
// static normalize(v): v / v.length() componentwise division (CPM/vec3.cuh:226-241, 391-402)
static inline V3 vnormalize_static(V3 a) {
    if (vnull(a)) return a;
    float l = vlength(a);
    return v3(a.x / l, a.y / l, a.z / l);
}
static inline float vmax3(V3 a) { return std::fmax(std::fmax(a.x, a.y), a.z); }
static inline V3 vclamp_le(V3 a, float m) { return v3(std::fmin(a.x, m), std::fmin(a.y, m), std::fmin(a.z, m)); }
// vec3::equal with eps 1e-3 (CPM/vec3.cuh:15, 507-513)
static inline bool vequal_eps(V3 a, V3 b) {
    return std::fabs(a.x - b.x) < 0.001f && std::fabs(a.y - b.y) < 0.001f && std::fabs(a.z - b.z) < 0.001f;
}
static inline V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }
static inline void st3(float* p, V3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }

using namespace oracle_rng;

// -------------------------------------------------------------- scene -------
struct Mat { V3 diffuse, specular, emission; float ior, opaque, shininess; };

struct Scene {
    int ntri = 0;
    std::vector<float> pos, nrm;        // 9 floats per triangle (v0 v1 v2)
    std::vector<int> tri_model;         // model index of each triangle, non-decreasing
    std::vector<float> tri_diffuse;     // optional per-triangle diffuse override (3 per tri)
    int nmodel = 0;
    std::vector<Mat> mats;              // one per model
    std::vector<int> mfirst, mcount;    // triangle range of each model
    std::vector<float> maabb;           // 6 per model: min xyz, max xyz
    int light_model = 0;
    V3 light_intensity;
    float default_ior = 1.f;
    // critical angle table: (n1, n2) -> cos(asin(n2/n1)) for n2/n1 < 1
    std::vector<std::pair<std::pair<uint32_t, uint32_t>, float>> ca;
    float scene_aabb[6];
};

static uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// CPM/PhotonTracing.cu:71-77
static void calc_angle(Scene& s, float eta1, float eta2) {
    float eta = eta2 / eta1;
    if (eta < 1.f) {
        auto key = std::make_pair(fbits(eta1), fbits(eta2));
        for (auto& kv : s.ca) if (kv.first == key) return;
        float cang = std::cos(std::asin(eta));
        s.ca.push_back(std::make_pair(key, cang));
    }
}
// CPM/PhotonTracing.cu:79-125 (the hash map only stores these pairs; lookup is by exact bits)
static void build_critical_angles(Scene& s) {
    s.ca.clear();
    for (int i = 0; i < s.nmodel - 1; i++)
        for (int j = i + 1; j < s.nmodel; j++) {
            calc_angle(s, s.mats[i].ior, s.mats[j].ior);
            calc_angle(s, s.mats[j].ior, s.mats[i].ior);
        }
    for (int i = 0; i < s.nmodel; i++) {
        calc_angle(s, s.default_ior, s.mats[i].ior);
        calc_angle(s, s.mats[i].ior, s.default_ior);
    }
}
static bool ca_lookup(const Scene& s, float n1, float n2, float& out) {
    auto key = std::make_pair(fbits(n1), fbits(n2));
    for (auto& kv : s.ca) if (kv.first == key) { out = kv.second; return true; }
    return false;
}

// --------------------------------------------------------- intersection ----
struct Ray { V3 o, d; };

// AABB slab test with division (CPM/AABB.cuh:115-127, 200-208)
static bool aabb_hit(const float* c, const Ray& r) {
    float tmin = 0.0f, tmax = INFINITY;
    const float o[3] = {r.o.x, r.o.y, r.o.z};
    const float d[3] = {r.d.x, r.d.y, r.d.z};
    for (int i = 0; i < 3; i++) {
        bool sign = std::signbit(d[i]);
        float bmin = c[sign * 3 + i];
        float bmax = c[(!sign) * 3 + i];
        float dmin = (bmin - o[i]) / d[i];
        float dmax = (bmax - o[i]) / d[i];
        tmin = std::fmax(dmin, tmin);
        tmax = std::fmin(dmax, tmax);
    }
    return tmin <= tmax;
}

// Edge-function triangle test (CPM/Model.cuh:69-120)
static bool tri_hit(const Ray& ray, V3 v0, V3 v1, V3 v2, float& t, V3& uvw) {
    t = 0.f;
    V3 e1 = vsub(v1, v0), e2 = vsub(v2, v0);
    V3 n = vcross(e1, e2);
    float denom = 1.0f / vdot(n, n);
    float ndd = vdot(n, ray.d);
    if (std::fabs(ndd) < 1e-6f) return false;
    t = (vdot(n, v0) - vdot(n, ray.o)) / ndd;
    if (t < 0) return false;
    V3 P = vadd(ray.o, vscale(ray.d, t));
    V3 sd = vsub(P, v0);
    float w = vdot(n, vcross(e1, sd));
    if (w < 0) return false;
    V3 f = vsub(v0, v2);
    V3 g = vsub(P, v2);
    float v = vdot(n, vcross(f, g));
    if (v < 0) return false;
    w = w * denom;
    v = v * denom;
    float u = 1.f - v - w;
    if (u < 0) return false;
    uvw = v3(u, v, w);
    return true;
}

struct Hit { float t; int model; int tri; V3 uvw; };

// Closest hit over all models: model AABB gate, then a linear triangle loop with
// strict '<' (CPM/Model.cuh:366-446), models combined with the 'intersection == 0'
// sentinel and strict '<' (CPM/PhotonTracing.cu:187-198, CPM/Raytracer.cuh:73-84).
static bool intersect(const Scene& s, const Ray& ray, Hit& h) {
    float best = 0.f;
    int bm = -1;
    Hit cand{};
    for (int m = 0; m < s.nmodel; m++) {
        if (!aabb_hit(&s.maabb[6 * m], ray)) continue;
        float tm = FLT_MAX;
        int bt = -1;
        V3 buvw{};
        for (int i = 0; i < s.mcount[m]; i++) {
            int tri = s.mfirst[m] + i;
            const float* p = &s.pos[9 * tri];
            float t; V3 uvw;
            bool ok = tri_hit(ray, ld3(p), ld3(p + 3), ld3(p + 6), t, uvw);
            if (ok && t < tm) { tm = t; bt = tri; buvw = uvw; }
        }
        if (bt < 0) continue;
        if (best == 0.f || tm < best) { best = tm; bm = m; cand.t = tm; cand.model = m; cand.tri = bt; cand.uvw = buvw; }
    }
    if (bm < 0) return false;
    h = cand;
    return true;
}

// interpolated shading normal: n0*u, n1*v, n2*w, add, member-normalize (CPM/Model.cuh:436-443)
static V3 smooth_normal(const Scene& s, const Hit& h) {
    const float* n = &s.nrm[9 * h.tri];
    V3 n0 = vscale(ld3(n), h.uvw.x), n1 = vscale(ld3(n + 3), h.uvw.y), n2 = vscale(ld3(n + 6), h.uvw.z);
    return vnormalize_member(vadd(vadd(n0, n1), n2));
}

static V3 tri_diffuse(const Scene& s, const Hit& h) {
    if (!s.tri_diffuse.empty()) return ld3(&s.tri_diffuse[3 * h.tri]);
    return s.mats[h.model].diffuse;
}

// ------------------------------------------------------------ ray ops ------
// CPM/Ray.cuh:64-71
static Ray reflect(const Ray& r, V3 from, V3 n) {
    float dnd = vdot(r.d, n);
    V3 refl = vsub(r.d, vscale(vscale(n, 2.f), dnd));
    Ray o;
    o.d = vnormalize_static(refl);
    o.o = vadd(from, vscale(n, 0.01f));
    return o;
}
// CPM/Ray.cuh:85-96
static bool refract(const Ray& r, V3 from, V3 n, float r1, float r2, Ray& out) {
    float eta = r1 / r2;
    float c1 = -vdot(r.d, n);
    float w = eta * c1;
    float c2m = (w - eta) * (w + eta);
    if (c2m < -1.f) return false;
    out.d = vadd(vscale(r.d, eta), vscale(n, w - std::sqrt(1.f + c2m)));
    out.o = vadd(from, vscale(vneg(n), 0.01f));
    return true;
}
// CPM/Ray.cuh:16-56: Marsaglia disc, rejected into the hemisphere of n
static Ray reflect_spherical(V3 from, V3 n, Stream& st) {
    V3 d;
    do {
        float x1, x2, s1, s2;
        do {
            x1 = -1.f + st.next() * 2.f;
            x2 = -1.f + st.next() * 2.f;
            s1 = x1 * x1;
            s2 = x2 * x2;
        } while (s1 + s2 >= 1);
        float f = std::sqrt(1.f - s1 - s2);
        d = v3(2.f * x1 * f, 2.f * x2 * f, 1.f - 2.f * (s1 + s2));
    } while (vdot(d, n) < 0);
    Ray r;
    r.d = vnormalize_static(d);
    r.o = vadd(from, vscale(r.d, 0.0001f));
    return r;
}

// ------------------------------------------------------------ tracing ------
enum PathType { DIF = 0, SPEC = 1, ABSORB = 2, REFR = 3, NONE = 4 };

struct TraceOpts {
    uint64_t seed;
    int max_bounces;
    uint32_t tag;
};

struct PhotonRec { V3 pos, power, dir; int64_t path; int bounce; };

// Fresnel-Schlick with the integer powers as products (CPM/PhotonTracing.cu:215-218)
static inline float schlick(float cosNL, float n1, float n2) {
    float q = (n1 - n2) / (n1 + n2);
    float f0 = q * q;
    float c = 1.f - cosNL;
    float c2 = c * c;
    float c5 = c2 * c2 * c;
    return f0 + (1.f - f0) * c5;
}

struct MediumEntry { float ior; int id; };

// One photon path.  Appends its photons (in bounce order) to gl / ca.
// Photon power is intensity / global capacity for every photon (CPM/PhotonTracing.cu:369).
static void trace_path(const Scene& s, const TraceOpts& o, int64_t p, V3 power,
                       std::vector<PhotonRec>& gl, std::vector<PhotonRec>& cau, int* draws_out) {
    Stream st(o.seed, (uint64_t)p, o.tag);
    const int L = s.light_model;
    const int nt = s.mcount[L];
    // light point: triangle index imap_to_range(u, 0, ntri-1) = roundf(0 + u*(ntri-1))
    int k = (int)std::round(0 + st.next() * (float)(nt - 1));
    int tri = s.mfirst[L] + k;
    float bx = st.next();
    float by = 0.f + st.next() * ((1.f - bx) - 0.f);
    float bz = 1.f - bx - by;
    const float* tp = &s.pos[9 * tri];
    const float* tn = &s.nrm[9 * tri];
    V3 point = vadd(vadd(vscale(ld3(tp), bx), vscale(ld3(tp + 3), by)), vscale(ld3(tp + 6), bz));
    V3 lnorm = vadd(vadd(vscale(ld3(tn), bx), vscale(ld3(tn + 3), by)), vscale(ld3(tn + 6), bz));
    Ray ray;
    ray.o = vadd(point, vscale(lnorm, 0.0001f));
    float prob, dt;
    int tries = 0;
    do {
        if (++tries > (1 << 16)) { if (draws_out) *draws_out = (int)st.n; return; }   // light without a usable normal
        ray.d.x = -1.f + st.next() * 2.f;
        ray.d.y = -1.f + st.next() * 2.f;
        ray.d.z = -1.f + st.next() * 2.f;
        ray.d = vnormalize_member(ray.d);
        prob = st.next();
        dt = vdot(ray.d, lnorm);
        if (dt < 0) { dt = -dt; ray.d = vscale(ray.d, -1.f); }
    } while (prob > dt);

    std::vector<MediumEntry> stack;   // photon_trace_stack (CPM/PhotonTraceStack.cuh:40-116)
    const size_t stack_cap = (size_t)o.max_bounces;
    int diffuse_surfs = 0;
    PathType last = NONE;

    for (int b = 0; b < o.max_bounces; b++) {
        Hit h;
        if (!intersect(s, ray, h)) break;       // a miss ends the path, nothing stored
        const Mat& m = s.mats[h.model];
        V3 n = smooth_normal(s, h);
        V3 ip = vadd(vscale(ray.d, h.t), ray.o);
        if (vdot(ray.d, n) > 0) n = vscale(n, -1.f);
        float cosNL = vdot(vneg(ray.d), n);
        V3 mdiff = tri_diffuse(s, h);

        // destiny (CPM/PhotonTracing.cu:220-276)
        PathType dest;
        bool refr = false;
        if (m.opaque != 1.f) {
            float n1, n2;
            if (stack.empty()) { n1 = s.default_ior; n2 = m.ior; }
            else {
                MediumEntry top = stack.back();
                if (top.id == h.model) { n1 = top.ior; n2 = stack.size() == 1 ? s.default_ior : stack[stack.size() - 2].ior; }
                else { n1 = top.ior; n2 = m.ior; }
            }
            float cang;
            bool tir = ca_lookup(s, n1, n2, cang) && cosNL <= cang;
            if (!tir) {
                float pr = 1.f - schlick(cosNL, n1, n2);
                float e = st.next();
                refr = !(e > pr);
            }
        }
        if (refr) dest = REFR;
        else {
            float max_lp = vmax3(power);
            float e = 0.f + st.next() * (2.f - 0.f);
            float pd = vmax3(vmul(mdiff, power)) / max_lp;
            if (e <= pd) dest = DIF;
            else {
                float ps = vmax3(vmul(m.specular, power)) / max_lp;
                dest = (e <= pd + ps) ? SPEC : ABSORB;
            }
        }

        Ray nr{};
        bool alive = true;
        if (dest == REFR) {
            float n1, n2;
            if (!stack.empty() && stack.back().id == h.model) {
                MediumEntry top = stack.back();
                n2 = stack.size() == 1 ? s.default_ior : stack[stack.size() - 2].ior;
                n1 = top.ior;
                stack.pop_back();
            } else {
                bool was_empty = stack.empty();
                float top_ior = was_empty ? 0.f : stack.back().ior;
                if (stack.size() < stack_cap) stack.push_back(MediumEntry{m.ior, h.model});
                n1 = was_empty ? s.default_ior : top_ior;
                n2 = m.ior;
            }
            if (!refract(ray, ip, n, n1, n2, nr)) alive = false;   // no usable ray: path ends
        } else if (dest == DIF || (dest == ABSORB && !vequal_eps(m.specular, v3(1.f, 1.f, 1.f)))) {
            bool caustic = (last == SPEC || last == REFR) && diffuse_surfs == 0;
            PhotonRec rec{ip, power, ray.d, p, b};
            (caustic ? cau : gl).push_back(rec);
        } else if (dest == SPEC) {
            nr = reflect(ray, ip, n);
        }
        if (dest == DIF) nr = reflect_spherical(ip, n, st);
        if (dest == DIF) diffuse_surfs++;
        last = dest;
        if (dest == ABSORB || !alive) break;
        ray = nr;
    }
    if (draws_out) *draws_out = (int)st.n;
}

// ------------------------------------------------------------- grid --------
struct Grid {
    float aabb[6];
    int gx = 0, gy = 0, gz = 0;
    float cell = 0.f;
    std::vector<uint32_t> starts, sizes;
    std::vector<uint32_t> order;   // sorted slot -> source photon index (stable within a cell)
};

// CPM/PhotonGrid.cu:41-56
static void grid_dims(const float* aabb, int n, int desired, int& gx, int& gy, int& gz, float& cell) {
    float sx = std::fabs(aabb[3] - aabb[0]);
    float sy = std::fabs(aabb[4] - aabb[1]);
    float sz = std::fabs(aabb[5] - aabb[2]);
    int N = (n + desired - 1) / desired;
    float volume = sx * sy * sz;
    cell = std::cbrt(volume / N);
    gx = (int)std::ceil(sx / cell);
    gy = (int)std::ceil(sy / cell);
    gz = (int)std::ceil(sz / cell);
}
// CPM/PhotonGrid.cu:10-38
static inline void cell_coords(const float* mn, V3 p, int gx, int gy, int gz, float cell, int& x, int& y, int& z) {
    x = (int)((p.x - mn[0]) / cell);
    y = (int)((p.y - mn[1]) / cell);
    z = (int)((p.z - mn[2]) / cell);
    x = std::min(std::max(x, 0), gx - 1);
    y = std::min(std::max(y, 0), gy - 1);
    z = std::min(std::max(z, 0), gz - 1);
}
static inline uint32_t cell_index(int x, int y, int z, int gx, int gy) {
    return (uint32_t)(x + y * gx + z * gx * gy);
}

// sub-cell of a point inside its cell: fractional part of the cell quotient
static inline int sub_coord(float p, float mn, float cell, int c, int S) {
    float u = (p - mn) / cell;
    float f = u - (float)c;
    int s = (int)(f * (float)S);
    return std::min(std::max(s, 0), S - 1);
}

// Auto sub-division: about 2k photons per sub-cell slab of a surface crossing the fullest cell
static int auto_subdiv(uint32_t max_count, int k_hint) {
    double per = (double)max_count / (2.0 * std::max(k_hint, 1));
    int S = 1;
    while (S < 8 && (double)(2 * S) * (2 * S) <= per) S *= 2;
    return S;
}

// count -> (re-grid if a cell holds more than 5x desired) -> exclusive scan -> stable scatter.
// Inside a cell photons are ordered by sub-cell (S^3 per cell), then by index.
static void grid_build(Grid& g, const float* pos, int n, const float* aabb, int desired, int S_req = 1,
                       int* S_out = nullptr, uint32_t* max_out = nullptr) {
    std::memcpy(g.aabb, aabb, sizeof(g.aabb));
    std::vector<uint32_t> cid(n);
    for (int pass = 0; pass < 2; pass++) {
        int want = pass == 0 ? desired : desired / 5;
        grid_dims(aabb, n, want, g.gx, g.gy, g.gz, g.cell);
        size_t cells = (size_t)g.gx * g.gy * g.gz;
        g.sizes.assign(cells, 0);
        for (int i = 0; i < n; i++) {
            int x, y, z;
            cell_coords(aabb, ld3(pos + 3 * (size_t)i), g.gx, g.gy, g.gz, g.cell, x, y, z);
            cid[i] = cell_index(x, y, z, g.gx, g.gy);
            g.sizes[cid[i]]++;
        }
        uint32_t mx = 0;
        for (auto c : g.sizes) mx = std::max(mx, c);
        if (max_out) *max_out = mx;
        if (pass == 0 && !(mx > (uint32_t)(5 * desired))) break;
    }
    const int S = S_req > 0 ? S_req : auto_subdiv(max_out ? *max_out : 0, 64);
    if (S_out) *S_out = S;
    size_t cells = g.sizes.size();
    g.starts.assign(cells, 0);
    uint32_t acc = 0;
    for (size_t c = 0; c < cells; c++) { g.starts[c] = acc; acc += g.sizes[c]; }
    // stable counting sort by key = cell * S^3 + sub-cell
    const size_t S3 = (size_t)S * S * S;
    std::vector<uint32_t> key(n);
    std::vector<uint32_t> kcount(cells * S3 + 1, 0);
    for (int i = 0; i < n; i++) {
        const float* p = pos + 3 * (size_t)i;
        int x, y, z;
        cell_coords(aabb, ld3(p), g.gx, g.gy, g.gz, g.cell, x, y, z);
        uint32_t sk = (uint32_t)(sub_coord(p[0], aabb[0], g.cell, x, S) +
                                 S * (sub_coord(p[1], aabb[1], g.cell, y, S) + S * sub_coord(p[2], aabb[2], g.cell, z, S)));
        key[i] = cid[i] * (uint32_t)S3 + sk;
        kcount[key[i]]++;
    }
    std::vector<uint32_t> kstart(cells * S3 + 1, 0);
    uint32_t a2 = 0;
    for (size_t k = 0; k < cells * S3; k++) { kstart[k] = a2; a2 += kcount[k]; }
    kstart[cells * S3] = a2;
    g.order.assign(n, 0);
    for (int i = 0; i < n; i++) g.order[kstart[key[i]]++] = (uint32_t)i;
}

// --------------------------------------------------------------- kNN -------
struct GridView {   // a grid plus the photon arrays in sorted (slot) order
    const float* aabb; int gx, gy, gz; float cell;
    const uint32_t* starts; const uint32_t* sizes;
    const float* spos; const float* sdir; const float* spow;   // 3 floats per slot
    const uint32_t* sid;                                         // source id per slot
};

struct Nb { float d; uint32_t slot; uint32_t id; };

// Cell walk order of CPM/PhotonGrid.cu:257-284: home cell first, then the clamped
// cube in z, y, x order without the home cell.  Calls f(slot, dist) for dist <= r.
template <class F>
static void walk(const GridView& g, V3 q, float r, F&& f) {
    int hx, hy, hz;
    cell_coords(g.aabb, q, g.gx, g.gy, g.gz, g.cell, hx, hy, hz);
    uint32_t home = cell_index(hx, hy, hz, g.gx, g.gy);
    int rc = (int)std::ceil(r / g.cell);
    int x0 = std::max(0, hx - rc), y0 = std::max(0, hy - rc), z0 = std::max(0, hz - rc);
    int x1 = std::min(g.gx - 1, hx + rc), y1 = std::min(g.gy - 1, hy + rc), z1 = std::min(g.gz - 1, hz + rc);
    auto visit = [&](uint32_t c) {
        uint32_t st = g.starts[c], sz = g.sizes[c];
        for (uint32_t i = 0; i < sz; i++) {
            uint32_t slot = st + i;
            V3 d = vsub(ld3(g.spos + 3 * (size_t)slot), q);
            float dist = vlength(d);
            if (dist <= r) f(slot, dist);
        }
    };
    visit(home);
    for (int z = z0; z <= z1; z++)
        for (int y = y0; y <= y1; y++)
            for (int x = x0; x <= x1; x++) {
                uint32_t c = cell_index(x, y, z, g.gx, g.gy);
                if (c != home) visit(c);
            }
}

// Bounded max-heap with the exact push / sift rules of CPM/PhotonMaxHeap.cuh:45-107.
struct RefHeap {
    std::vector<std::pair<uint32_t, float>> a;
    int k;
    explicit RefHeap(int kk) : k(kk) { a.reserve(kk); }
    void sift_up(size_t i) {
        while (i > 0) {
            size_t p = (i - 1) / 2;
            if (a[i].second <= a[p].second) break;
            std::swap(a[i], a[p]);
            i = p;
        }
    }
    void sift_down(size_t i) {
        size_t lo = i;
        while (true) {
            size_t largest = i;
            size_t l = 2 * i + 1, r = 2 * i + 2;
            if (l < a.size() && a[l].second > a[lo].second) { largest = l; lo = l; }
            if (r < a.size() && a[r].second > a[lo].second) { largest = r; lo = r; }
            if (largest == i) break;
            std::swap(a[i], a[lo]);
            i = largest;
        }
    }
    void push(uint32_t idx, float d) {
        if ((int)a.size() < k) { a.push_back({idx, d}); sift_up(a.size() - 1); }
        else if (d < a[0].second) { a[0] = {idx, d}; sift_down(0); }
    }
};

// canonical kNN: the k smallest (distance, source id) pairs with distance <= r
static void knn_canonical(const GridView& g, V3 q, float r, int k, std::vector<Nb>& out) {
    out.clear();
    walk(g, q, r, [&](uint32_t slot, float d) { out.push_back(Nb{d, slot, g.sid[slot]}); });
    auto less = [](const Nb& a, const Nb& b) { return a.d < b.d || (a.d == b.d && a.id < b.id); };
    if ((int)out.size() > k) {
        std::nth_element(out.begin(), out.begin() + k, out.end(), less);
        out.resize(k);
    }
    std::sort(out.begin(), out.end(), less);
}
// reference heap kNN: same walk, PhotonMaxHeap semantics; result in heap array order
static void knn_heap(const GridView& g, V3 q, float r, int k, std::vector<Nb>& out) {
    RefHeap h(k);
    walk(g, q, r, [&](uint32_t slot, float d) { h.push(slot, d); });
    out.clear();
    for (auto& e : h.a) out.push_back(Nb{e.second, e.first, g.sid[e.first]});
}

// radiance estimate (CPM/Raytracer.cuh:110-138).  rk = distance of the heap root,
// i.e. the largest selected distance; sum in the order of 'nb'.
static V3 estimate(const GridView& g, const std::vector<Nb>& nb, V3 n, const float* dirs, const float* pows) {
    V3 res = v3(0.f, 0.f, 0.f);
    if (nb.empty()) return res;
    const float alpha = 1.818f, beta = 1.953f;
    float r = 0.f;
    for (auto& e : nb) r = std::max(r, e.d);
    float fr = r * r;
    for (auto& e : nb) {
        V3 pd = ld3(dirs + 3 * (size_t)e.slot);
        float c = vdot(n, vneg(pd));
        if (c > 0) {
            float d = e.d;
            float filter = alpha * (1.f - (1.f - std::exp(-beta * d * d / (2 * fr))) / (1.f - std::exp(-beta)));
            res = vadd(res, vscale(ld3(pows + 3 * (size_t)e.slot), filter));
        }
    }
    float common = 1.f / (3.14159265358979f * (r * r) * 1);
    return vscale(res, common);
}

// ---------------------------------------------------------- eye pass -------
struct Camera {
    V3 pos, fwd, right, up;
    float vw, vh, focal;
    int W, H;
};
// CPM/Camera.cuh:67-81 (u along the row, v from the bottom row up)
static V3 camera_dir(const Camera& c, int x, int y) {
    float u = ((float)x + 0.5f) / c.W;
    float v = ((float)y + 0.5f) / c.H;
    V3 hor = vscale(c.right, c.vw);
    V3 ver = vscale(c.up, c.vh);
    V3 llc = vsub(vsub(vscale(vadd(c.pos, c.fwd), c.focal), vscale(hor, 0.5f)), vscale(ver, 0.5f));
    return vsub(vadd(vadd(llc, vscale(hor, u)), vscale(ver, v)), c.pos);
}
// CPM/Raytracer.cuh:95-107
static V3 hdr(V3 rgb) {
    const float exposure = 0.6f, gamma = 2.2f;
    float t = (float)std::pow((double)exposure, -1);
    V3 e = v3(std::exp(-t * rgb.x), std::exp(-t * rgb.y), std::exp(-t * rgb.z));
    V3 m = vsub(v3(1.f, 1.f, 1.f), e);
    const float rg = 1.0f / gamma;
    return v3(std::pow(m.x, rg), std::pow(m.y, rg), std::pow(m.z, rg));
}

struct RenderOpts {
    int max_depth;
    float r_global, r_caustic;
    int k_global, k_caustic;
    int knn_heap_mode;      // 1: reference max-heap selection, 0: canonical (distance, id)
    int faithful_caustic;   // 1: caustic estimate reads the global map's dir/power (CPM/Raytracer.cuh:203-204)
    int hits_only = 0;      // 1: record the eye path's hits, skip the estimates (they do not steer the path)
};

// One hit of an eye path: where the reference's render_trace would gather
// (point, triangle, shading normal), whether it takes the global estimate
// (flags bit 0), and the path weight `coef` its colour is multiplied by.
struct HitRec { V3 p; int tri; V3 n; uint32_t flags; V3 coef; };

// Per-pixel state of RaytracePlanner + MediumManager with the reference's index
// arithmetic (CPM/MediumManager.cuh:17-79, MMInnerStack.cuh:131, MMOuterStack.cuh:269).
// Storage starts zeroed for every pixel.
struct PixelState {
    int D;              // max_depth: outer capacity and planner capacity
    int DC;             // (max_depth + 1) / 2: inner depth capacity
    int outer_size = 0;
    std::vector<int> cont;            // inner size of the container at each outer position
    std::vector<MediumEntry> data;    // [slot][depth]
    struct Plan { Ray ray; int depth; V3 coef; bool in_object; };
    std::vector<Plan> plans;
    int nplans = 0;
    bool overflow = false;
    explicit PixelState(int d) : D(d), DC((d + 1) / 2) {
        cont.assign(D + 2, 0);
        data.assign((size_t)(D + 2) * DC, MediumEntry{0.f, 0});
        plans.resize(D);
    }
    MediumEntry& at(int slot, int depth) {
        if (slot < 0 || slot > D + 1 || depth < 0 || depth >= DC) { overflow = true; thread_local MediumEntry dummy; dummy = MediumEntry{0.f, 0}; return dummy; }
        return data[(size_t)slot * DC + depth];
    }
};

struct Rgi { float n1, n2; bool in_obj; };

static Rgi get_refractive_indices(PixelState& ps, float def, int model_id, float ior) {
    int L = ps.outer_size;
    if (L == 0) return Rgi{def, ior, true};
    int s = ps.cont[L - 1];
    if (s == 0) return Rgi{def, ior, true};
    MediumEntry med = ps.at(L, s - 1);
    if (med.id == model_id) {
        bool in_obj = s > 1;
        return Rgi{ior, in_obj ? ps.at(L, s - 2).ior : def, in_obj};
    }
    return Rgi{med.ior, ior, true};
}
static void increase_depth(PixelState& ps, bool& max_level) {
    int L = ps.outer_size;
    if (L == 0) { ps.outer_size = 1; L = 1; }
    if (L < ps.D) {
        int count = (ps.D + 1) / 2;
        int other_size = ps.cont[L - 1];
        if (!(ps.outer_size > ps.D - 1)) {
            int to = std::max(other_size - 0, 0);
            int from = std::max(to - count, 0);
            for (int i = from; i < to; i++) ps.at(L, i) = ps.at(L - 1, i);
            ps.cont[ps.outer_size] = to - from;
            ps.outer_size++;
        }
        max_level = false;
    } else {
        max_level = true;
    }
}
static void reduce_depth(PixelState& ps, bool& max_level) {
    if (!max_level && ps.outer_size > 0) ps.outer_size--;
    max_level = false;
}
static void inform(PixelState& ps, int model_id, float ior, bool max_level) {
    int pos = ps.outer_size - 1 - (max_level ? 0 : 1);
    if (pos < 0) { ps.overflow = true; return; }
    int s = ps.cont[pos];
    if (s != 0) {
        MediumEntry med = ps.at(s, s - 1);
        if (med.id == model_id) ps.cont[pos] = s - 1;
    } else {
        if (!(ps.DC == 0 || s > ps.DC - 1)) {
            ps.at(s, s) = MediumEntry{ior, model_id};
            ps.cont[pos] = s + 1;
        }
    }
}
static void push_refraction(PixelState& ps, bool& max_level, const Ray& r, int depth, V3 coef,
                            int model_id, float ior, float opaque, bool in_obj) {
    increase_depth(ps, max_level);
    inform(ps, model_id, ior, max_level);
    if (!(ps.D == 0 || ps.nplans > ps.D - 1)) {
        ps.plans[ps.nplans++] = PixelState::Plan{r, depth + 1, vscale(coef, 1.f - opaque), in_obj};
    }
}
static bool pop_refraction(PixelState& ps, bool& max_level, Ray& r, int& depth, V3& coef, bool& in_obj) {
    reduce_depth(ps, max_level);
    if (ps.nplans == 0) return false;
    const PixelState::Plan& p = ps.plans[--ps.nplans];
    r = p.ray; depth = p.depth; coef = p.coef; in_obj = p.in_object;
    return true;
}

struct Maps {
    GridView g;           // global map
    bool has_c;
    GridView c;           // caustic map
};

// render_trace (CPM/Raytracer.cuh:140-241); returns the pre-tone-map radiance
static V3 render_trace(const Scene& s, const Maps& maps, const RenderOpts& o, Ray ray, int* nhits, bool* overflow,
                       std::vector<HitRec>* rec = nullptr) {
    PixelState ps(o.max_depth);
    int new_depth = 0, cur = -1;
    V3 acc = v3(0.f, 0.f, 0.f), coef = v3(1.f, 1.f, 1.f);
    bool max_level = false;
    bool in_obj = false;
    std::vector<Nb> nb;
    int hits = 0;
    while ((cur < o.max_depth && cur != new_depth) || pop_refraction(ps, max_level, ray, new_depth, coef, in_obj)) {
        cur = new_depth;
        Hit h;
        if (!intersect(s, ray, h)) continue;
        hits++;
        const Mat& m = s.mats[h.model];
        V3 n = smooth_normal(s, h);
        V3 ip = vadd(vscale(ray.d, h.t), ray.o);
        if (in_obj && vdot(ray.d, n) > 0) n = vscale(n, -1.f);
        V3 color = v3(0.f, 0.f, 0.f);
        V3 mdiff = tri_diffuse(s, h);
        if (rec) rec->push_back(HitRec{ip, h.tri, n, (!in_obj && !vnull(mdiff)) ? 1u : 0u, coef});
        if (o.hits_only) {
            // the estimates below only colour the hit; the path goes on the same way
        } else if (!in_obj && !vnull(mdiff)) {
            V3 di_op = vscale(mdiff, m.opaque);
            if (o.knn_heap_mode) knn_heap(maps.g, ip, o.r_global, o.k_global, nb);
            else knn_canonical(maps.g, ip, o.r_global, o.k_global, nb);
            V3 re = estimate(maps.g, nb, n, maps.g.sdir, maps.g.spow);
            color = vadd(color, vscale(vmul(re, di_op), 4.f));
        }
        color = vadd(color, m.emission);
        if (maps.has_c && !o.hits_only) {
            if (o.knn_heap_mode) knn_heap(maps.c, ip, o.r_caustic, o.k_caustic, nb);
            else knn_canonical(maps.c, ip, o.r_caustic, o.k_caustic, nb);
            if ((int)nb.size() == o.k_caustic) {
                const float* dd = o.faithful_caustic ? maps.g.sdir : maps.c.sdir;
                const float* pp = o.faithful_caustic ? maps.g.spow : maps.c.spow;
                V3 t = estimate(maps.c, nb, n, dd, pp);
                color = vadd(color, vscale(t, m.opaque));
            }
        }
        color = vclamp_le(color, 1.f);
        acc = vadd(acc, vmul(color, coef));
        if (m.opaque < 1.f && cur != o.max_depth - 1) {
            Rgi ri = get_refractive_indices(ps, s.default_ior, h.model, m.ior);
            Ray nr;
            if (refract(ray, ip, n, ri.n1, ri.n2, nr))
                push_refraction(ps, max_level, nr, cur, coef, h.model, m.ior, m.opaque, ri.in_obj);
        }
        if (!in_obj && !vnull(m.specular) && cur != o.max_depth - 1) {
            Ray nr = reflect(ray, ip, n);
            float c = std::pow(std::fmax(vdot(nr.d, vneg(ray.d)), 0.0f), m.shininess);
            coef = vmul(coef, vscale(vscale(m.specular, m.opaque), c));
            ray = nr;
            new_depth = cur + 1;
        }
    }
    if (nhits) *nhits = hits;
    if (overflow) *overflow = ps.overflow;
    return acc;
}

static void fill_scene_derived(Scene& s) {
    s.mfirst.assign(s.nmodel, 0);
    s.mcount.assign(s.nmodel, 0);
    s.maabb.assign(6 * (size_t)s.nmodel, 0.f);
    std::vector<int> seen(s.nmodel, 0);
    for (int t = 0; t < s.ntri; t++) {
        int m = s.tri_model[t];
        if (!seen[m]) { s.mfirst[m] = t; seen[m] = 1; }
        s.mcount[m]++;
        for (int v = 0; v < 3; v++) {
            const float* p = &s.pos[9 * (size_t)t + 3 * v];
            float* b = &s.maabb[6 * (size_t)m];
            bool first = (s.mcount[m] == 1 && v == 0);
            for (int a = 0; a < 3; a++) {
                if (first) { b[a] = p[a]; b[a + 3] = p[a]; }
                else { if (p[a] > b[a + 3]) b[a + 3] = p[a]; if (p[a] < b[a]) b[a] = p[a]; }
            }
        }
    }
    // scene AABB: union of model AABBs (CPM/Initializer.cu:197-200)
    for (int a = 0; a < 3; a++) { s.scene_aabb[a] = FLT_MAX; s.scene_aabb[a + 3] = -FLT_MAX; }
    for (int m = 0; m < s.nmodel; m++)
        for (int a = 0; a < 3; a++) {
            s.scene_aabb[a] = std::min(s.scene_aabb[a], s.maabb[6 * m + a]);
            s.scene_aabb[a + 3] = std::max(s.scene_aabb[a + 3], s.maabb[6 * m + a + 3]);
        }
    build_critical_angles(s);
}

}  // namespace

// ============================================================ C ABI =========
extern "C" {

// raw Philox-4x32-10 block: ctr[4] is replaced by the output
void orc_philox_raw(uint32_t* ctr, const uint32_t* key) { philox10(ctr, key[0], key[1]); }

void orc_philox_uniforms(uint64_t seed, uint32_t tag, uint64_t path, int n, float* out) {
    Stream st(seed, path, tag);
    for (int i = 0; i < n; i++) out[i] = st.next();
}

// mats: 12 floats per model (diffuse3, specular3, emission3, ior, opaque, shininess)
void* orc_scene_create(int ntri, const float* pos, const float* nrm, const int* tri_model,
                       const float* tri_diffuse, int nmodel, const float* mats,
                       int light_model, const float* light_intensity, float default_ior) {
    Scene* s = new Scene();
    s->ntri = ntri;
    s->pos.assign(pos, pos + 9 * (size_t)ntri);
    s->nrm.assign(nrm, nrm + 9 * (size_t)ntri);
    s->tri_model.assign(tri_model, tri_model + ntri);
    if (tri_diffuse) s->tri_diffuse.assign(tri_diffuse, tri_diffuse + 3 * (size_t)ntri);
    s->nmodel = nmodel;
    for (int m = 0; m < nmodel; m++) {
        const float* q = mats + 12 * m;
        Mat mt;
        mt.diffuse = ld3(q); mt.specular = ld3(q + 3); mt.emission = ld3(q + 6);
        mt.ior = q[9]; mt.opaque = q[10]; mt.shininess = q[11];
        s->mats.push_back(mt);
    }
    s->light_model = light_model;
    s->light_intensity = ld3(light_intensity);
    s->default_ior = default_ior;
    fill_scene_derived(*s);
    return s;
}
void orc_scene_destroy(void* h) { delete (Scene*)h; }
void orc_scene_aabb(void* h, float* out6) { std::memcpy(out6, ((Scene*)h)->scene_aabb, 24); }
int orc_scene_critical_angles(void* h, float* out, int cap) {   // (n1, n2, cos) triples
    Scene* s = (Scene*)h;
    int n = 0;
    for (auto& kv : s->ca) {
        if (n < cap) {
            float a, b; std::memcpy(&a, &kv.first.first, 4); std::memcpy(&b, &kv.first.second, 4);
            out[3 * n] = a; out[3 * n + 1] = b; out[3 * n + 2] = kv.second;
        }
        n++;
    }
    return n;
}

// closest hit for a batch of rays: out_t, out_model, out_tri, out_normal (smooth, unflipped)
void orc_intersect(void* h, int n, const float* orig, const float* dir,
                   float* out_t, int* out_model, int* out_tri, float* out_n) {
    Scene* s = (Scene*)h;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        Ray r{ld3(orig + 3 * (size_t)i), ld3(dir + 3 * (size_t)i)};
        Hit hh;
        if (intersect(*s, r, hh)) {
            out_t[i] = hh.t; out_model[i] = hh.model; out_tri[i] = hh.tri;
            st3(out_n + 3 * (size_t)i, smooth_normal(*s, hh));
        } else {
            out_t[i] = -1.f; out_model[i] = -1; out_tri[i] = -1; st3(out_n + 3 * (size_t)i, v3(0, 0, 0));
        }
    }
}

// Trace until both maps hold their capacity (canonical order: path, then bounce).
// Output arrays are 3 floats per photon; out_path/out_bounce may be null.
// Returns the number of paths traced, or -1 when max_paths was exhausted first.
int64_t orc_trace_photons(void* h, uint64_t seed, uint32_t tag, int max_bounces,
                          int64_t cap_g, int64_t cap_c, int64_t max_paths,
                          float* g_pos, float* g_pow, float* g_dir, int64_t* g_path, int* g_bounce,
                          float* c_pos, float* c_pow, float* c_dir, int64_t* c_path, int* c_bounce,
                          int64_t* out_ng, int64_t* out_nc) {
    Scene* s = (Scene*)h;
    TraceOpts o{seed, max_bounces, tag};
    V3 power = v3(s->light_intensity.x / (float)cap_g, s->light_intensity.y / (float)cap_g,
                  s->light_intensity.z / (float)cap_g);
    int64_t ng = 0, nc = 0, p0 = 0;
    const int64_t chunk = 8192;
    std::vector<std::vector<PhotonRec>> gl(chunk), ca(chunk);
    while ((ng < cap_g || nc < cap_c) && p0 < max_paths) {
        int64_t cnt = std::min(chunk, max_paths - p0);
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t i = 0; i < cnt; i++) {
            gl[i].clear(); ca[i].clear();
            trace_path(*s, o, p0 + i, power, gl[i], ca[i], nullptr);
        }
        for (int64_t i = 0; i < cnt && (ng < cap_g || nc < cap_c); i++) {
            for (auto& r : gl[i]) if (ng < cap_g) {
                st3(g_pos + 3 * ng, r.pos); st3(g_pow + 3 * ng, r.power); st3(g_dir + 3 * ng, r.dir);
                if (g_path) g_path[ng] = r.path;
                if (g_bounce) g_bounce[ng] = r.bounce;
                ng++;
            }
            for (auto& r : ca[i]) if (nc < cap_c) {
                st3(c_pos + 3 * nc, r.pos); st3(c_pow + 3 * nc, r.power); st3(c_dir + 3 * nc, r.dir);
                if (c_path) c_path[nc] = r.path;
                if (c_bounce) c_bounce[nc] = r.bounce;
                nc++;
            }
            if (ng >= cap_g && nc >= cap_c) { p0 += i + 1; goto done; }
        }
        p0 += cnt;
    }
done:
    *out_ng = ng; *out_nc = nc;
    if (ng < cap_g || nc < cap_c) return -1;
    return p0;
}

// Per-path photon output for paths [p0, p1) without a capacity limit (power of
// every photon = intensity / power_cap).  counts[2*(p-p0)+{0,1}] = photons of the
// path in the global / caustic list; draws[p-p0] = uniforms the path consumed.
// Photons of all paths are written in path order into the g_* and c_* arrays,
// which must hold (p1-p0)*max_bounces entries each.
void orc_trace_paths(void* h, uint64_t seed, uint32_t tag, int max_bounces, int64_t power_cap,
                     int64_t p0, int64_t p1, int* counts, int* draws,
                     float* g_pos, float* g_dir, int* g_bounce, float* c_pos, float* c_dir, int* c_bounce,
                     int64_t* out_ng, int64_t* out_nc) {
    Scene* s = (Scene*)h;
    TraceOpts o{seed, max_bounces, tag};
    V3 power = v3(s->light_intensity.x / (float)power_cap, s->light_intensity.y / (float)power_cap,
                  s->light_intensity.z / (float)power_cap);
    int64_t n = p1 - p0;
    std::vector<std::vector<PhotonRec>> gl(n), ca(n);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; i++) trace_path(*s, o, p0 + i, power, gl[i], ca[i], draws ? draws + i : nullptr);
    int64_t ng = 0, nc = 0;
    for (int64_t i = 0; i < n; i++) {
        counts[2 * i] = (int)gl[i].size(); counts[2 * i + 1] = (int)ca[i].size();
        for (auto& r : gl[i]) { st3(g_pos + 3 * ng, r.pos); st3(g_dir + 3 * ng, r.dir); g_bounce[ng] = r.bounce; ng++; }
        for (auto& r : ca[i]) { st3(c_pos + 3 * nc, r.pos); st3(c_dir + 3 * nc, r.dir); c_bounce[nc] = r.bounce; nc++; }
    }
    *out_ng = ng; *out_nc = nc;
}

// Grid build.  sub_div: sub-cells per cell axis of the in-cell order (1, 2, 4, 8;
// 0 = automatic as the product chooses it); out_sub receives it.
// out_dims = (gx, gy, gz); out_cell; starts/sizes must hold
// max_cells entries; order holds n.  Returns the cell count, or -(cells) if
// max_cells was too small (nothing written but dims).
int64_t orc_grid_build(const float* pos, int n, const float* aabb, int desired, int sub_div, int* out_sub,
                       int* out_dims, float* out_cell, uint32_t* starts, uint32_t* sizes,
                       uint32_t* order, int64_t max_cells) {
    Grid g;
    uint32_t mx = 0;
    grid_build(g, pos, n, aabb, desired, sub_div, out_sub, &mx);
    out_dims[0] = g.gx; out_dims[1] = g.gy; out_dims[2] = g.gz;
    *out_cell = g.cell;
    int64_t cells = (int64_t)g.sizes.size();
    if (cells > max_cells) return -cells;
    std::memcpy(starts, g.starts.data(), 4 * cells);
    std::memcpy(sizes, g.sizes.data(), 4 * cells);
    std::memcpy(order, g.order.data(), 4 * (size_t)n);
    return cells;
}

static GridView make_view(const float* aabb, const int* dims, float cell, const uint32_t* starts,
                          const uint32_t* sizes, const float* spos, const float* sdir, const float* spow,
                          const uint32_t* sid) {
    GridView g;
    g.aabb = aabb; g.gx = dims[0]; g.gy = dims[1]; g.gz = dims[2]; g.cell = cell;
    g.starts = starts; g.sizes = sizes; g.spos = spos; g.sdir = sdir; g.spow = spow; g.sid = sid;
    return g;
}

// kNN + estimate for a batch of query points.  out_ids: k per query (source ids,
// ascending (distance, id) in canonical mode, heap order in heap mode; unused = 0xffffffff);
// out_cnt: neighbours found; out_rk: largest selected distance; out_rad: radiance (3/query).
void orc_gather(const float* aabb, const int* dims, float cell, const uint32_t* starts,
                const uint32_t* sizes, const float* spos, const float* sdir, const float* spow,
                const uint32_t* sid, int nq, const float* qpos, const float* qnrm, float r, int k,
                int heap_mode, uint32_t* out_ids, int* out_cnt, float* out_rk, float* out_rad) {
    GridView g = make_view(aabb, dims, cell, starts, sizes, spos, sdir, spow, sid);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nq; i++) {
        std::vector<Nb> nb;
        V3 q = ld3(qpos + 3 * (size_t)i);
        if (heap_mode) knn_heap(g, q, r, k, nb); else knn_canonical(g, q, r, k, nb);
        float rk = 0.f;
        for (int j = 0; j < k; j++) out_ids[(size_t)i * k + j] = j < (int)nb.size() ? nb[j].id : 0xffffffffu;
        for (auto& e : nb) rk = std::max(rk, e.d);
        out_cnt[i] = (int)nb.size();
        out_rk[i] = rk;
        if (out_rad) st3(out_rad + 3 * (size_t)i, estimate(g, nb, ld3(qnrm + 3 * (size_t)i), sdir, spow));
    }
}

// Camera basis from (position, direction, up, vertical fov, W, H): CPM/Camera.cuh:43-65
void orc_camera(const float* position, const float* direction, const float* upv, float fov_deg, int W, int H,
                float* out /* pos3 fwd3 right3 up3 vw vh focal */) {
    const float pi = 3.141592653589793f;
    float aspect = (float)W / (float)H;
    float theta = fov_deg * pi / 180.0f;
    float hh = std::tan(theta / 2);
    float vh = 2.0f * hh;
    float vw = aspect * vh;
    V3 fwd = vnormalize_static(ld3(direction));
    V3 right = vnormalize_static(vcross(fwd, ld3(upv)));
    V3 up = vcross(right, fwd);
    st3(out, ld3(position)); st3(out + 3, fwd); st3(out + 6, right); st3(out + 9, up);
    out[12] = vw; out[13] = vh; out[14] = 1.0f;
}

// Eye pass over pixel rows [y0, y1) (row 0 = bottom row).  cam: 15 floats as from
// orc_camera.  Maps: global grid required; caustic optional (c_dims null -> none).
// out_rad: 3 floats per pixel of the rows (pre tone map); out_ldr: tone-mapped floats;
// out_rgb8: 3 bytes; out_hits: hits per pixel.  Returns the number of pixels whose
// medium storage overflowed the per-pixel range (0 on well-formed scenes).
int orc_render(void* h, const float* cam, int W, int H, int y0, int y1,
               const float* g_aabb, const int* g_dims, float g_cell, const uint32_t* g_starts,
               const uint32_t* g_sizes, const float* g_spos, const float* g_sdir, const float* g_spow,
               const uint32_t* g_sid,
               const int* c_dims, float c_cell, const uint32_t* c_starts, const uint32_t* c_sizes,
               const float* c_spos, const float* c_sdir, const float* c_spow, const uint32_t* c_sid,
               int max_depth, float r_global, int k_global, float r_caustic, int k_caustic,
               int heap_mode, int faithful_caustic,
               float* out_rad, float* out_ldr, uint8_t* out_rgb8, int* out_hits) {
    Scene* s = (Scene*)h;
    Camera c;
    c.pos = ld3(cam); c.fwd = ld3(cam + 3); c.right = ld3(cam + 6); c.up = ld3(cam + 9);
    c.vw = cam[12]; c.vh = cam[13]; c.focal = cam[14]; c.W = W; c.H = H;
    Maps maps;
    maps.g = make_view(g_aabb, g_dims, g_cell, g_starts, g_sizes, g_spos, g_sdir, g_spow, g_sid);
    maps.has_c = c_dims != nullptr;
    if (maps.has_c) maps.c = make_view(g_aabb, c_dims, c_cell, c_starts, c_sizes, c_spos, c_sdir, c_spow, c_sid);
    RenderOpts o{max_depth, r_global, r_caustic, k_global, k_caustic, heap_mode, faithful_caustic};
    int overflow_px = 0;
    int64_t npx = (int64_t)(y1 - y0) * W;
#pragma omp parallel for schedule(dynamic, 32) reduction(+ : overflow_px)
    for (int64_t i = 0; i < npx; i++) {
        int x = (int)(i % W), y = y0 + (int)(i / W);
        Ray r;
        r.o = c.pos;
        r.d = vnormalize_static(camera_dir(c, x, y));
        int hits = 0; bool ovf = false;
        V3 rad = render_trace(*s, maps, o, r, &hits, &ovf);
        if (ovf) overflow_px++;
        V3 l = vclamp_le(hdr(rad), 1.f);
        if (out_rad) st3(out_rad + 3 * i, rad);
        if (out_ldr) st3(out_ldr + 3 * i, l);
        if (out_rgb8) {
            out_rgb8[3 * i] = (uint8_t)(l.x * 255);
            out_rgb8[3 * i + 1] = (uint8_t)(l.y * 255);
            out_rgb8[3 * i + 2] = (uint8_t)(l.z * 255);
        }
        if (out_hits) out_hits[i] = hits;
    }
    return overflow_px;
}

// The eye paths of the given pixels (px[i] = y * W + x) as the reference's
// render_trace walks them (CPM/Raytracer.cuh:140-241), without the estimates:
// per hit, a = (point, triangle bits), b = (shading normal, flags bits: 1 when
// the hit takes the global estimate), c = (path weight, pixel bits), in the
// order the path meets them.  counts[i] = hits of pixel i; the records hold
// `cap` entries.  Returns the number of hits written (-1: cap too small).
int64_t orc_eye_hits(void* h, const float* cam, int W, int H, int64_t npx, const int64_t* px, int max_depth,
                     int* counts, float* out_a, float* out_b, float* out_c, int64_t cap) {
    Scene* s = (Scene*)h;
    Camera c;
    c.pos = ld3(cam); c.fwd = ld3(cam + 3); c.right = ld3(cam + 6); c.up = ld3(cam + 9);
    c.vw = cam[12]; c.vh = cam[13]; c.focal = cam[14]; c.W = W; c.H = H;
    Maps maps{};
    maps.has_c = false;
    RenderOpts o{max_depth, 0.f, 0.f, 0, 0, 0, 0, 1};
    std::vector<std::vector<HitRec>> recs((size_t)npx);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < npx; i++) {
        const int x = (int)(px[i] % W), y = (int)(px[i] / W);
        Ray r;
        r.o = c.pos;
        r.d = vnormalize_static(camera_dir(c, x, y));
        (void)render_trace(*s, maps, o, r, nullptr, nullptr, &recs[i]);
    }
    int64_t k = 0;
    for (int64_t i = 0; i < npx; i++) {
        counts[i] = (int)recs[i].size();
        for (const HitRec& q : recs[i]) {
            if (k >= cap) return -1;
            const uint32_t pix = (uint32_t)px[i];
            st3(out_a + 4 * k, q.p); std::memcpy(out_a + 4 * k + 3, &q.tri, 4);
            st3(out_b + 4 * k, q.n); std::memcpy(out_b + 4 * k + 3, &q.flags, 4);
            st3(out_c + 4 * k, q.coef); std::memcpy(out_c + 4 * k + 3, &pix, 4);
            k++;
        }
    }
    return k;
}

// normalised eye-ray directions for pixels (xs[i], ys[i]); cam as from orc_camera
void orc_camera_rays(const float* cam, int W, int H, int n, const int* xs, const int* ys, float* out) {
    Camera c;
    c.pos = ld3(cam); c.fwd = ld3(cam + 3); c.right = ld3(cam + 6); c.up = ld3(cam + 9);
    c.vw = cam[12]; c.vh = cam[13]; c.focal = cam[14]; c.W = W; c.H = H;
    for (int i = 0; i < n; i++) st3(out + 3 * (size_t)i, vnormalize_static(camera_dir(c, xs[i], ys[i])));
}

// reflect / refract (origin3 dir3) and refract success, as Ray::reflect / Ray::refract
void orc_ray_ops(int n, const float* dir, const float* from, const float* nrm, const float* etas,
                 float* out_reflect, float* out_refract, int* out_ok) {
    for (int i = 0; i < n; i++) {
        Ray r; r.o = v3(0, 0, 0); r.d = ld3(dir + 3 * (size_t)i);
        Ray a = reflect(r, ld3(from + 3 * (size_t)i), ld3(nrm + 3 * (size_t)i));
        Ray b; b.o = v3(0, 0, 0); b.d = v3(0, 0, 0);
        out_ok[i] = refract(r, ld3(from + 3 * (size_t)i), ld3(nrm + 3 * (size_t)i), etas[2 * i], etas[2 * i + 1], b);
        st3(out_reflect + 6 * (size_t)i, a.o); st3(out_reflect + 6 * (size_t)i + 3, a.d);
        st3(out_refract + 6 * (size_t)i, b.o); st3(out_refract + 6 * (size_t)i + 3, b.d);
    }
}

// tone map + clamp to <= 1
void orc_hdr(int n, const float* rgb, float* out) {
    for (int i = 0; i < n; i++) st3(out + 3 * (size_t)i, vclamp_le(hdr(ld3(rgb + 3 * (size_t)i)), 1.f));
}

// Inclusive / exclusive sequential scan (the known-answer check of the grid scan).
void orc_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive) {
    uint32_t acc = 0;
    for (int64_t i = 0; i < n; i++) {
        if (inclusive) { acc += in[i]; out[i] = acc; }
        else { out[i] = acc; acc += in[i]; }
    }
}

}  // extern "C"
