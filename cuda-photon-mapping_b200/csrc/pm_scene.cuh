// pm_scene.cuh -- device scene layout and closest-hit query (BVH traversal).
//
// The reference intersects every ray with every triangle of every model whose
// AABB the ray meets (CudaPhotonMapping/Model.cuh:366-446, AABB.cuh:103-111,
// PhotonTracing.cu:178-213).  Here a binary BVH over all triangles culls the
// search; the answer is kept identical to the reference's:
//   * each triangle is tested with the reference's edge-function test
//     (Model.cuh:69-120); the per-triangle terms that do not depend on the ray
//     (v1-v0, v0-v2, the plane normal, 1/|n|^2, n.v0) are precomputed with the
//     same operations, so every tested value is bit-identical;
//   * the winner is the smallest (t, triangle index) pair.  Triangles are
//     sorted by model, so this is the reference's order: models in index
//     order with strict '<', triangles in index order with strict '<';
//   * a triangle may only win if the reference's slab test of its model's
//     AABB passes for the ray (evaluated lazily, once per model per ray);
//   * BVH node boxes are padded, and a node is skipped only when its entry
//     distance is strictly larger than the best t, so no candidate that could
//     win (including exact ties) is culled.  (The slab arithmetic is
//     fma(box, 1/d, -o/d); the padding dwarfs its rounding.)
#pragma once
#include "pm_device.cuh"

namespace pm {

// Triangle record: 5 float4 = 80 bytes
//   q0 = (v0, n.v0)   q1 = (v1 - v0, 1/(n.n))   q2 = (v2, model bits)
//   q3 = (v0 - v2, 0) q4 = (n, 0)   n = cross(v1 - v0, v2 - v0)
// Leaf-ordered record (tri_leaf): 4 float4 = 64 bytes, one aligned line:
//   q0, q1, q2 as above, (n, the triangle index bits); the test forms v0 - v2
//   from q0 and q2 (the same float subtraction that made q3)
struct DevScene {
    const float4* tri;        // 5 per triangle
    const float* tri_pos;     // 9 per triangle (vertex positions, as given)
    const float* tri_nrm;     // 9 per triangle (vertex normals)
    const float* tri_diffuse; // 3 per triangle or null
    const float4* nodes;      // 4 per interior node: both children's (lo, ref), (hi, -)
    const int* prim;          // leaf triangle indices
    const float4* tri_leaf;   // 4 per triangle in leaf order (record j = triangle prim[j], its index
                              // in the last float4's w), so a leaf's triangles are contiguous
    const float* maabb;       // 6 per model (min xyz, max xyz)
    const float* mats;        // 12 per model
    const float* ca;          // critical angle table: (n1, n2, cos) triples
    int nca;
    int ntri, nmodel;
    int light_first, light_count;
    float default_ior;
};

struct Material {
    V3 diffuse, specular, emission;
    float ior, opaque, shininess;
};
__device__ __forceinline__ Material load_mat(const DevScene& S, int m) {
    const float* q = S.mats + 12 * m;
    Material r;
    r.diffuse = ld3(q); r.specular = ld3(q + 3); r.emission = ld3(q + 6);
    r.ior = q[9]; r.opaque = q[10]; r.shininess = q[11];
    return r;
}
__device__ __forceinline__ V3 tri_albedo(const DevScene& S, int tri, const Material& m) {
    return S.tri_diffuse ? ld3(S.tri_diffuse + 3 * (size_t)tri) : m.diffuse;
}
__device__ __forceinline__ bool critical_angle(const DevScene& S, float n1, float n2, float& out) {
    for (int i = 0; i < S.nca; i++) {
        if (__float_as_uint(S.ca[3 * i]) == __float_as_uint(n1) && __float_as_uint(S.ca[3 * i + 1]) == __float_as_uint(n2)) {
            out = S.ca[3 * i + 2];
            return true;
        }
    }
    return false;
}

// the reference's model AABB test: division, signbit corner choice, fmaxf/fminf
__device__ __forceinline__ bool model_gate(const float* c, V3 o, V3 d) {
    float tmin = 0.0f, tmax = __int_as_float(0x7f800000);
    const float oo[3] = {o.x, o.y, o.z};
    const float dd[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        int s = signbit(dd[i]) ? 1 : 0;
        float bmin = c[s * 3 + i];
        float bmax = c[(1 - s) * 3 + i];
        float dmin = (bmin - oo[i]) / dd[i];
        float dmax = (bmax - oo[i]) / dd[i];
        tmin = fmaxf(dmin, tmin);
        tmax = fminf(dmax, tmax);
    }
    return tmin <= tmax;
}

__device__ __forceinline__ int hit_model_raw(const DevScene& S, int tri) {
    return __float_as_int(__ldg(&S.tri[5 * (size_t)tri + 2].w));
}

struct Hit {
    float t;
    int tri;
    V3 uvw;
};

// edge-function test with precomputed terms on a leaf-ordered triangle record
// (T[3].w its triangle index, q2.w its model); returns false when the triangle
// belongs to a model below min_model or cannot be a better (t, index)
// candidate than (best_t, best_tri).  The record's index and model come with
// the 16-byte loads the test makes anyway, the model only once the plane test
// has passed.
__device__ __forceinline__ bool tri_test(const float4* __restrict__ T, V3 o, V3 d, float best_t, int best_tri,
                                         int min_model, float& t_out, V3& uvw, int& tri_out, int& m_out) {
    const float4 q0 = __ldg(T), q4 = __ldg(T + 3);
    const int tri = __float_as_int(q4.w);
    V3 n = xyz(q4);
    float ndd = vdot(n, d);
    if (fabsf(ndd) < 1e-6f) return false;
    float t = (q0.w - vdot(n, o)) / ndd;
    if (t < 0) return false;
    if (t > best_t || (t == best_t && tri > best_tri)) return false;
    const float4 q1 = __ldg(T + 1), q2 = __ldg(T + 2);
    const int m = __float_as_int(q2.w);
    if (m < min_model) return false;
    V3 v0 = xyz(q0);
    V3 P = vadd(o, vscale(d, t));
    float w = vdot(n, vcross(xyz(q1), vsub(P, v0)));
    if (w < 0) return false;
    float v = vdot(n, vcross(vsub(v0, xyz(q2)), vsub(P, xyz(q2))));
    if (v < 0) return false;
    w = w * q1.w;
    v = v * q1.w;
    float u = 1.f - v - w;
    if (u < 0) return false;
    t_out = t;
    uvw = v3(u, v, w);
    tri_out = tri;
    m_out = m;
    return true;
}

__device__ __forceinline__ float safe_inv(float x) { return 1.0f / (x == 0.0f ? 1e-30f : x); }

// BVH traversal state of one ray.  A query is one or two passes (see
// intersect below); each pass returns the smallest (t, triangle) with t > 0
// among the triangles of models >= min_model whose model gate passes.  The
// first pass (min_model == 0) also records the largest model index with a
// gated hit at exactly t == 0 (zmodel, -1 if none), its lowest such triangle
// and that triangle's barycentrics; the second pass keeps that record and
// ignores hits at t == 0 (every one of them belongs to a model <= zmodel).
//
// Traversal is while-while with postponed leaves (Aila & Laine, "Understanding
// the efficiency of ray traversal on GPUs", HPG 2009): lanes descend interior
// nodes until every lane of the warp holds a leaf, then test triangles
// together.  Each interior node carries both children's boxes.  The state is
// resumable: trav_step runs one descend + leaf round, so a caller can stop a
// warp's traversal between rounds and give finished lanes new rays.
constexpr int TRAV_SENTINEL = 0x76543210;
constexpr int TRAV_STACK = 64;
constexpr int TRAV_NONE = 0x7fffffff;

// Traversal stacks.  LocalStack: the whole stack in per-thread local memory.
// SplitStack: entries [0, H) in a shared-memory column of the block (entry i of
// thread t at column[i * STRIDE], so the 32 lanes of a warp always use 32
// different banks whatever their depths) and the deeper entries in local
// memory.  Lanes of a warp sit at different depths, so a local-memory stack
// touches a different 128-byte line per lane; the shared column does not.
struct LocalStack {
    int a[TRAV_STACK];
    __device__ __forceinline__ int get(int i) const { return a[i]; }
    __device__ __forceinline__ void set(int i, int v) { a[i] = v; }
};
template <int H, int STRIDE>
struct SplitStack {
    int* col;                    // this thread's column of the block's shared stack
    int deep[TRAV_STACK - H];
    __device__ __forceinline__ int get(int i) const { return i < H ? col[i * STRIDE] : deep[i - H]; }
    __device__ __forceinline__ void set(int i, int v) {
        if (i < H) col[i * STRIDE] = v;
        else deep[i - H] = v;
    }
};

struct Trav {
    float ix, iy, iz, ox, oy, oz;      // slab terms: 1/d and o/d
    float best_t;
    int best_tri;
    V3 best_uvw;
    int zmodel, ztri;
    V3 zuvw;
    unsigned long long gate_known, gate_pass;
    int node, leaf, sp, min_model;
};

template <class Stk>
__device__ __forceinline__ void trav_pass(Trav& T, int min_model, Stk& stack) {
    T.best_t = __int_as_float(0x7f800000);
    T.best_tri = TRAV_NONE;
    T.best_uvw = v3(0.f, 0.f, 0.f);
    T.min_model = min_model;
    T.node = 0;
    T.leaf = 0;
    T.sp = 0;
    stack.set(0, TRAV_SENTINEL);
}

template <class Stk>
__device__ __forceinline__ void trav_init(Trav& T, V3 o, V3 d, Stk& stack) {
    T.ix = safe_inv(d.x); T.iy = safe_inv(d.y); T.iz = safe_inv(d.z);
    T.ox = o.x * T.ix; T.oy = o.y * T.iy; T.oz = o.z * T.iz;
    T.zmodel = -1;
    T.ztri = TRAV_NONE;
    T.zuvw = v3(0.f, 0.f, 0.f);
    T.gate_known = 0ull;
    T.gate_pass = 0ull;
    trav_pass(T, 0, stack);
}

// Work counters of a traversal (the tracer's work-counting launch): interior
// nodes visited (each visit tests both children's boxes) and triangle tests.
// NoWork compiles to nothing.
struct NoWork {
    __device__ __forceinline__ void node() {}
    __device__ __forceinline__ void tris(int) {}
};
struct Work {
    unsigned nodes = 0, tri_tests = 0;
    __device__ __forceinline__ void node() { nodes++; }
    __device__ __forceinline__ void tris(int c) { tri_tests += (unsigned)c; }
};

// One round: descend until this lane holds a leaf (or every active lane does,
// or, CUT > 0, no more than CUT lanes still descend), then test the held
// leaves.  Returns true when the pass is complete; a lane stopped before its
// leaf keeps its place (node, stack) for the next round.
template <int CUT = 0, class Stk, class W = NoWork>
__device__ __forceinline__ bool trav_step(const DevScene& S, Trav& T, V3 o, V3 d, Stk& stack, W&& work = W()) {
    int node = T.node, leaf = T.leaf, sp = T.sp;
    // Box slabs as fused multiply-adds: the boxes are padded far beyond the
    // rounding of either form, so culling stays conservative and the answer
    // (decided by the exact triangle tests) is the same; the fused form is
    // half the instructions of the node test.
    const float ix = T.ix, iy = T.iy, iz = T.iz, nox = -T.ox, noy = -T.oy, noz = -T.oz;
    while ((unsigned)node < (unsigned)TRAV_SENTINEL) {
        work.node();
        const float4* N = S.nodes + 4 * (size_t)node;
        const float4 a0 = __ldg(N), b0 = __ldg(N + 1), a1 = __ldg(N + 2), b1 = __ldg(N + 3);
        const float best_t = T.best_t;
        float t0x = __fmaf_rn(a0.x, ix, nox), t1x = __fmaf_rn(b0.x, ix, nox);
        float t0y = __fmaf_rn(a0.y, iy, noy), t1y = __fmaf_rn(b0.y, iy, noy);
        float t0z = __fmaf_rn(a0.z, iz, noz), t1z = __fmaf_rn(b0.z, iz, noz);
        const float c0min = fmax3(fminf(t0x, t1x), fminf(t0y, t1y), fmaxf(fminf(t0z, t1z), 0.0f));
        const float c0max = fmin3(fmaxf(t0x, t1x), fmaxf(t0y, t1y), fminf(fmaxf(t0z, t1z), best_t));
        t0x = __fmaf_rn(a1.x, ix, nox); t1x = __fmaf_rn(b1.x, ix, nox);
        t0y = __fmaf_rn(a1.y, iy, noy); t1y = __fmaf_rn(b1.y, iy, noy);
        t0z = __fmaf_rn(a1.z, iz, noz); t1z = __fmaf_rn(b1.z, iz, noz);
        const float c1min = fmax3(fminf(t0x, t1x), fminf(t0y, t1y), fmaxf(fminf(t0z, t1z), 0.0f));
        const float c1max = fmin3(fmaxf(t0x, t1x), fmaxf(t0y, t1y), fminf(fmaxf(t0z, t1z), best_t));
        const bool h0 = c0min <= c0max, h1 = c1min <= c1max;
        if (!h0 && !h1) {
            node = stack.get(sp--);
        } else {
            const int r0 = __float_as_int(a0.w), r1 = __float_as_int(a1.w);
            node = h0 ? r0 : r1;
            if (h0 && h1) {
                int other = r1;
                if (c1min < c0min) { node = r1; other = r0; }
                if (sp < TRAV_STACK - 1) stack.set(++sp, other);
            }
        }
        if (node < 0 && leaf >= 0) {   // first leaf: postpone it, keep descending
            leaf = node;
            node = stack.get(sp--);
        }
        if (!__any_sync(__activemask(), leaf >= 0)) break;   // every lane holds a leaf
        if (CUT > 0 && __popc(__activemask()) <= CUT) break;
    }
    while (leaf < 0) {
        const int packed = ~leaf;
        const int first = packed >> 8, count = packed & 255;
        work.tris(count);
        for (int i = 0; i < count; i++) {
            const float4* Q = S.tri_leaf + 4 * (size_t)(first + i);
            float t; V3 uvw; int tri, m;
            if (!tri_test(Q, o, d, T.best_t, T.best_tri, T.min_model, t, uvw, tri, m)) continue;
            const bool zero = t == 0.0f;
            if (zero && (T.min_model != 0 || m < T.zmodel || (m == T.zmodel && tri > T.ztri))) continue;
            bool pass;
            if (m < 64) {
                const unsigned long long bit = 1ull << m;
                if (!(T.gate_known & bit)) {
                    T.gate_known |= bit;
                    if (model_gate(S.maabb + 6 * m, o, d)) T.gate_pass |= bit;
                }
                pass = (T.gate_pass & bit) != 0ull;
            } else {
                pass = model_gate(S.maabb + 6 * m, o, d);
            }
            if (!pass) continue;
            if (zero) { T.zmodel = m; T.ztri = tri; T.zuvw = uvw; }
            else { T.best_t = t; T.best_tri = tri; T.best_uvw = uvw; }
        }
        leaf = node;                    // another postponed leaf: process it as well
        if (node < 0) node = stack.get(sp--);
    }
    T.node = node; T.leaf = leaf; T.sp = sp;
    return node == TRAV_SENTINEL;
}

// After a completed pass, apply the reference's model-loop semantics
// (PhotonTracing.cu:187-198, Raytracer.cuh:73-84): a running "intersection"
// that starts at 0 means "no hit yet", so a model whose nearest hit is at
// exactly t = 0 is taken only when no later model is hit at all.  With z the
// last model hit at t = 0, the answer is the nearest (t, triangle) hit among
// models after z, else z's hit.  Returns TRAV_AGAIN after starting the second
// pass (models > z), TRAV_HIT with h filled, or TRAV_MISS.
enum { TRAV_HIT = 0, TRAV_MISS = 1, TRAV_AGAIN = 2 };
template <class Stk>
__device__ __forceinline__ int trav_resolve(const DevScene& S, Trav& T, Hit& h, Stk& stack) {
    if (T.best_tri != TRAV_NONE &&
        (T.min_model != 0 || T.zmodel < 0 || hit_model_raw(S, T.best_tri) > T.zmodel)) {
        h.t = T.best_t; h.tri = T.best_tri; h.uvw = T.best_uvw;
        return TRAV_HIT;
    }
    if (T.zmodel < 0) return TRAV_MISS;
    if (T.min_model == 0) {
        trav_pass(T, T.zmodel + 1, stack);
        return TRAV_AGAIN;
    }
    h.t = 0.0f; h.tri = T.ztri; h.uvw = T.zuvw;
    return TRAV_HIT;
}

// Closest hit of one ray, both passes run to completion.
static __device__ __noinline__ bool intersect(const DevScene& S, V3 o, V3 d, Hit& h) {
    LocalStack stack;
    Trav T;
    trav_init(T, o, d, stack);
    while (true) {
        while (!trav_step(S, T, o, d, stack)) {}
        const int r = trav_resolve(S, T, h, stack);
        if (r != TRAV_AGAIN) return r == TRAV_HIT;
    }
}

// interpolated vertex normal, reciprocal-normalised (Model.cuh:436-443)
__device__ __forceinline__ V3 shading_normal(const DevScene& S, const Hit& h) {
    const float* n = S.tri_nrm + 9 * (size_t)h.tri;
    V3 n0 = vscale(ld3(n), h.uvw.x), n1 = vscale(ld3(n + 3), h.uvw.y), n2 = vscale(ld3(n + 6), h.uvw.z);
    return vnorm_recip(vadd(vadd(n0, n1), n2));
}
__device__ __forceinline__ int hit_model(const DevScene& S, int tri) {
    return __float_as_int(__ldg(&S.tri[5 * (size_t)tri + 2].w));
}

// ----------------------------------------------------------- ray helpers --
struct Ray { V3 o, d; };

__device__ __forceinline__ Ray ray_reflect(const Ray& r, V3 from, V3 n) {   // Ray.cuh:64-71
    float dnd = vdot(r.d, n);
    V3 refl = vsub(r.d, vscale(vscale(n, 2.f), dnd));
    Ray o;
    o.d = vnorm_div(refl);
    o.o = vadd(from, vscale(n, 0.01f));
    return o;
}
__device__ __forceinline__ bool ray_refract(const Ray& r, V3 from, V3 n, float r1, float r2, Ray& out) {   // Ray.cuh:85-96
    float eta = r1 / r2;
    float c1 = -vdot(r.d, n);
    float w = eta * c1;
    float c2m = (w - eta) * (w + eta);
    if (c2m < -1.f) return false;
    out.d = vadd(vscale(r.d, eta), vscale(n, w - sqrtf(1.f + c2m)));
    out.o = vadd(from, vscale(vneg(n), 0.01f));
    return true;
}

}  // namespace pm
