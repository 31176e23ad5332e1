// pm_bvh.cpp -- host BVH builder for the closest-hit queries of pm_scene.cuh.
//
// The reference has no acceleration structure: every ray tests every triangle
// of every model whose box it meets (CudaPhotonMapping/Model.cuh:366-446); its
// kd-tree code only reduces a model's triangles to one AABB
// (KdTree.cu:395-464).  This is a binary BVH built with binned SAH (32 bins on
// each centroid axis; a range of <= 4 triangles becomes a leaf when testing
// them costs no more than the best split; depth <= 60), stored as
// interior nodes that carry both children's boxes, so one 64-byte fetch tests
// both children.  Boxes are padded so that culling is conservative with
// respect to the exact triangle test; the traversal (pm_scene.cuh) keeps the
// reference's answer.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace pm {

namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float* p) {
        for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    float area() const {
        if (lo[0] > hi[0]) return 0.f;
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node {
    Box box;
    int first = 0;
    int count = 0;
};

struct Task { int node, b, e, depth; };

constexpr int BINS = 32;        // SAH bins per axis
constexpr int LEAF_MAX = 4;     // larger ranges are always split
constexpr float SAH_CT = 1.0f;  // cost of an interior visit (one 64-byte node, two slab tests) ...
constexpr float SAH_CI = 1.2f;  // ... and of one triangle test (one 64-byte leaf-ordered record)

}  // namespace

// nodes_out: 16 floats per interior node (both children's boxes and refs, see below);
// node 0 is the root.  prim: leaf triangle indices.
void build_bvh(const float* tri_pos, int ntri, float pad, std::vector<float>& nodes_out, std::vector<int>& prim) {
    std::vector<Box> pb(ntri);
    std::vector<float> cen(3 * (size_t)ntri);
    for (int t = 0; t < ntri; t++) {
        for (int v = 0; v < 3; v++) pb[t].grow(tri_pos + 9 * (size_t)t + 3 * v);
        for (int a = 0; a < 3; a++) cen[3 * (size_t)t + a] = 0.5f * (pb[t].lo[a] + pb[t].hi[a]);
    }
    prim.resize(ntri);
    for (int t = 0; t < ntri; t++) prim[t] = t;
    std::vector<Node> nodes(1);
    std::vector<Task> stack;
    stack.push_back(Task{0, 0, ntri, 0});
    while (!stack.empty()) {
        Task tk = stack.back();
        stack.pop_back();
        Box nb, cb;
        for (int i = tk.b; i < tk.e; i++) { nb.grow(pb[prim[i]]); cb.grow(&cen[3 * (size_t)prim[i]]); }
        nodes[tk.node].box = nb;
        const int n = tk.e - tk.b;
        auto make_leaf = [&]() { nodes[tk.node].first = tk.b; nodes[tk.node].count = n; };
        if (n <= 1 || (tk.depth >= 60 && n <= 255)) { make_leaf(); continue; }
        // binned SAH over all three axes; cost = CT + CI (A_l n_l + A_r n_r) / A
        float ext[3];
        for (int a = 0; a < 3; a++) ext[a] = cb.hi[a] - cb.lo[a];
        float best = FLT_MAX;
        int baxis = -1, bsplit = -1;
        for (int axis = 0; axis < 3; axis++) {
            if (!(ext[axis] > 0.f)) continue;
            Box bb[BINS];
            int bc[BINS] = {0};
            for (int i = tk.b; i < tk.e; i++) {
                const int t = prim[i];
                int k = (int)((cen[3 * (size_t)t + axis] - cb.lo[axis]) / ext[axis] * BINS);
                k = std::min(std::max(k, 0), BINS - 1);
                bc[k]++;
                bb[k].grow(pb[t]);
            }
            Box left[BINS];
            int lc[BINS];
            Box acc; int ac = 0;
            for (int k = 0; k < BINS; k++) { acc.grow(bb[k]); ac += bc[k]; left[k] = acc; lc[k] = ac; }
            Box racc; int rc = 0;
            for (int k = BINS - 1; k > 0; k--) {
                racc.grow(bb[k]); rc += bc[k];
                if (lc[k - 1] == 0 || rc == 0) continue;
                float c = left[k - 1].area() * lc[k - 1] + racc.area() * rc;
                if (c < best) { best = c; baxis = axis; bsplit = k; }
            }
        }
        const float A = nb.area();
        const float split_cost = A > 0.f && baxis >= 0 ? SAH_CT + SAH_CI * best / A : FLT_MAX;
        if (n <= LEAF_MAX && SAH_CI * (float)n <= split_cost) { make_leaf(); continue; }
        int mid;
        if (baxis < 0) {
            // all centroids coincide: keep order, split by count
            mid = tk.b + n / 2;
        } else {
            const int axis = baxis;
            auto bin_of = [&](int t) {
                int k = (int)((cen[3 * (size_t)t + axis] - cb.lo[axis]) / ext[axis] * BINS);
                return std::min(std::max(k, 0), BINS - 1);
            };
            int* it = std::partition(prim.data() + tk.b, prim.data() + tk.e, [&](int t) { return bin_of(t) < bsplit; });
            mid = (int)(it - prim.data());
            if (mid == tk.b || mid == tk.e) {
                mid = tk.b + n / 2;
                std::nth_element(prim.data() + tk.b, prim.data() + mid, prim.data() + tk.e, [&](int x, int y) {
                    return cen[3 * (size_t)x + axis] < cen[3 * (size_t)y + axis];
                });
            }
        }
        int left_idx = (int)nodes.size();
        nodes.resize(nodes.size() + 2);
        nodes[tk.node].first = left_idx;
        nodes[tk.node].count = 0;
        stack.push_back(Task{left_idx + 1, mid, tk.e, tk.depth + 1});
        stack.push_back(Task{left_idx, tk.b, mid, tk.depth + 1});
    }
    // Output: interior nodes only, each holding both children's padded boxes
    // (16 floats = 4 x float4): (lo0, ref0), (hi0, 0), (lo1, ref1), (hi1, 0).
    // ref >= 0: interior node index; ref < 0: leaf, ~ref = first << 8 | count.
    std::vector<int> remap(nodes.size(), -1);
    int ninterior = 0;
    for (size_t i = 0; i < nodes.size(); i++)
        if (nodes[i].count == 0) remap[i] = ninterior++;
    auto ref_of = [&](size_t c) -> int {
        if (nodes[c].count == 0) return remap[c];
        return ~((nodes[c].first << 8) | nodes[c].count);
    };
    auto put_box = [&](float* o, const Box& b, int ref) {
        for (int a = 0; a < 3; a++) {
            float span = std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a]));
            float p = pad + span * 1e-5f;
            o[a] = b.lo[a] - p;
            o[4 + a] = b.hi[a] + p;
        }
        std::memcpy(&o[3], &ref, 4);
        o[7] = 0.f;
    };
    if (ninterior == 0) {
        // a single leaf: one interior node holding it and an empty box
        nodes_out.assign(16, 0.f);
        put_box(&nodes_out[0], nodes[0].box, ref_of(0));
        Box empty;
        for (int a = 0; a < 3; a++) { nodes_out[8 + a] = 3.0e38f; nodes_out[12 + a] = -3.0e38f; }
        int r = ~0;
        std::memcpy(&nodes_out[11], &r, 4);
        (void)empty;
        return;
    }
    nodes_out.assign(16 * (size_t)ninterior, 0.f);
    for (size_t i = 0; i < nodes.size(); i++) {
        if (nodes[i].count != 0) continue;
        float* o = &nodes_out[16 * (size_t)remap[i]];
        size_t c0 = nodes[i].first, c1 = c0 + 1;
        put_box(o, nodes[c0].box, ref_of(c0));
        put_box(o + 8, nodes[c1].box, ref_of(c1));
    }
}

}  // namespace pm
