// ref_driver.cu -- host-side harness around the reference's own render code.
//
// TEST INFRASTRUCTURE ONLY (used by tests/golden/make_golden.py and by
// bench.py's reference / cpu_baseline leg).  Compiled by oracle/Makefile from
// the reference sources where they lie (-I <reference>/CudaPhotonMapping), as
// a single translation unit with oracle/ref_host/shim.h pre-included.  Nothing
// here re-implements reference behaviour: every entry point builds the
// reference's own objects (Model, Camera, Ray, PhotonGrid, PhotonMaxHeap,
// Raytracer, RaytracePlanner, MediumManager) on the host and calls their
// __host__ __device__ methods, i.e. the reference's CPU mode
// (CPM/Raytracer.cuh:281-299).
//
// Two things the reference does through the GPU are done directly here:
//  * global parameters: the cpu_* globals that GlobalParams::set_* and the
//    set_*_parameters helpers would write (CPM/GlobalParams.cu) are assigned
//    directly, because those helpers also call cudaMemcpyToSymbol;
//  * per-pixel medium storage is zeroed before every pixel (the reference's
//    GPU path cudaMemsets it once, CPM/RaytracePlanner.cu:261,269; its CPU path
//    leaves it uninitialised and shares it across pixels).  This pins the
//    otherwise undefined reads of CPM/MediumManager.cuh:319,324 to zeros.
// Members the harness assigns directly are private in the reference: the
// explicitly private ones are read as public; the class-default private
// members of PhotonGrid are reached through pointers to members formed in
// explicit instantiations (access checking does not apply there).
#define private public
#define protected public
#include "Raytracer.cuh"
#include "PhotonGrid.cu"
#include "PhotonMaxHeap.cu"
#include "GlobalParams.cu"
#include "MediumContent.cu"
#include "MMInnerStack.cu"
#include "RayPlan.cu"
#include "MathFunctions.cu"
#include "ModelConstructInfo.cu"
#include "ObjLoader.cpp"
#undef private
#undef protected

#include <cstdint>

namespace {
template <typename Tag, typename Tag::type M> struct Reach { friend typename Tag::type member(Tag) { return M; } };
#define PM_REACH(NAME, CLS, TYPE, FIELD) \
    struct NAME { typedef TYPE CLS::*type; friend type member(NAME); }; \
    template struct Reach<NAME, &CLS::FIELD>;
PM_REACH(G_pos, PhotonGrid, cpm::vec3*, p_positions)
PM_REACH(G_dir, PhotonGrid, cpm::vec3*, p_directions)
PM_REACH(G_pow, PhotonGrid, cpm::vec3*, p_powers)
PM_REACH(G_num, PhotonGrid, int, num_photons)
PM_REACH(G_aabb, PhotonGrid, AABB, scene_aabb)
PM_REACH(G_size, PhotonGrid, GridSize3D, grid_size)
PM_REACH(G_cell, PhotonGrid, float, cell_size)
PM_REACH(G_starts, PhotonGrid, uint*, cell_starts)
PM_REACH(G_sizes, PhotonGrid, uint*, cell_sizes)
struct G_sizing { typedef void (PhotonGrid::*type)(int); friend type member(G_sizing); };
template struct Reach<G_sizing, &PhotonGrid::compute_grid_and_cell_size>;
}  // namespace

// the reference's check_cuda lives in CudaUtils.cu, whose static CudaSynchronizer
// would create a CUDA context at load time; the harness never calls CUDA.
void check_cuda(cudaError_t result, char const* const func, const char* const file, int const line) {
    if (result) fprintf(stderr, "cuda error %d at %s:%d %s\n", (int)result, file, line, func);
}

#include "ref_scene.h"
using ref_host::HostScene;
using ref_host::V;

extern "C" {

// Models from a triangle soup sorted by model: mats = 12 floats per model
// (diffuse3, specular3, emission3, ior, opaque, shininess).  Model ids are the
// model indices, as CPM/Initializer.cu:11-16 assigns them.
void* ref_scene_create(int ntri, const float* pos, const float* nrm, const int* tri_model,
                       int nmodel, const float* mats, int light_model, const float* light_intensity) {
    return ref_host::make_scene(ntri, pos, nrm, tri_model, nmodel, mats, light_model, light_intensity);
}
void ref_scene_destroy(void* h) { delete (HostScene*)h; }

// Camera(position, direction, up, fov, W, H) -> pos3 fwd3 right3 up3 vw vh focal
void ref_camera(const float* position, const float* direction, const float* upv, float fov, int W, int H, float* out) {
    Camera c(V(position), V(direction), V(upv), fov, W, H);
    const cpm::vec3* v[4] = {&c.position, &c.forward, &c.right, &c.up};
    for (int i = 0; i < 4; i++) { out[3 * i] = v[i]->x; out[3 * i + 1] = v[i]->y; out[3 * i + 2] = v[i]->z; }
    out[12] = c.viewport_width; out[13] = c.viewport_height; out[14] = c.focal_length;
}

// normalised eye-ray directions for pixels (xs[i], ys[i])
void ref_camera_rays(const float* position, const float* direction, const float* upv, float fov, int W, int H,
                     int n, const int* xs, const int* ys, float* out_dir) {
    Camera c(V(position), V(direction), V(upv), fov, W, H);
    for (int i = 0; i < n; i++) {
        cpm::Ray r(c.position, c.generate_ray_direction(xs[i], ys[i]));
        out_dir[3 * i] = r.direction.x; out_dir[3 * i + 1] = r.direction.y; out_dir[3 * i + 2] = r.direction.z;
    }
}

// Raytracer::find_intersection over the models (CPM/Raytracer.cuh:66-93), reverse_normal = false
void ref_intersect(void* h, int n, const float* orig, const float* dir, float* out_point, int* out_model, float* out_n) {
    HostScene* s = (HostScene*)h;
    Raytracer rt;
    rt.scene.models = s->models.data();
    rt.scene.models_number = (int)s->models.size();
    for (int i = 0; i < n; i++) {
        cpm::Ray r;
        r.origin = V(orig + 3 * i); r.direction = V(dir + 3 * i);
        Model* m = nullptr; cpm::vec3 nn, p;
        bool ok = rt.find_intersection(r, false, m, nn, p);
        out_model[i] = ok ? m->get_id() : -1;
        out_point[3 * i] = p.x; out_point[3 * i + 1] = p.y; out_point[3 * i + 2] = p.z;
        out_n[3 * i] = nn.x; out_n[3 * i + 1] = nn.y; out_n[3 * i + 2] = nn.z;
    }
}

// Ray::reflect and Ray::refract (CPM/Ray.cuh:64-96): out = origin3 dir3 ok
void ref_ray_ops(int n, const float* dir, const float* from, const float* nrm, const float* etas,
                 float* out_reflect, float* out_refract, int* out_ok) {
    for (int i = 0; i < n; i++) {
        cpm::Ray r; r.direction = V(dir + 3 * i);
        cpm::Ray a = r.reflect(V(from + 3 * i), V(nrm + 3 * i));
        cpm::Ray b;
        out_ok[i] = r.refract(V(from + 3 * i), V(nrm + 3 * i), etas[2 * i], etas[2 * i + 1], b);
        float* o = out_reflect + 6 * i;
        o[0] = a.origin.x; o[1] = a.origin.y; o[2] = a.origin.z; o[3] = a.direction.x; o[4] = a.direction.y; o[5] = a.direction.z;
        o = out_refract + 6 * i;
        o[0] = b.origin.x; o[1] = b.origin.y; o[2] = b.origin.z; o[3] = b.direction.x; o[4] = b.direction.y; o[5] = b.direction.z;
    }
}

// Raytracer::HDR followed by clamp_min(1) (CPM/Raytracer.cuh:95-107, 238-239)
void ref_hdr(int n, const float* rgb, float* out) {
    Raytracer rt;
    for (int i = 0; i < n; i++) {
        cpm::vec3 c = rt.HDR(V(rgb + 3 * i));
        c.clamp_min(1.f);
        out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
    }
}

namespace {
struct HostGrid {
    std::vector<cpm::vec3> p, d, w;
    std::vector<uint32_t> starts, sizes;
    PhotonGrid g;
};
static void fill_grid(HostGrid& hg, int nph, const float* aabb, const int* dims, float cell,
                      const uint32_t* starts, const uint32_t* sizes, const float* spos, const float* sdir,
                      const float* spow) {
    hg.p.resize(nph > 0 ? nph : 1); hg.d.resize(nph > 0 ? nph : 1); hg.w.resize(nph > 0 ? nph : 1);
    for (int i = 0; i < nph; i++) { hg.p[i] = V(spos + 3 * i); hg.d[i] = V(sdir + 3 * i); hg.w[i] = V(spow + 3 * i); }
    size_t cells = (size_t)dims[0] * dims[1] * dims[2];
    hg.starts.assign(starts, starts + cells);
    hg.sizes.assign(sizes, sizes + cells);
    hg.g.*member(G_pos()) = hg.p.data(); hg.g.*member(G_dir()) = hg.d.data(); hg.g.*member(G_pow()) = hg.w.data();
    hg.g.*member(G_num()) = nph;
    for (int i = 0; i < 6; i++) (hg.g.*member(G_aabb())).corners[i] = aabb[i];
    hg.g.*member(G_size()) = GridSize3D{dims[0], dims[1], dims[2]};
    hg.g.*member(G_cell()) = cell;
    hg.g.*member(G_starts()) = hg.starts.data();
    hg.g.*member(G_sizes()) = hg.sizes.data();
}
// An empty one-cell grid: find_nearests on it finds nothing (stands for "no caustic map").
static void empty_grid(HostGrid& hg, const float* aabb) {
    static const uint32_t zero = 0;
    const int dims[3] = {1, 1, 1};
    float big = 1e6f;
    fill_grid(hg, 0, aabb, dims, big, &zero, &zero, nullptr, nullptr, nullptr);
}
static void set_globals(int max_depth, float def_ior, int k_global, int k_caustic) {
    GlobalParams::cpu_max_depth = max_depth;
    GlobalParams::cpu_default_refractive_index = def_ior;
    GlobalParams::cpu_global_photon_num = k_global;
    GlobalParams::cpu_caustic_photon_num = k_caustic;
}
}  // namespace

// PhotonGrid::find_nearests with PhotonMaxHeap (CPM/PhotonGrid.cu:257-284):
// out_slots / out_dist: k per query in heap array order, out_cnt: heap size,
// out_full: the return value, out_rad: Raytracer::get_color_from_photon_grid.
void ref_gather(int nph, const float* aabb, const int* dims, float cell, const uint32_t* starts,
                const uint32_t* sizes, const float* spos, const float* sdir, const float* spow,
                int nq, const float* qpos, const float* qnrm, float r, int k,
                uint32_t* out_slots, float* out_dist, int* out_cnt, int* out_full, float* out_rad) {
    HostGrid hg;
    fill_grid(hg, nph, aabb, dims, cell, starts, sizes, spos, sdir, spow);
    std::vector<PhotonMaxHeapItem> heap(k > 0 ? k : 1);
    cpu_photon_heap_data = heap.data();
    cpu_photon_heap_capacity = k;
    PhotonMaxHeap mh;
    Raytracer rt;
    for (int i = 0; i < nq; i++) {
        bool full = hg.g.find_nearests(V(qpos + 3 * i), r, k, mh, 0, 1);
        out_full[i] = full;
        out_cnt[i] = (int)mh.get_size();
        for (int j = 0; j < k; j++) {
            out_slots[(size_t)i * k + j] = j < (int)mh.get_size() ? heap[j].idx : 0xffffffffu;
            out_dist[(size_t)i * k + j] = j < (int)mh.get_size() ? heap[j].distance : -1.f;
        }
        cpm::vec3 c = rt.get_color_from_photon_grid(heap.data(), mh.get_size(), hg.d.data(), hg.w.data(),
                                                    V(qnrm + 3 * i), 0, 1);
        out_rad[3 * i] = c.x; out_rad[3 * i + 1] = c.y; out_rad[3 * i + 2] = c.z;
    }
}

// The reference's grid sizing for n photons in the scene box aabb (min xyz,
// max xyz): PhotonGrid(n, aabb) + compute_grid_and_cell_size(desired)
// (CPM/PhotonGrid.cu:41-56), the per-cell counts of analyze_density's kernel
// taken on the host with the reference's hash_position (:10-38, :76-90), and
// analyze_density's re-grid rule (:112-116): a cell above 5 x desired means
// compute_grid_and_cell_size(desired / 5).  out_dims / out_cell: the final
// grid; out_max: the largest cell count of the first grid; returns 1 when the
// re-grid happened.
int ref_grid_sizing(int n, const float* pos, const float* aabb, int desired, int* out_dims, float* out_cell,
                    uint32_t* out_max) {
    AABB box;
    for (int i = 0; i < 6; i++) box.corners[i] = aabb[i];
    PhotonGrid g(n, box);
    (g.*member(G_sizing()))(desired);
    const GridSize3D gs = g.*member(G_size());
    const float cell = g.*member(G_cell());
    std::vector<uint32_t> counts((size_t)gs.x * gs.y * gs.z, 0);
    const cpm::vec3 mn(aabb[0], aabb[1], aabb[2]);
    for (int i = 0; i < n; i++) counts[hash_position(mn, V(pos + 3 * (size_t)i), gs, cell)]++;
    uint32_t mx = 0;
    for (uint32_t c : counts) mx = std::max(mx, c);
    *out_max = mx;
    int regrid = 0;
    if (mx > 5 * desired) {
        (g.*member(G_sizing()))(desired / 5);
        regrid = 1;
    }
    const GridSize3D f = g.*member(G_size());
    out_dims[0] = f.x; out_dims[1] = f.y; out_dims[2] = f.z;
    *out_cell = g.*member(G_cell());
    return regrid;
}

// The reference's CPU mode over pixel rows [y0, y1): per pixel, Camera ray +
// Raytracer::render_trace (tone-mapped, clamped) and the uchar3 conversion of
// CPM/Raytracer.cuh:288-292.  c_dims == null: no caustic map (an empty grid).
void ref_render(void* h, const float* position, const float* direction, const float* upv, float fov, int W, int H,
                int y0, int y1, int nph, const float* aabb, const int* dims, float cell, const uint32_t* starts,
                const uint32_t* sizes, const float* spos, const float* sdir, const float* spow,
                int nph_c, const int* c_dims, float c_cell, const uint32_t* c_starts, const uint32_t* c_sizes,
                const float* c_spos, const float* c_sdir, const float* c_spow,
                int max_depth, float def_ior, int k_global, int k_caustic, float* out_ldr, uint8_t* out_rgb8) {
    HostScene* s = (HostScene*)h;
    s->camera = Camera(V(position), V(direction), V(upv), fov, W, H);
    HostGrid gg, cg;
    fill_grid(gg, nph, aabb, dims, cell, starts, sizes, spos, sdir, spow);
    if (c_dims) fill_grid(cg, nph_c, aabb, c_dims, c_cell, c_starts, c_sizes, c_spos, c_sdir, c_spow);
    else empty_grid(cg, aabb);
    set_globals(max_depth, def_ior, k_global, k_caustic);

    int D = max_depth, DC = (max_depth + 1) / 2;
    int kmax = std::max(k_global, k_caustic);
    std::vector<PhotonMaxHeapItem> heap(kmax > 0 ? kmax : 1);
    cpu_photon_heap_data = heap.data(); cpu_photon_heap_capacity = kmax;
    std::vector<MMInnerData> inner((size_t)(D + 2) * DC);
    std::vector<MMInnerContainer> outer(D + 2);
    std::vector<RayPlan> plans(D);
    cpu_mm_inner_data = inner.data(); cpu_mm_inner_capacity = DC;
    cpu_mm_outer_data = outer.data(); cpu_mm_outer_capacity = D;
    cpu_raytrace_planner_data = plans.data(); cpu_raytrace_planner_capacity = D;
    MediumManager mm;
    cpm::rayplan_stack planner;
    PhotonMaxHeap heaps[1];

    Raytracer rt;
    rt.scene = Scene(s->models.data(), (int)s->models.size(), &s->light, 1, s->camera);
    rt.ray_planner.array_size = 1;
    rt.ray_planner.medium_managers = &mm;
    rt.ray_planner.planner = &planner;
    rt.heaps = heaps;
    rt.diffuse_grid = gg.g;
    rt.specular_grid = cg.g;

    size_t o = 0;
    for (int j = y0; j < y1; j++) {
        for (int i = 0; i < W; i++, o++) {
            std::memset((void*)inner.data(), 0, sizeof(MMInnerData) * inner.size());
            for (auto& c : outer) c.set_size(0);
            mm = MediumManager();
            planner.set_size(0);
            cpm::vec3 dir = rt.scene.camera.generate_ray_direction(i, j);
            cpm::Ray ray(rt.scene.camera.position, dir);
            cpm::vec3 c = rt.render_trace(ray, false, 0);
            if (out_ldr) { out_ldr[3 * o] = c.x; out_ldr[3 * o + 1] = c.y; out_ldr[3 * o + 2] = c.z; }
            if (out_rgb8) {
                uchar3 u = make_uchar3(c.x * 255, c.y * 255, c.z * 255);
                out_rgb8[3 * o] = u.x; out_rgb8[3 * o + 1] = u.y; out_rgb8[3 * o + 2] = u.z;
            }
        }
    }
}

// The reference's OBJ loader (CPM/ObjLoader.cpp loadOBJ) on dir/file, its
// ModelConstructInfo list flattened: per model the type (0 triangle, 1 quad,
// 2 polygon), vertex count, material (diffuse, specular, emission, index,
// opaque, shininess) and name; all models' vertex positions and normals
// concatenated.  Null when the loader throws.
struct RefObj {
    std::vector<ModelConstructInfo> models;
    std::vector<std::string> names;
};

void* ref_obj_load(const char* dir, const char* file, int* out_models, int* out_vertices) {
    try {
        auto r = loadOBJ(dir, file);
        RefObj* o = new RefObj();
        o->models = std::move(r.first);
        o->names = std::move(r.second);
        int nv = 0;
        for (auto& m : o->models) nv += m.size;
        *out_models = (int)o->models.size();
        *out_vertices = nv;
        return o;
    } catch (...) {
        return nullptr;
    }
}

void ref_obj_model(void* h, int m, int* type, int* size, float* mat12, char* name, int name_len) {
    const RefObj* o = (const RefObj*)h;
    const ModelConstructInfo& mi = o->models[m];
    *type = (int)mi.type;
    *size = mi.size;
    const Material& t = mi.material;
    const float v[12] = {t.diffuse.x, t.diffuse.y, t.diffuse.z, t.specular.x, t.specular.y, t.specular.z,
                         t.emission.x, t.emission.y, t.emission.z, t.refr_index, t.opaque, t.shininess};
    std::memcpy(mat12, v, sizeof v);
    std::snprintf(name, (size_t)name_len, "%s", o->names[m].c_str());
}

void ref_obj_vertices(void* h, float* pos, float* nrm) {
    const RefObj* o = (const RefObj*)h;
    size_t k = 0;
    for (auto& m : o->models)
        for (int i = 0; i < m.size; i++, k++) {
            pos[3 * k] = m.positions[i].x; pos[3 * k + 1] = m.positions[i].y; pos[3 * k + 2] = m.positions[i].z;
            nrm[3 * k] = m.normals[i].x; nrm[3 * k + 1] = m.normals[i].y; nrm[3 * k + 2] = m.normals[i].z;
        }
}

void ref_obj_free(void* h) {
    RefObj* o = (RefObj*)h;
    for (auto& m : o->models) { free(m.positions); free(m.texcoords); free(m.normals); }
    delete o;
}

}  // extern "C"
