// ref_trace.cu -- host harness that runs the reference's own photon tracer.
//
// TEST INFRASTRUCTURE ONLY (tests/test_oracle_pins.py).  It pins the oracle's
// restatement of the photon pass (oracle/pm_oracle.cpp trace_path) to the
// reference's code: CPM/PhotonTracing.cu is compiled from the reference
// sources where they lie, as host code (oracle/ref_host/trace_shim.h says
// how), and driven one photon path at a time.  Every decision of a path is
// taken by the reference's own functions:
//   light point    Model::gpu_get_random_point_with_normal   CPM/Model.cuh:202-243
//   bounce         trace                                     CPM/PhotonTracing.cu:278-326
//                  find_intersection                         :178-213 (Model::intersection, AABB)
//                  destiny / refract_destity / FresnelSchlick :215-276
//                  get_refraction_pair / get_update_refraction_pair :127-176
//                  photon_trace_stack                        CPM/PhotonTraceStack.cuh:40-116
//                  critical angles: compute_critical_angles  :79-125 (CAHashMap, CPM/HashMap.cuh)
//                  Ray::reflect / refract / reflect_spherical CPM/Ray.cuh:16-96
//                  PathOperator                              CPM/PathOperator.cuh
//                  PhotonArray::add                          CPM/PhotonArray.cuh:31-42
// The random draws come from the injected per-path stream (oracle/philox.h)
// through the reference's own curand_uniform call sites.
//
// What the harness itself states is the new-path branch and the bounce loop of
// the `emit` kernel (CPM/PhotonTracing.cu:344-373): a __global__ body cannot be
// called on the host, and its loop only ends when both photon arrays fill,
// which the host build of PhotonArray::add never reports (it writes without
// counting, CPM/PhotonArray.cuh:33-37).  The statements below follow those
// lines one for one, with two defined behaviours the reference leaves open:
//   * a miss ends the path (trace returns no value on a miss, :291-293): the
//     harness asks the reference's find_intersection first and stops there;
//   * a path is one stream: draws restart at each path's own stream, where
//     the reference shares one curand state across a thread's paths (:350).
// The bounce limit is the reference's PHOTON_BOUNCE_NUM (10, :20), also the
// medium stack's depth (:397-398).
//
// The same driver also runs on the GPU (ref_gpu_trace_paths): there the
// reference's functions are its device build, whose vec3 arithmetic rounds
// toward zero (CPM/vec3.cuh:18-20) and whose other float expressions nvcc
// compiles with its default contractions -- the reference's GPU numerics,
// one photon path per thread with the same injected streams.
//
// The reference is compiled in both of nvcc's passes; the kernels below run
// it on the device, the host functions after them drive it on the host.
#include "PhotonTracing.cuh"
#include "RefractiveTable.cuh"
#include "GlobalParams.cuh"
#include "PhotonArray.cuh"
#include "PhotonTraceStack.cuh"
#include "Array.cuh"
#include "PathOperator.cuh"
#include "HashMap.cuh"
#include "Pair.cuh"
#include "Timer.cuh"
#include "CudaUtils.cuh"
// CPM/PhotonTracing.cu:107 is MSVC's `for each (auto kv in ca_table)`; the
// two words are used nowhere else in the file outside comments and strings.
#define each
#define in :
#include "PhotonTracing.cu"
#undef in
#undef each
#include "PhotonTraceStack.cu"
#include "GlobalParams.cu"
#include "Pair.cu"
#include "MediumContent.cu"
#include "MMInnerStack.cu"
#include "RayPlan.cu"
#include "CudaRandom.cu"

#include <new>
#include "../philox.h"

// ------------------------------------------------ the reference on the GPU --
// Each thread's injected path stream (curand_uniform reads it in the device pass).
__device__ oracle_rng::Stream* pm_ref_dev_streams;
#ifdef __CUDA_ARCH__
__device__ float pm_ref_dev_uniform() { return pm_ref_dev_streams[threadIdx.x + blockIdx.x * blockDim.x].next(); }
#endif

// The values the reference's host code gives its device globals through
// cudaMemcpyToSymbol (set_pt_stack_parameters, GlobalParams, trace_photons:406).
__global__ void ref_gpu_setup(MMInnerData* stack_data, idxtype stack_capacity, float default_ior,
                              cudaRandomStateT* states, oracle_rng::Stream* streams) {
    gpu_pt_stack_data = stack_data;
    gpu_pt_stack_capacity = stack_capacity;
    GlobalParams::gpu_default_refractive_index = default_ior;
    curand_states = states;
    pm_ref_dev_streams = streams;
}

// One photon path per thread: path p0 + thread, the statements of the emit
// kernel's new-path branch and bounce loop (CPM/PhotonTracing.cu:345-373) as
// the host driver below states them, the photons of each trace() call caught
// in the thread's two one-photon arrays.  Records: [thread][k] of 3 floats for
// position and direction, k < PHOTON_BOUNCE_NUM.
__global__ void ref_gpu_trace(SubScene scene, LightSource ls, CAHashMap critical_angles,
                              PathOperator* path_operators, cpm::photon_trace_stack* trace_stacks,
                              cudaRandomStateT* gen_states, cpm::PhotonArray* arrays, cpm::Photon* slots,
                              idxtype threads_num, float power_cap, uint64_t seed, uint32_t tag, int64_t p0,
                              int* counts, int* draws, float* g_rec, float* c_rec, int* g_bounce, int* c_bounce) {
    const idxtype threadId = threadIdx.x + blockIdx.x * blockDim.x;
    if (threadId >= threads_num) return;
    oracle_rng::Stream& st = pm_ref_dev_streams[threadId];
    st = oracle_rng::Stream(seed, (uint64_t)(p0 + (int64_t)threadId), tag);
    counts[2 * threadId] = 0;
    counts[2 * threadId + 1] = 0;
    int cur_bounce_num = 0;
    path_operators[threadId].clear();
    trace_stacks[threadId].set_size(0);
    cudaRandomStateT local_state = gen_states[threadId];
    auto rand_point_on_light_source = ls.model_owner->gpu_get_random_point_with_normal(local_state);
    cpm::Ray ray;
    ray.origin = rand_point_on_light_source.first + rand_point_on_light_source.second * 0.0001f;
    float prob;
    float dot;
    int tries = 0;
    do {
        if (++tries > (1 << 16)) { draws[threadId] = -1; return; }
        ray.direction.x = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.y = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.z = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.normalize();
        prob = curand_uniform(&local_state);
        dot = cpm::vec3::dot(ray.direction, rand_point_on_light_source.second);
        if (dot < 0) {
            dot = -dot;
            ray.direction *= -1;
        }
    } while (prob > dot);
    gen_states[threadId] = local_state;
    cpm::vec3 pp = ls.intensity / power_cap;
    cpm::PhotonArray* spec = arrays + 2 * (size_t)threadId;
    cpm::PhotonArray* diff = spec + 1;
    cpm::Photon* slot_c = slots + 2 * (size_t)threadId;
    cpm::Photon* slot_g = slot_c + 1;
    int ng = 0, nc = 0;
    bool generate_new_ray = false;
    while (!generate_new_ray) {
        {
            cpm::vec3 n, p, sp, df;
            int id;
            float ior, opaque;
            if (!find_intersection(scene, ray, n, p, id, ior, opaque, sp, df)) break;
        }
        new (spec) cpm::PhotonArray(slot_c, 0, 1);
        new (diff) cpm::PhotonArray(slot_g, 0, 1);
        generate_new_ray = trace(scene, ray, pp, spec, diff, path_operators, critical_angles, threads_num,
                                 trace_stacks);
        const size_t r = (size_t)threadId * PHOTON_BOUNCE_NUM;
        if (spec->get_size() > 0) {
            float* o = c_rec + 6 * (r + nc);
            o[0] = slot_c->pos.x; o[1] = slot_c->pos.y; o[2] = slot_c->pos.z;
            o[3] = slot_c->inc_dir.x; o[4] = slot_c->inc_dir.y; o[5] = slot_c->inc_dir.z;
            c_bounce[r + nc] = cur_bounce_num;
            nc++;
        }
        if (diff->get_size() > 0) {
            float* o = g_rec + 6 * (r + ng);
            o[0] = slot_g->pos.x; o[1] = slot_g->pos.y; o[2] = slot_g->pos.z;
            o[3] = slot_g->inc_dir.x; o[4] = slot_g->inc_dir.y; o[5] = slot_g->inc_dir.z;
            g_bounce[r + ng] = cur_bounce_num;
            ng++;
        }
        cur_bounce_num++;
        generate_new_ray = generate_new_ray || (cur_bounce_num > PHOTON_BOUNCE_NUM - 1);
    }
    counts[2 * threadId] = ng;
    counts[2 * threadId + 1] = nc;
    draws[threadId] = (int)st.n;
}

#ifndef __CUDA_ARCH__
#include <omp.h>
#include <cstring>
#include <vector>
#include "ref_scene.h"

// the CUDA runtime itself, for the GPU driver (the shim maps these names to
// host stand-ins for the reference's own host code above)
#undef cudaMalloc
#undef cudaFree
#undef cudaMemcpy
#undef cudaGetLastError
static cudaError_t real_malloc(void** p, size_t bytes) { return cudaMalloc(p, bytes); }
static cudaError_t real_memset(void* p, int v, size_t bytes) { return cudaMemset(p, v, bytes); }
static cudaError_t real_memcpy(void* d, const void* s, size_t b, cudaMemcpyKind k) { return cudaMemcpy(d, s, b, k); }
static cudaError_t real_free(void* p) { return cudaFree(p); }
static cudaError_t real_last_error() { return cudaGetLastError(); }
static cudaError_t real_sync() { return cudaDeviceSynchronize(); }

thread_local uint3 pm_ref_thread_idx;
thread_local uint3 pm_ref_block_idx;
thread_local dim3 pm_ref_block_dim;
static thread_local oracle_rng::Stream* pm_ref_stream = nullptr;

float pm_ref_uniform() { return pm_ref_stream->next(); }

// Defined in CPM/CudaUtils.cu, whose static CudaSynchronizer would create a
// CUDA context at load time; the harness never launches anything.
void check_cuda(cudaError_t result, char const* const func, const char* const file, int const line) {
    if (result) fprintf(stderr, "cuda error %d at %s:%d %s\n", (int)result, file, line, func);
}
int calculate_max_blocks_number(int, void*) { return 1; }

namespace {

struct Rec { cpm::vec3 pos, power, dir; int bounce; };

// a photon slot of a one-photon PhotonArray, marked unwritten
static const uint32_t kUnwritten = 0x7fc0dead;
static void mark(cpm::Photon& p) { std::memcpy(&p.pos.x, &kUnwritten, 4); }
static bool written(const cpm::Photon& p) { return std::memcmp(&p.pos.x, &kUnwritten, 4) != 0; }

// One photon path (CPM/PhotonTracing.cu:345-373).  Returns the uniforms drawn,
// or -1 when the light's direction loop did not accept within 2^16 tries.
static int trace_one(const SubScene& scene, const LightSource& ls, CAHashMap critical_angles,
                     PathOperator* path_operators, cpm::photon_trace_stack* trace_stacks,
                     cudaRandomStateT* gen_states, idxtype threads_num, idxtype threadId, float power_cap,
                     uint64_t seed, uint32_t tag, int64_t path, std::vector<Rec>& gl, std::vector<Rec>& cau) {
    oracle_rng::Stream st(seed, (uint64_t)path, tag);
    pm_ref_stream = &st;
    // :346-369, the new-path branch
    int cur_bounce_num = 0;
    path_operators[threadId].clear();
    trace_stacks[threadId].set_size(0);
    cudaRandomStateT local_state = gen_states[threadId];
    auto rand_point_on_light_source = ls.model_owner->gpu_get_random_point_with_normal(local_state);
    cpm::Ray ray;
    ray.origin = rand_point_on_light_source.first + rand_point_on_light_source.second * 0.0001f;
    float prob;
    float dot;
    int tries = 0;
    do {
        if (++tries > (1 << 16)) return -1;
        ray.direction.x = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.y = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.z = fmap_to_range(curand_uniform(&local_state), -1.f, 1.f);
        ray.direction.normalize();
        prob = curand_uniform(&local_state);
        dot = cpm::vec3::dot(ray.direction, rand_point_on_light_source.second);
        if (dot < 0) {
            dot = -dot;
            ray.direction *= -1;
        }
    } while (prob > dot);
    gen_states[threadId] = local_state;
    cpm::vec3 pp = ls.intensity / power_cap;

    // :371-373, the bounce loop; one-photon arrays show whether trace stored
    cpm::Photon slot_c, slot_g;
    bool generate_new_ray = false;
    while (!generate_new_ray) {
        {
            cpm::vec3 n, p, spec, diff;
            int id;
            float ior, opaque;
            if (!find_intersection(scene, ray, n, p, id, ior, opaque, spec, diff)) break;
        }
        mark(slot_c); mark(slot_g);
        cpm::PhotonArray specular_photons(&slot_c, 0, 1), diffuse_photons(&slot_g, 0, 1);
        generate_new_ray = trace(scene, ray, pp, &specular_photons, &diffuse_photons, path_operators,
                                 critical_angles, threads_num, trace_stacks);
        if (written(slot_c)) cau.push_back(Rec{slot_c.pos, slot_c.power, slot_c.inc_dir, cur_bounce_num});
        if (written(slot_g)) gl.push_back(Rec{slot_g.pos, slot_g.power, slot_g.inc_dir, cur_bounce_num});
        cur_bounce_num++;
        generate_new_ray = generate_new_ray || (cur_bounce_num > PHOTON_BOUNCE_NUM - 1);
    }
    pm_ref_stream = nullptr;
    return (int)st.n;
}

static void put3(float* o, const cpm::vec3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

}  // namespace

extern "C" {

void* ref_trace_scene_create(int ntri, const float* pos, const float* nrm, const int* tri_model, int nmodel,
                             const float* mats, int light_model, const float* light_intensity) {
    return ref_host::make_scene(ntri, pos, nrm, tri_model, nmodel, mats, light_model, light_intensity);
}
void ref_trace_scene_destroy(void* h) { delete (ref_host::HostScene*)h; }

// The reference's critical-angle table for the scene (compute_critical_angles,
// CPM/PhotonTracing.cu:79-125): out = (n1, n2, cos) triples of the occupied
// hash slots in slot order.  Returns their number.
int ref_trace_critical_angles(void* h, float default_ior, float* out, int cap) {
    ref_host::HostScene* s = (ref_host::HostScene*)h;
    GlobalParams::cpu_default_refractive_index = default_ior;
    Scene scene(s->models.data(), (int)s->models.size(), &s->light, 1, s->camera);
    CAHashMap* table = compute_critical_angles(scene);
    int n = 0;
    for (idxtype i = 0; i < CAHashMap::kHashTableCapacity; i++) {
        const CAHashMap::KeyValue& kv = table->data[i];
        if (kv.key_packed == CAHashMap::kEmptyPacked) continue;
        if (n < cap) {
            uint32_t a = (uint32_t)(kv.key_packed >> 32), b = (uint32_t)kv.key_packed;
            std::memcpy(out + 3 * n, &a, 4); std::memcpy(out + 3 * n + 1, &b, 4);
            out[3 * n + 2] = kv.value;
        }
        n++;
    }
    std::free(table->data);
    std::free(table);
    return n;
}

// Photon paths [p0, p1) through the reference's tracer, nthreads host threads
// each acting as one reference thread.  Photon power = intensity / power_cap.
// counts[2*(p-p0)+{0,1}] = photons of the path in the global / caustic list,
// draws[p-p0] = uniforms the path consumed (-1: light direction loop gave up).
// Photons are written in path order, bounce order within a path; the g_* and
// c_* arrays hold (p1-p0) * 10 entries.
void ref_trace_paths(void* h, float default_ior, uint64_t seed, uint32_t tag, int64_t power_cap, int64_t p0,
                     int64_t p1, int nthreads, int* counts, int* draws, float* g_pos, float* g_pow, float* g_dir,
                     int* g_bounce, float* c_pos, float* c_pow, float* c_dir, int* c_bounce, int64_t* out_ng,
                     int64_t* out_nc) {
    ref_host::HostScene* s = (ref_host::HostScene*)h;
    GlobalParams::cpu_default_refractive_index = default_ior;
    Scene full(s->models.data(), (int)s->models.size(), &s->light, 1, s->camera);
    CAHashMap* table = compute_critical_angles(full);
    CAHashMap critical_angles;
    std::memcpy(&critical_angles, table, sizeof(CAHashMap));
    SubScene scene(full);
    const LightSource ls = s->light;

    if (nthreads < 1) nthreads = 1;
    const idxtype threads_num = (idxtype)nthreads;
    std::vector<PathOperator> path_operators(threads_num);
    std::vector<cpm::photon_trace_stack> trace_stacks(threads_num);
    std::vector<MMInnerData> stack_data((size_t)threads_num * PHOTON_BOUNCE_NUM);
    set_pt_stack_parameters(stack_data.data(), stack_data.data(), PHOTON_BOUNCE_NUM);
    std::vector<cudaRandomStateT> states(threads_num);
    std::memset((void*)states.data(), 0, sizeof(cudaRandomStateT) * threads_num);
    curand_states = states.data();

    const int64_t n = p1 - p0;
    std::vector<std::vector<Rec>> gl(n), cau(n);
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num();
        pm_ref_thread_idx = make_uint3((unsigned)t, 0, 0);
        pm_ref_block_idx = make_uint3(0, 0, 0);
        pm_ref_block_dim = dim3((unsigned)nthreads, 1, 1);
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < n; i++)
            draws[i] = trace_one(scene, ls, critical_angles, path_operators.data(), trace_stacks.data(),
                                 states.data(), threads_num, (idxtype)t, (float)power_cap, seed, tag, p0 + i,
                                 gl[i], cau[i]);
    }
    int64_t ng = 0, nc = 0;
    for (int64_t i = 0; i < n; i++) {
        counts[2 * i] = (int)gl[i].size();
        counts[2 * i + 1] = (int)cau[i].size();
        for (auto& r : gl[i]) {
            put3(g_pos + 3 * ng, r.pos); put3(g_pow + 3 * ng, r.power); put3(g_dir + 3 * ng, r.dir);
            g_bounce[ng++] = r.bounce;
        }
        for (auto& r : cau[i]) {
            put3(c_pos + 3 * nc, r.pos); put3(c_pow + 3 * nc, r.power); put3(c_dir + 3 * nc, r.dir);
            c_bounce[nc++] = r.bounce;
        }
    }
    *out_ng = ng;
    *out_nc = nc;
    curand_states = nullptr;
    std::free(table->data);
    std::free(table);
}

// The same path range on the GPU through the reference's device build (see
// ref_gpu_trace), one path per thread.  Outputs as ref_trace_paths without the
// powers.  Returns 0, or the CUDA error code of the first failing call (every
// buffer is released either way).
int ref_gpu_trace_paths(void* h, float default_ior, uint64_t seed, uint32_t tag, int64_t power_cap, int64_t p0,
                        int64_t p1, int* counts, int* draws, float* g_pos, float* g_dir, int* g_bounce, float* c_pos,
                        float* c_dir, int* c_bounce, int64_t* out_ng, int64_t* out_nc) {
    ref_host::HostScene* s = (ref_host::HostScene*)h;
    const int64_t n = p1 - p0;
    *out_ng = *out_nc = 0;
    if (n <= 0) return 0;
    const int M = (int)s->models.size();
    const int light = (int)(s->light.model_owner - s->models.data());
    std::vector<void*> owned;
    cudaError_t e = cudaSuccess;
    auto dalloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (e == cudaSuccess) e = real_malloc(&p, bytes ? bytes : 16);
        if (e == cudaSuccess) { owned.push_back(p); if (real_memset(p, 0, bytes ? bytes : 16) != cudaSuccess) e = cudaErrorUnknown; }
        return p;
    };
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = real_memcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    };
    // models with their vertex arrays on the device (CPM/Initializer.cu builds the same)
    std::vector<Model> dmodels(s->models);
    for (int m = 0; m < M && e == cudaSuccess; m++) {
        const size_t bytes = sizeof(cpm::vec3) * (size_t)s->models[m].mci.size;
        cpm::vec3* dp = (cpm::vec3*)dalloc(bytes);
        cpm::vec3* dn = (cpm::vec3*)dalloc(bytes);
        up(dp, s->pos[m], bytes);
        up(dn, s->nrm[m], bytes);
        dmodels[m].mci.positions = dp;
        dmodels[m].mci.normals = dn;
    }
    Model* d_models = (Model*)dalloc(sizeof(Model) * (size_t)M);
    up(d_models, dmodels.data(), sizeof(Model) * (size_t)M);
    LightSource dl = s->light;
    dl.model_owner = d_models + light;
    Scene dscene(d_models, M, nullptr, 0, s->camera);
    SubScene scene(dscene);
    // the critical-angle table, built by the reference's host code, copied as its trace_photons does
    GlobalParams::cpu_default_refractive_index = default_ior;
    Scene hscene(s->models.data(), M, &s->light, 1, s->camera);
    CAHashMap* table = compute_critical_angles(hscene);
    const size_t table_bytes = sizeof(CAHashMap::KeyValue) * CAHashMap::kHashTableCapacity;
    CAHashMap dca((CAHashMap::KeyValue*)dalloc(table_bytes));
    up(dca.data, table->data, table_bytes);
    std::free(table->data);
    std::free(table);
    // per-path state
    const idxtype T = (idxtype)n;
    MMInnerData* stack_data = (MMInnerData*)dalloc(sizeof(MMInnerData) * (size_t)T * PHOTON_BOUNCE_NUM);
    auto* stacks = (cpm::photon_trace_stack*)dalloc(sizeof(cpm::photon_trace_stack) * (size_t)T);
    auto* ops = (PathOperator*)dalloc(sizeof(PathOperator) * (size_t)T);
    auto* states = (cudaRandomStateT*)dalloc(sizeof(cudaRandomStateT) * (size_t)T);
    auto* streams = (oracle_rng::Stream*)dalloc(sizeof(oracle_rng::Stream) * (size_t)T);
    auto* arrays = (cpm::PhotonArray*)dalloc(sizeof(cpm::PhotonArray) * 2 * (size_t)T);
    auto* slots = (cpm::Photon*)dalloc(sizeof(cpm::Photon) * 2 * (size_t)T);
    int* d_counts = (int*)dalloc(sizeof(int) * 2 * (size_t)T);
    int* d_draws = (int*)dalloc(sizeof(int) * (size_t)T);
    const size_t R = (size_t)T * PHOTON_BOUNCE_NUM;
    float* d_g = (float*)dalloc(sizeof(float) * 6 * R);
    float* d_c = (float*)dalloc(sizeof(float) * 6 * R);
    int* d_gb = (int*)dalloc(sizeof(int) * R);
    int* d_cb = (int*)dalloc(sizeof(int) * R);
    if (e == cudaSuccess) {
        ref_gpu_setup<<<1, 1>>>(stack_data, PHOTON_BOUNCE_NUM, default_ior, states, streams);
        e = real_last_error();
    }
    if (e == cudaSuccess) {
        const unsigned threads = 128, blocks = (unsigned)((n + threads - 1) / threads);
        ref_gpu_trace<<<blocks, threads>>>(scene, dl, dca, ops, stacks, states, arrays, slots, T, (float)power_cap,
                                           seed, tag, p0, d_counts, d_draws, d_g, d_c, d_gb, d_cb);
        e = real_last_error();
    }
    if (e == cudaSuccess) e = real_sync();
    std::vector<int> hc(2 * (size_t)T), hgb(R), hcb(R);
    std::vector<float> hg(6 * R), hcr(6 * R);
    auto down = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess) e = real_memcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    };
    down(hc.data(), d_counts, hc.size() * 4);
    down(draws, d_draws, sizeof(int) * (size_t)T);
    down(hg.data(), d_g, hg.size() * 4);
    down(hcr.data(), d_c, hcr.size() * 4);
    down(hgb.data(), d_gb, hgb.size() * 4);
    down(hcb.data(), d_cb, hcb.size() * 4);
    for (void* p : owned) real_free(p);
    if (e != cudaSuccess) return (int)e;
    int64_t ng = 0, nc = 0;
    for (int64_t i = 0; i < n; i++) {
        counts[2 * i] = hc[2 * i];
        counts[2 * i + 1] = hc[2 * i + 1];
        for (int k = 0; k < hc[2 * i]; k++, ng++) {
            const float* r = &hg[6 * ((size_t)i * PHOTON_BOUNCE_NUM + k)];
            std::memcpy(g_pos + 3 * ng, r, 12); std::memcpy(g_dir + 3 * ng, r + 3, 12);
            g_bounce[ng] = hgb[(size_t)i * PHOTON_BOUNCE_NUM + k];
        }
        for (int k = 0; k < hc[2 * i + 1]; k++, nc++) {
            const float* r = &hcr[6 * ((size_t)i * PHOTON_BOUNCE_NUM + k)];
            std::memcpy(c_pos + 3 * nc, r, 12); std::memcpy(c_dir + 3 * nc, r + 3, 12);
            c_bounce[nc] = hcb[(size_t)i * PHOTON_BOUNCE_NUM + k];
        }
    }
    *out_ng = ng;
    *out_nc = nc;
    return 0;
}

}  // extern "C"
#endif  // !__CUDA_ARCH__
