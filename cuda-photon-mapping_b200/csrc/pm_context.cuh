// pm_context.cuh -- the library context (opaque pm_ctx of the C ABI) and the
// host helpers the entry points share.  Internal: not part of the ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/pm_api.h"
#include "pm_gather.cuh"
#include "pm_mlp.cuh"
#include "pm_scene.cuh"

namespace pm {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct MapState {
    int64_t n = 0;                       // photons in the list
    DevBuf pos, dir, pow;                // traced-order list (3 floats per photon)
    DevBuf rec;                          // a traced list's (position, direction) records, 32 B per photon
    bool has_rec = false;                // rec holds the current list
    bool uniform_pow = false;            // every photon of the list has power pow_value (a traced map)
    bool lists_pending = false;          // dir / pow lists not written yet (a traced map: rec and pow_value
                                         // hold them; written by the first pm_get_photons / pm_save_photons)
    bool spow_pending = false;           // the grid's sorted power not written yet (uniform: pow_value)
    float pow_value[3] = {0, 0, 0};
    bool built = false;
    int dims[3] = {0, 0, 0};
    float cell = 0.f;
    int64_t cells = 0;
    float aabb[6] = {0, 0, 0, 0, 0, 0};
    int S = 1;
    DevBuf starts, sizes, gpos, gdir, gpow, key_counts, key_starts;
    DevBuf cid, keys0, keys1, vals0, vals1, hist, scan_ws, small, counts2;
};

}  // namespace pm

struct pm_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    // pinned host words the small per-call device reads land in (a read into
    // pageable memory is staged by the driver): [0] status, [2..3] photon
    // totals, [4..5] grid count maxima, [6..7] request count
    uint32_t* hbuf = nullptr;
    std::string err;
    int sm_count = 148;
    int trace_refill = 0;      // k_trace refill threshold; 0: the kernel's default
    // scene
    bool has_scene = false;
    int ntri = 0, nmodel = 0, light_model = 0, light_first = 0, light_count = 0, nca = 0;
    float light_intensity[3] = {1, 1, 1};
    float default_ior = 1.f;
    float aabb[6] = {0, 0, 0, 0, 0, 0};
    bool has_tri_diffuse = false;
    pm::DevBuf tri, tri_pos, tri_nrm, tri_diffuse, nodes, prim, maabb, mats, ca;
    pm::MapState maps[2];
    // photon-pass scratch
    pm::DevBuf counter, stage, cnt_g, cnt_c, scan_g, scan_c, totals, trace_ws, scratch_pow;
    // the tracer's work-counting launch (pm_trace_work): rays, node visits, triangle tests
    pm::DevBuf work;
    bool count_work = false;
    // render scratch
    pm::DevBuf req_a, req_b, req_c, req_counter, px_base, px_count, est_g, est_c;
    pm::DevBuf status, gws;
    // learned radiance cache
    bool has_cache = false;
    pm::DevBuf cache_w32, cache_w16, cache_m, cache_v, cache_grad, cache_loss;
    // BVH: builder for the next pm_set_scene; the current scene's builder, size, build time
    int bvh_builder = 0, scene_bvh_builder = 0;
    int64_t bvh_nodes = 0;
    float bvh_ms = 0.f;
    pm::DevBuf bvh_scratch, tri_leaf;
    // host copies for the eye pass's block order: 6 AABB floats and 12 material floats per model
    std::vector<float> h_maabb, h_mats;
    pm::DevBuf eye_order;
    pm::DevBuf rq_keys, rq_k0, rq_k1, rq_v0, rq_v1, rq_hist, rq_ws;   // the gather's request order
    // training steps queued without a loss run on their own stream; whatever
    // reads or writes the cache (or synchronises the context) waits for them
    cudaStream_t train_st = nullptr;
    cudaEvent_t train_fork = nullptr, train_done = nullptr;
    bool train_pending = false;
    // bumped by every call that rebuilds or re-initialises what a captured
    // learned graph reads (scene, photon lists, grids, cache): a graph made
    // before such a call refuses to run
    uint64_t generation = 0;
    // pm_frame's eye pass runs on its own stream beside the photon pass, its
    // request ordering beside the grid build
    cudaStream_t frame_st = nullptr;
    cudaEvent_t frame_fork = nullptr, frame_done = nullptr;
    bool eye_order_valid = false;   // eye_order holds the order for eye_order_cam on this scene
    pm_camera eye_order_cam = {};
    std::vector<int> h_eye_order;   // host copy of eye_order
    pm::DevBuf eye_band;            // the blocks of a row band (pm_render_rows), in eye_order's order
    pm::DevBuf est_mlp, est_fb, probe_pos, probe_nrm, probe_req, probe_est, tile_flag, learned_counts, fallback_list;
    pm_cache_opts cache_opts = {};
    float cache_lo[3] = {0, 0, 0}, cache_inv[3] = {1, 1, 1};
    int cache_step = 0;
    cudaEvent_t ev[14] = {};
    float stage_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t launches = 0;      // kernels this context has launched
    int64_t last_requests = 0; // gather requests of the last pm_render
    int64_t last_pixels = 0;
    // photons per traced path seen by the last pm_trace_photons on this scene
    // (sizes the next call's first batch; the output never depends on it)
    double yield_g = 0.0, yield_c = 0.0;
    int yield_bounces = 0;
};

namespace pm {

int fail(pm_ctx* c, int code, const std::string& msg);
int cuda_fail(pm_ctx* c, cudaError_t e, const char* what);
// grow-only device buffer (1/8 headroom on growth)
cudaError_t ensure(DevBuf& b, size_t bytes);
void release(DevBuf& b);
// every device buffer the context owns; a hash of the addresses and sizes of
// some buffers (changes whenever one of them is allocated, grown or released)
std::vector<DevBuf*> all_buffers(pm_ctx* ctx);
uint64_t buffer_fingerprint(const std::vector<DevBuf*>& bufs);
template <class T> T* P(DevBuf& b) { return (T*)b.p; }
DevScene dev_scene(pm_ctx* c);
// reads and clears the device status word; PM_ERR_TIMEOUT / PM_ERR_OVERFLOW
int check_status(pm_ctx* ctx, const char* what);
float elapsed(cudaEvent_t a, cudaEvent_t b);
// gather view of map m, estimates read from est_src's direction / power arrays
GatherGrid grid_of(MapState& m, MapState& est_src);
// order the context's stream after the training steps still queued on the training stream
int cache_fence(pm_ctx* ctx);
// the radiance cache's network as the kernels read it
MlpNet cache_net(pm_ctx* ctx);
// a frame's checks: scene, grid, camera size, depth and k ranges
int render_checks(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o);
// Launch order of the eye pass's pixel blocks (eye_blocks entries): first the
// blocks that overlap the screen rectangle of a specular or refractive model
// (their pixels spawn chains of reflected / refracted rays, the longest jobs
// of the pass), then the others, each part in image order.  Returns the
// number of blocks put first.
int64_t eye_block_order(const pm_ctx* ctx, const pm_camera* cam, std::vector<int>& order);
// the learned render's option checks (PM_OK or the failure recorded on ctx)
int learned_checks(pm_ctx* ctx, const pm_learned_opts* lo);

}  // namespace pm

#define CK(expr)                                                        \
    do {                                                                \
        cudaError_t e_ = (expr);                                        \
        if (e_ != cudaSuccess) return pm::cuda_fail(ctx, e_, #expr);        \
    } while (0)

// Grow-only device buffer; a grown buffer gets 1/8 headroom so sizes that
// wobble from call to call (batch sizes follow measured yields) do not
// re-allocate every time.

#define ENSURE(buf, bytes) CK(ensure(buf, bytes))
