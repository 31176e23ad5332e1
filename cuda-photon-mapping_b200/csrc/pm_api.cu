// pm_api.cu -- context, device memory and the C ABI of include/pm_api.h.
#include <algorithm>
#include <functional>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/pm_api.h"
#include "pm_device.cuh"
#include "pm_gather.cuh"
#include "pm_grid.cuh"
#include "pm_lbvh.cuh"
#include "pm_learned.cuh"
#include "pm_mlp.cuh"
#include "pm_render.cuh"
#include "pm_scan.cuh"
#include "pm_scene.cuh"
#include "pm_trace.cuh"

namespace pm {
void build_bvh(const float* tri_pos, int ntri, float pad, std::vector<float>& nodes_out, std::vector<int>& prim);
}

using namespace pm;

#include "pm_context.cuh"

namespace pm {

int fail(pm_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}
int cuda_fail(pm_ctx* c, cudaError_t e, const char* what) {
    return fail(c, e == cudaErrorMemoryAllocation ? PM_ERR_OOM : PM_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}
cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.p) bytes += bytes / 8;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e == cudaSuccess) b.bytes = bytes;
    else (void)cudaGetLastError();   // a failed allocation leaves no error behind for the next launch check
    return e;
}
void release(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}
std::vector<DevBuf*> all_buffers(pm_ctx* ctx) {
    std::vector<DevBuf*> v = {&ctx->tri, &ctx->tri_pos, &ctx->tri_nrm, &ctx->tri_diffuse, &ctx->nodes, &ctx->prim,
                              &ctx->maabb, &ctx->mats, &ctx->ca, &ctx->counter, &ctx->stage,
                              &ctx->cnt_g, &ctx->cnt_c, &ctx->scan_g, &ctx->scan_c, &ctx->totals, &ctx->trace_ws,
                              &ctx->scratch_pow, &ctx->req_a, &ctx->req_b, &ctx->req_c, &ctx->req_counter,
                              &ctx->px_base, &ctx->px_count, &ctx->est_g, &ctx->est_c, &ctx->status, &ctx->gws,
                              &ctx->cache_w32, &ctx->cache_w16, &ctx->cache_m, &ctx->cache_v, &ctx->cache_grad,
                              &ctx->cache_loss, &ctx->est_mlp, &ctx->est_fb, &ctx->probe_pos, &ctx->probe_nrm,
                              &ctx->probe_req, &ctx->probe_est, &ctx->tile_flag, &ctx->learned_counts,
                              &ctx->fallback_list, &ctx->bvh_scratch, &ctx->tri_leaf, &ctx->eye_order, &ctx->rq_keys,
                              &ctx->rq_k0, &ctx->rq_k1, &ctx->rq_v0, &ctx->rq_v1, &ctx->rq_hist, &ctx->rq_ws,
                              &ctx->work, &ctx->eye_band};
    for (auto& m : ctx->maps)
        for (DevBuf* b : {&m.pos, &m.dir, &m.pow, &m.starts, &m.sizes, &m.gpos, &m.gdir, &m.gpow, &m.cid, &m.keys0,
                          &m.keys1, &m.vals0, &m.vals1, &m.hist, &m.scan_ws, &m.small, &m.key_counts,
                          &m.key_starts, &m.counts2, &m.rec})
            v.push_back(b);
    return v;
}
uint64_t buffer_fingerprint(const std::vector<DevBuf*>& bufs) {
    uint64_t h = 1469598103934665603ull;   // FNV-1a over the buffers' addresses and sizes
    for (DevBuf* b : bufs)
        for (uint64_t w : {(uint64_t)(uintptr_t)b->p, (uint64_t)b->bytes})
            for (int i = 0; i < 8; i++) h = (h ^ ((w >> (8 * i)) & 0xff)) * 1099511628211ull;
    return h;
}


DevScene dev_scene(pm_ctx* c) {
    DevScene S;
    S.tri = P<float4>(c->tri);
    S.tri_pos = P<float>(c->tri_pos);
    S.tri_nrm = P<float>(c->tri_nrm);
    S.tri_diffuse = c->has_tri_diffuse ? P<float>(c->tri_diffuse) : nullptr;
    S.nodes = P<float4>(c->nodes);
    S.prim = P<int>(c->prim);
    S.tri_leaf = P<float4>(c->tri_leaf);
    S.maabb = P<float>(c->maabb);
    S.mats = P<float>(c->mats);
    S.ca = P<float>(c->ca);
    S.nca = c->nca;
    S.ntri = c->ntri;
    S.nmodel = c->nmodel;
    S.light_first = c->light_first;
    S.light_count = c->light_count;
    S.default_ior = c->default_ior;
    return S;
}

int check_status(pm_ctx* ctx, const char* what) {
    if (int rc = cache_fence(ctx)) return rc;
    CK(cudaMemcpyAsync(ctx->hbuf, ctx->status.p, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const uint32_t bits = ctx->hbuf[0];
    if (bits) {
        CK(cudaMemsetAsync(ctx->status.p, 0, 4, ctx->st));
        char buf[160];
        snprintf(buf, sizeof buf, "%s: device status 0x%x (1 timeout, 2 overflow, 4 stack, 8 bad input)", what, bits);
        return fail(ctx, (bits & ST_TIMEOUT) ? PM_ERR_TIMEOUT : PM_ERR_OVERFLOW, buf);
    }
    return PM_OK;
}

// critical-angle table as the reference builds it (PhotonTracing.cu:71-125)
void add_angle(std::vector<float>& t, float e1, float e2) {
    float eta = e2 / e1;
    if (!(eta < 1.f)) return;
    for (size_t i = 0; i < t.size(); i += 3) {
        uint32_t a, b, x, y;
        std::memcpy(&a, &t[i], 4); std::memcpy(&b, &t[i + 1], 4);
        std::memcpy(&x, &e1, 4); std::memcpy(&y, &e2, 4);
        if (a == x && b == y) return;
    }
    float ca = std::cos(std::asin(eta));
    t.push_back(e1); t.push_back(e2); t.push_back(ca);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return -1.f;
    return ms;
}

int valid_map(pm_ctx* ctx, int map) {
    if (map != PM_MAP_GLOBAL && map != PM_MAP_CAUSTIC) return fail(ctx, PM_ERR_INVALID, "map must be 0 (global) or 1 (caustic)");
    return PM_OK;
}

GatherGrid grid_of(MapState& m, MapState& est_src) {
    GatherGrid G;
    G.gpos = P<float4>(m.gpos);
    G.gdir = P<float>(est_src.gdir);
    G.gpow = P<float>(est_src.gpow);
    G.key_starts = P<uint32_t>(m.key_starts);
    G.mn[0] = m.aabb[0]; G.mn[1] = m.aabb[1]; G.mn[2] = m.aabb[2];
    G.gx = m.dims[0]; G.gy = m.dims[1]; G.gz = m.dims[2];
    G.cell = m.cell;
    G.S = m.S;
    G.guess = GATHER_GUESS;
    G.pow_uniform = est_src.uniform_pow;
    for (int c = 0; c < 3; c++) G.pw[c] = est_src.pow_value[c];
    return G;
}

int cache_fence(pm_ctx* ctx) {
    if (ctx->train_pending) {
        CK(cudaStreamWaitEvent(ctx->st, ctx->train_done, 0));
        ctx->train_pending = false;
    }
    return PM_OK;
}

MlpNet cache_net(pm_ctx* ctx) {
    MlpNet net;
    net.w = P<__nv_bfloat16>(ctx->cache_w16);
    for (int a = 0; a < 3; a++) { net.lo[a] = ctx->cache_lo[a]; net.inv[a] = ctx->cache_inv[a]; }
    net.out_scale = ctx->cache_opts.out_scale;
    net.freq0 = (float)(1 << ctx->cache_opts.octave0);
    return net;
}

int learned_checks(pm_ctx* ctx, const pm_learned_opts* lo) {
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    if (lo->tile < 1 || lo->tile > 256 || lo->probes < 1 || lo->probes > 64 || lo->max_rel_err != lo->max_rel_err ||
        !(lo->noise_z >= 0.f && lo->noise_z <= 100.f))
        return fail(ctx, PM_ERR_INVALID, "learned options: tile 1..256, probes 1..64, max_rel_err not NaN, noise_z 0..100");
    return PM_OK;
}

int render_checks(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o) {
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene");
    if (o->max_depth < 0 || o->max_depth > RENDER_MAX_DEPTH) return fail(ctx, PM_ERR_INVALID, "max_depth must be 0..5");
    if (o->k_global < 0 || o->k_global > 256 || o->k_caustic < 0 || o->k_caustic > 256)
        return fail(ctx, PM_ERR_INVALID, "k must be 0..256");
    if (cam->width <= 0 || cam->height <= 0) return fail(ctx, PM_ERR_INVALID, "bad camera size");
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    MapState& C = ctx->maps[PM_MAP_CAUSTIC];
    if (!G.built) return fail(ctx, PM_ERR_INVALID, "global map grid not built");
    if (C.built && o->faithful_caustic && C.n > G.n)
        return fail(ctx, PM_ERR_INVALID, "faithful caustic estimate reads the global map with caustic indices: "
                                         "the caustic map must not be larger than the global map");
    return PM_OK;
}

int64_t eye_block_order(const pm_ctx* ctx, const pm_camera* cam, std::vector<int>& order) {
    const int W = cam->width, H = cam->height;
    const int64_t npx = (int64_t)W * H, nb = eye_blocks(npx), T = eye_threads();
    // the kernel's camera: direction(u, v) = A + hor u + ver v, A = llc - pos
    double pos[3], hor[3], ver[3], A[3];
    for (int a = 0; a < 3; a++) {
        pos[a] = cam->position[a];
        hor[a] = (double)cam->right[a] * cam->viewport_w;
        ver[a] = (double)cam->up[a] * cam->viewport_h;
        A[a] = (pos[a] + cam->forward[a]) * cam->focal - 0.5 * hor[a] - 0.5 * ver[a] - pos[a];
    }
    auto cross = [](const double* x, const double* y, double* z) {
        z[0] = x[1] * y[2] - x[2] * y[1]; z[1] = x[2] * y[0] - x[0] * y[2]; z[2] = x[0] * y[1] - x[1] * y[0];
    };
    auto dot = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    double hv[3];
    cross(hor, ver, hv);
    struct Rect { int x0, x1, y0, y1; };
    std::vector<Rect> rects;
    const int M = (int)ctx->h_mats.size() / 12;
    for (int m = 0; m < M; m++) {
        const float* mt = &ctx->h_mats[12 * (size_t)m];
        const bool deep = mt[3] > 0.f || mt[4] > 0.f || mt[5] > 0.f || mt[10] < 1.f;
        if (!deep) continue;
        const float* bx = &ctx->h_maabb[6 * (size_t)m];
        if (bx[0] > bx[3]) continue;   // a model without triangles
        double u0 = 1e30, u1 = -1e30, v0 = 1e30, v1 = -1e30;
        bool whole = false;
        for (int c = 0; c < 8 && !whole; c++) {
            double D[3] = {(c & 1 ? bx[3] : bx[0]) - pos[0], (c & 2 ? bx[4] : bx[1]) - pos[1],
                           (c & 4 ? bx[5] : bx[2]) - pos[2]};
            // s D - u hor - v ver = A  (Cramer's rule)
            const double det = dot(D, hv);
            if (!(std::fabs(det) > 1e-12)) { whole = true; break; }
            const double sc = dot(A, hv) / det;
            double t[3];
            cross(A, ver, t);
            const double u = -dot(D, t) / det;   // det[D, A, -ver] / det
            cross(hor, A, t);
            const double v = -dot(D, t) / det;   // det[D, -hor, A] / det
            if (!(sc > 0.0)) { whole = true; break; }
            u0 = std::min(u0, u); u1 = std::max(u1, u); v0 = std::min(v0, v); v1 = std::max(v1, v);
        }
        if (whole) { order.resize((size_t)nb); for (int64_t b = 0; b < nb; b++) order[(size_t)b] = (int)b; return nb; }
        Rect r;
        r.x0 = (int)std::max(0.0, std::floor(u0 * W - 0.5) - 1.0);
        r.x1 = (int)std::min((double)W - 1, std::ceil(u1 * W - 0.5) + 1.0);
        r.y0 = (int)std::max(0.0, std::floor(v0 * H - 0.5) - 1.0);
        r.y1 = (int)std::min((double)H - 1, std::ceil(v1 * H - 0.5) + 1.0);
        if (r.x0 <= r.x1 && r.y0 <= r.y1) rects.push_back(r);
    }
    order.clear();
    order.reserve((size_t)nb);
    std::vector<int> rest;
    rest.reserve((size_t)nb);
    for (int64_t b = 0; b < nb; b++) {
        const int64_t p0 = b * T, p1 = std::min(p0 + T - 1, npx - 1);
        const int r0 = (int)(p0 / W), r1 = (int)(p1 / W);
        bool hot = false;
        for (const Rect& r : rects) {
            if (r1 < r.y0 || r0 > r.y1) continue;
            if (r0 != r1) { hot = true; break; }
            const int c0 = (int)(p0 % W), c1 = (int)(p1 % W);
            if (c1 >= r.x0 && c0 <= r.x1) { hot = true; break; }
        }
        (hot ? order : rest).push_back((int)b);
    }
    const int64_t first = (int64_t)order.size();
    order.insert(order.end(), rest.begin(), rest.end());
    return first;
}

}  // namespace pm

extern "C" {

int pm_create(pm_ctx** out, const pm_device_opts* opts) {
    if (!out) return PM_ERR_INVALID;
    *out = nullptr;
    pm_ctx* ctx = new pm_ctx();
    ctx->device = opts ? opts->device : 0;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) { delete ctx; return PM_ERR_CUDA; }
    e = cudaHostAlloc((void**)&ctx->hbuf, 64, cudaHostAllocDefault);
    if (e != cudaSuccess) { ctx->hbuf = nullptr; delete ctx; return PM_ERR_OOM; }
    std::memset(ctx->hbuf, 0, 64);
    if (opts && opts->stream) {
        ctx->st = (cudaStream_t)opts->stream;
    } else {
        e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete ctx; return PM_ERR_CUDA; }
        ctx->own_stream = true;
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    // tuning knob for the photon tracer's lane refill (1..32 lanes); the photons
    // traced do not depend on it
    if (const char* r = std::getenv("PM_TRACE_REFILL")) ctx->trace_refill = std::atoi(r);
    for (auto& ev : ctx->ev) {
        if (cudaEventCreate(&ev) != cudaSuccess) { pm_destroy(ctx); return PM_ERR_CUDA; }
    }
    if (ensure(ctx->status, 16) != cudaSuccess || cudaMemsetAsync(ctx->status.p, 0, 16, ctx->st) != cudaSuccess) {
        pm_destroy(ctx);
        return PM_ERR_OOM;
    }
    *out = ctx;
    return PM_OK;
}

void pm_destroy(pm_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    if (ctx->train_st) {
        cudaStreamSynchronize(ctx->train_st);
        cudaStreamDestroy(ctx->train_st);
    }
    if (ctx->frame_st) {
        cudaStreamSynchronize(ctx->frame_st);
        cudaStreamDestroy(ctx->frame_st);
    }
    if (ctx->frame_fork) cudaEventDestroy(ctx->frame_fork);
    if (ctx->hbuf) cudaFreeHost(ctx->hbuf);
    if (ctx->frame_done) cudaEventDestroy(ctx->frame_done);
    if (ctx->train_fork) cudaEventDestroy(ctx->train_fork);
    if (ctx->train_done) cudaEventDestroy(ctx->train_done);
    for (DevBuf* b : all_buffers(ctx)) release(*b);
    for (auto& ev : ctx->ev) if (ev) cudaEventDestroy(ev);
    if (ctx->own_stream && ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

const char* pm_last_error(const pm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pm_sync(pm_ctx* ctx) {
    if (!ctx) return PM_ERR_INVALID;
    if (int rc = cache_fence(ctx)) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return PM_OK;
}

int pm_status(pm_ctx* ctx, uint32_t* out_bits) {
    if (!ctx || !out_bits) return PM_ERR_INVALID;
    CK(cudaMemcpyAsync(out_bits, ctx->status.p, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemsetAsync(ctx->status.p, 0, 4, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PM_OK;
}

int pm_launch_count(pm_ctx* ctx, int64_t* out) {
    if (!ctx || !out) return PM_ERR_INVALID;
    *out = ctx->launches;
    return PM_OK;
}

namespace {

MlpInputs cache_inputs(const float* pos, const float* nrm, int64_t n) {
    MlpInputs in{};
    in.n = n;
    in.pos3 = pos;
    in.nrm3 = nrm;
    return in;
}

// loss and gradient of n samples into ctx->cache_grad (zeroed first); loss_out: mean squared error
int cache_backprop(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                   int64_t n, float* loss_out, cudaStream_t st) {
    CK(cudaMemsetAsync(ctx->cache_grad.p, 0, (size_t)PM_CACHE_PARAMS * 4, st));
    CK(cudaMemsetAsync(ctx->cache_loss.p, 0, 4, st));
    const float grad_scale = 2.f / (3.f * (float)n);
    CK(mlp_train(cache_net(ctx), cache_inputs(pos, nrm, n), target, weight, grad_scale, P<float>(ctx->cache_grad),
                 P<float>(ctx->cache_loss), P<unsigned>(ctx->status), ctx->sm_count, st));
    ctx->launches += 1;
    if (loss_out) {
        float l = 0.f;
        CK(cudaMemcpyAsync(&l, ctx->cache_loss.p, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *loss_out = l / (3.f * (float)n);
    }
    return PM_OK;
}

uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

int pm_cache_init(pm_ctx* ctx, const pm_cache_opts* o) {
    if (!ctx || !o) return PM_ERR_INVALID;
    ctx->generation++;
    if (!(o->lr >= 0.f) || !(o->beta1 >= 0.f && o->beta1 < 1.f) || !(o->beta2 >= 0.f && o->beta2 < 1.f) ||
        !(o->eps > 0.f) || !(o->out_scale > 0.f) || o->octave0 < 0 || o->octave0 > 8)
        return fail(ctx, PM_ERR_INVALID, "cache options: lr >= 0, 0 <= beta < 1, eps > 0, out_scale > 0, octave0 0..8");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    const float* box = o->aabb;
    bool zero = true;
    for (int a = 0; a < 6; a++) zero = zero && box[a] == 0.f;
    if (zero) {
        if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "cache: no encoding box and no scene");
        box = ctx->aabb;
    }
    for (int a = 0; a < 3; a++) {
        const float ext = box[3 + a] - box[a];
        ctx->cache_lo[a] = box[a];
        ctx->cache_inv[a] = ext > 0.f ? 1.f / ext : 1.f;
    }
    ENSURE(ctx->cache_w32, (size_t)PM_CACHE_PARAMS * 4);
    ENSURE(ctx->cache_w16, (size_t)PM_CACHE_PARAMS * 2);
    ENSURE(ctx->cache_m, (size_t)PM_CACHE_PARAMS * 4);
    ENSURE(ctx->cache_v, (size_t)PM_CACHE_PARAMS * 4);
    ENSURE(ctx->cache_grad, (size_t)PM_CACHE_PARAMS * 4);
    ENSURE(ctx->cache_loss, 16);
    // He-uniform weights for the ReLU layers, a small output layer; padding zero
    std::vector<float> w(PM_CACHE_PARAMS, 0.f);
    uint64_t state = o->seed;
    for (int l = 0; l < MLP_LAYERS; l++) {
        const int fan_in = l == 0 ? MLP_FEATURES : MLP_DIM;
        const int outs = l == MLP_LAYERS - 1 ? 3 : MLP_DIM;
        const float b = (l == MLP_LAYERS - 1 ? 0.5f : 1.f) * std::sqrt(6.f / (float)fan_in);
        for (int r = 0; r < outs; r++)
            for (int c = 0; c < fan_in; c++) {
                const double u = (double)(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
                w[(size_t)l * MLP_LAYER_STRIDE + r * MLP_DIM + c] = (float)((2.0 * u - 1.0) * b);
            }
    }
    CK(cudaMemcpyAsync(ctx->cache_w32.p, w.data(), (size_t)PM_CACHE_PARAMS * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemsetAsync(ctx->cache_m.p, 0, (size_t)PM_CACHE_PARAMS * 4, ctx->st));
    CK(cudaMemsetAsync(ctx->cache_v.p, 0, (size_t)PM_CACHE_PARAMS * 4, ctx->st));
    CK(cudaMemsetAsync(ctx->cache_grad.p, 0, (size_t)PM_CACHE_PARAMS * 4, ctx->st));
    CK(mlp_to_bf16(P<float>(ctx->cache_w32), P<__nv_bfloat16>(ctx->cache_w16), ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->launches += 1;
    ctx->cache_opts = *o;
    ctx->cache_step = 0;
    ctx->has_cache = true;
    return PM_OK;
}

int pm_cache_train_step(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                        int64_t n, float* out_loss) {
    if (!ctx) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    if (n <= 0 || !pos || !nrm || !target) return fail(ctx, PM_ERR_INVALID, "cache train: n > 0 and sample arrays required");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    if (int rc = cache_backprop(ctx, pos, nrm, target, weight, n, out_loss, ctx->st)) return rc;
    ctx->cache_step++;
    const pm_cache_opts& o = ctx->cache_opts;
    CK(mlp_adam(P<float>(ctx->cache_w32), P<__nv_bfloat16>(ctx->cache_w16), P<float>(ctx->cache_grad),
                P<float>(ctx->cache_m), P<float>(ctx->cache_v), ctx->cache_step, o.lr, o.beta1, o.beta2, o.eps, ctx->st));
    ctx->launches += 1;
    return check_status(ctx, "cache train");
}

int pm_cache_train_steps(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                         int64_t n, int64_t batch, int steps, int64_t* inout_offset, float* out_loss) {
    if (!ctx) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    if (n <= 0 || batch <= 0 || steps < 0 || !pos || !nrm || !target)
        return fail(ctx, PM_ERR_INVALID, "cache train steps: n > 0, batch > 0, steps >= 0 and sample arrays required");
    CK(cudaSetDevice(ctx->device));
    const int64_t b = std::min(batch, n);
    int64_t off = inout_offset ? std::max<int64_t>(*inout_offset, 0) : 0;
    const pm_cache_opts& o = ctx->cache_opts;
    // Without a loss to report, the steps go to the context's training stream
    // (after everything queued so far) and the call returns: work issued next
    // that does not touch the cache (an eye pass, a photon pass) runs beside
    // them, and whatever touches the cache or synchronises waits for them.
    cudaStream_t st = ctx->st;
    if (!out_loss && steps > 0) {
        if (!ctx->train_st) {
            CK(cudaStreamCreateWithFlags(&ctx->train_st, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->train_fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->train_done, cudaEventDisableTiming));
        }
        CK(cudaEventRecord(ctx->train_fork, ctx->st));
        CK(cudaStreamWaitEvent(ctx->train_st, ctx->train_fork, 0));
        st = ctx->train_st;
    } else if (int rc = cache_fence(ctx)) {
        return rc;
    }
    for (int s = 0; s < steps; ++s) {
        if (off + b > n) off = 0;
        if (int rc = cache_backprop(ctx, pos + off * 3, nrm + off * 3, target + off * 3, weight ? weight + off : nullptr,
                                    b, s + 1 == steps ? out_loss : nullptr, st))
            return rc;
        ctx->cache_step++;
        CK(mlp_adam(P<float>(ctx->cache_w32), P<__nv_bfloat16>(ctx->cache_w16), P<float>(ctx->cache_grad),
                    P<float>(ctx->cache_m), P<float>(ctx->cache_v), ctx->cache_step, o.lr, o.beta1, o.beta2, o.eps,
                    st));
        ctx->launches += 1;
        off += b;
    }
    if (inout_offset) *inout_offset = off;
    if (st != ctx->st) {
        CK(cudaEventRecord(ctx->train_done, st));
        ctx->train_pending = true;
        // the steps' device status is reported by the next call that synchronises
        return PM_OK;
    }
    return out_loss ? check_status(ctx, "cache train steps") : PM_OK;
}

int pm_cache_gradient(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                      int64_t n, float* out_grad_host, float* out_loss) {
    if (!ctx || !out_grad_host) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    if (n <= 0 || !pos || !nrm || !target) return fail(ctx, PM_ERR_INVALID, "cache gradient: n > 0 and sample arrays required");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    if (int rc = cache_backprop(ctx, pos, nrm, target, weight, n, out_loss, ctx->st)) return rc;
    CK(cudaMemcpyAsync(out_grad_host, ctx->cache_grad.p, (size_t)PM_CACHE_PARAMS * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemsetAsync(ctx->cache_grad.p, 0, (size_t)PM_CACHE_PARAMS * 4, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return check_status(ctx, "cache gradient");
}

int pm_cache_infer(pm_ctx* ctx, const float* pos, const float* nrm, int64_t n, float* out_rgb) {
    if (!ctx) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    if (n < 0 || (n > 0 && (!pos || !nrm || !out_rgb))) return fail(ctx, PM_ERR_INVALID, "cache infer: bad arguments");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    CK(mlp_infer(cache_net(ctx), cache_inputs(pos, nrm, n), out_rgb, P<unsigned>(ctx->status), ctx->sm_count, ctx->st));
    if (n > 0) ctx->launches += 1;
    return check_status(ctx, "cache infer");
}

int pm_cache_get_params(pm_ctx* ctx, float* out) {
    if (!ctx || !out) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    CK(cudaMemcpyAsync(out, ctx->cache_w32.p, (size_t)PM_CACHE_PARAMS * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PM_OK;
}

int pm_cache_set_params(pm_ctx* ctx, const float* in) {
    if (!ctx || !in) return PM_ERR_INVALID;
    if (!ctx->has_cache) return fail(ctx, PM_ERR_INVALID, "cache not initialised");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    CK(cudaMemcpyAsync(ctx->cache_w32.p, in, (size_t)PM_CACHE_PARAMS * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(mlp_to_bf16(P<float>(ctx->cache_w32), P<__nv_bfloat16>(ctx->cache_w16), ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->launches += 1;
    return PM_OK;
}

int pm_get_requests(pm_ctx* ctx, pm_request_view* out) {
    if (!ctx || !out) return PM_ERR_INVALID;
    std::memset(out, 0, sizeof *out);
    out->count = ctx->last_requests;
    out->pixels = ctx->last_pixels;
    out->a = P<float>(ctx->req_a);
    out->b = P<float>(ctx->req_b);
    out->c = P<float>(ctx->req_c);
    out->px_base = P<uint32_t>(ctx->px_base);
    out->px_count = P<uint32_t>(ctx->px_count);
    out->est_global = P<float>(ctx->est_g);
    return PM_OK;
}

int pm_render_requests(pm_ctx* ctx, int64_t* out) {
    if (!ctx || !out) return PM_ERR_INVALID;
    *out = ctx->last_requests;
    return PM_OK;
}

int pm_stage_times(pm_ctx* ctx, float out_ms[8]) {
    if (!ctx || !out_ms) return PM_ERR_INVALID;
    for (int i = 0; i < 8; i++) out_ms[i] = ctx->stage_ms[i];
    return PM_OK;
}

int pm_set_scene(pm_ctx* ctx, const pm_scene_desc* sd) {
    if (!ctx || !sd) return PM_ERR_INVALID;
    ctx->generation++;
    if (sd->ntri <= 0 || !sd->tri_pos || !sd->tri_nrm || !sd->tri_model || sd->nmodel <= 0 || !sd->materials)
        return fail(ctx, PM_ERR_INVALID, "scene: empty or missing arrays");
    if (sd->light_model < 0 || sd->light_model >= sd->nmodel) return fail(ctx, PM_ERR_INVALID, "scene: light_model out of range");
    const int T = sd->ntri, M = sd->nmodel;
    std::vector<int> first(M, -1), count(M, 0);
    for (int t = 0; t < T; t++) {
        int m = sd->tri_model[t];
        if (m < 0 || m >= M) return fail(ctx, PM_ERR_INVALID, "scene: tri_model out of range");
        if (t > 0 && m < sd->tri_model[t - 1]) return fail(ctx, PM_ERR_INVALID, "scene: triangles must be sorted by model");
        if (first[m] < 0) first[m] = t;
        count[m]++;
    }
    if (count[sd->light_model] == 0) return fail(ctx, PM_ERR_INVALID, "scene: the light model has no triangles");
    CK(cudaSetDevice(ctx->device));

    // per-triangle records (same operations as the reference's triangle test)
    std::vector<float> rec(20 * (size_t)T);
    for (int t = 0; t < T; t++) {
        const float* p = sd->tri_pos + 9 * (size_t)t;
        float v0[3] = {p[0], p[1], p[2]}, v1[3] = {p[3], p[4], p[5]}, v2[3] = {p[6], p[7], p[8]};
        float e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
        float e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
        float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], -(e1[0] * e2[2] - e1[2] * e2[0]), e1[0] * e2[1] - e1[1] * e2[0]};
        float nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
        float denom = 1.0f / nn;
        float nd0 = n[0] * v0[0] + n[1] * v0[1] + n[2] * v0[2];
        float f[3] = {v0[0] - v2[0], v0[1] - v2[1], v0[2] - v2[2]};
        float* r = &rec[20 * (size_t)t];
        int m = sd->tri_model[t];
        r[0] = v0[0]; r[1] = v0[1]; r[2] = v0[2]; r[3] = nd0;
        r[4] = e1[0]; r[5] = e1[1]; r[6] = e1[2]; r[7] = denom;
        r[8] = v2[0]; r[9] = v2[1]; r[10] = v2[2]; std::memcpy(&r[11], &m, 4);
        r[12] = f[0]; r[13] = f[1]; r[14] = f[2]; r[15] = 0.f;
        r[16] = n[0]; r[17] = n[1]; r[18] = n[2]; r[19] = 0.f;
    }
    // model AABBs (first vertex, then grow) and the scene AABB (their union)
    std::vector<float> maabb(6 * (size_t)M, 0.f);
    for (int m = 0; m < M; m++) {
        if (count[m] == 0) continue;
        float* b = &maabb[6 * (size_t)m];
        const float* p0 = sd->tri_pos + 9 * (size_t)first[m];
        for (int a = 0; a < 3; a++) { b[a] = p0[a]; b[a + 3] = p0[a]; }
        for (int t = first[m]; t < first[m] + count[m]; t++)
            for (int v = 0; v < 3; v++) {
                const float* q = sd->tri_pos + 9 * (size_t)t + 3 * v;
                for (int a = 0; a < 3; a++) {
                    if (q[a] > b[a + 3]) b[a + 3] = q[a];
                    if (q[a] < b[a]) b[a] = q[a];
                }
            }
    }
    float aabb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int m = 0; m < M; m++) {
        if (count[m] == 0) continue;
        for (int a = 0; a < 3; a++) {
            aabb[a] = std::min(aabb[a], maabb[6 * m + a]);
            aabb[a + 3] = std::max(aabb[a + 3], maabb[6 * m + a + 3]);
        }
    }
    std::vector<float> ca;
    for (int i = 0; i < M - 1; i++)
        for (int j = i + 1; j < M; j++) {
            add_angle(ca, sd->materials[12 * i + 9], sd->materials[12 * j + 9]);
            add_angle(ca, sd->materials[12 * j + 9], sd->materials[12 * i + 9]);
        }
    for (int i = 0; i < M; i++) {
        add_angle(ca, sd->default_ior, sd->materials[12 * i + 9]);
        add_angle(ca, sd->materials[12 * i + 9], sd->default_ior);
    }
    float ext = std::max(std::max(aabb[3] - aabb[0], aabb[4] - aabb[1]), aabb[5] - aabb[2]);
    const float bvh_pad = 1e-4f * std::max(ext, 1.0f);
    const bool device_bvh = ctx->bvh_builder == PM_BVH_DEVICE_LBVH;
    if (device_bvh && T >= (1 << 23)) return fail(ctx, PM_ERR_INVALID, "device BVH builder: fewer than 2^23 triangles");
    std::vector<float> nodes;
    std::vector<int> prim;
    if (!device_bvh) {
        const auto t0 = std::chrono::steady_clock::now();
        build_bvh(sd->tri_pos, T, bvh_pad, nodes, prim);
        ctx->bvh_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        ctx->bvh_nodes = (int64_t)(nodes.size() / 16);
    } else {
        ctx->bvh_nodes = lbvh_node_count(T);
    }

    ctx->has_scene = false;   // until the new scene is complete
    ENSURE(ctx->tri, rec.size() * 4);
    ENSURE(ctx->tri_pos, 9 * (size_t)T * 4);
    ENSURE(ctx->tri_nrm, 9 * (size_t)T * 4);
    ENSURE(ctx->nodes, (size_t)ctx->bvh_nodes * 64);
    ENSURE(ctx->prim, (size_t)T * 4);
    ENSURE(ctx->maabb, maabb.size() * 4);
    ENSURE(ctx->mats, 12 * (size_t)M * 4);
    ENSURE(ctx->ca, std::max<size_t>(ca.size(), 3) * 4);
    CK(cudaMemcpyAsync(ctx->tri.p, rec.data(), rec.size() * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->tri_pos.p, sd->tri_pos, 9 * (size_t)T * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->tri_nrm.p, sd->tri_nrm, 9 * (size_t)T * 4, cudaMemcpyHostToDevice, ctx->st));
    if (!device_bvh) {
        CK(cudaMemcpyAsync(ctx->nodes.p, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->prim.p, prim.data(), prim.size() * 4, cudaMemcpyHostToDevice, ctx->st));
    } else {
        ENSURE(ctx->bvh_scratch, lbvh_scratch_bytes(T));
        int launches = 0;
        CK(cudaEventRecord(ctx->ev[9], ctx->st));
        CK(lbvh_build(P<float>(ctx->tri_pos), T, bvh_pad, P<float4>(ctx->nodes), P<int>(ctx->prim), ctx->bvh_scratch.p,
                      P<unsigned>(ctx->status), &launches, ctx->st));
        CK(cudaEventRecord(ctx->ev[10], ctx->st));
        CK(cudaEventSynchronize(ctx->ev[10]));
        ctx->bvh_ms = elapsed(ctx->ev[9], ctx->ev[10]);
        ctx->launches += launches;
        release(ctx->bvh_scratch);
        if (int rc = check_status(ctx, "device BVH build")) return rc;
    }
    ENSURE(ctx->tri_leaf, 64 * (size_t)T);
    CK(bvh_leaf_records(P<float4>(ctx->tri), P<int>(ctx->prim), T, P<float4>(ctx->tri_leaf), ctx->st));
    ctx->launches += 1;
    CK(cudaMemcpyAsync(ctx->maabb.p, maabb.data(), maabb.size() * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->mats.p, sd->materials, 12 * (size_t)M * 4, cudaMemcpyHostToDevice, ctx->st));
    if (!ca.empty()) CK(cudaMemcpyAsync(ctx->ca.p, ca.data(), ca.size() * 4, cudaMemcpyHostToDevice, ctx->st));
    ctx->has_tri_diffuse = sd->tri_diffuse != nullptr;
    if (sd->tri_diffuse) {
        ENSURE(ctx->tri_diffuse, 3 * (size_t)T * 4);
        CK(cudaMemcpyAsync(ctx->tri_diffuse.p, sd->tri_diffuse, 3 * (size_t)T * 4, cudaMemcpyHostToDevice, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));   // host vectors go out of scope
    ctx->ntri = T;
    ctx->nmodel = M;
    ctx->light_model = sd->light_model;
    ctx->light_first = first[sd->light_model];
    ctx->light_count = count[sd->light_model];
    ctx->nca = (int)(ca.size() / 3);
    for (int a = 0; a < 3; a++) ctx->light_intensity[a] = sd->light_intensity[a];
    ctx->default_ior = sd->default_ior;
    std::memcpy(ctx->aabb, aabb, sizeof aabb);
    ctx->has_scene = true;
    ctx->scene_bvh_builder = device_bvh ? PM_BVH_DEVICE_LBVH : PM_BVH_HOST_SAH;
    ctx->h_maabb = maabb;
    ctx->eye_order_valid = false;
    ctx->h_mats.assign(sd->materials, sd->materials + 12 * (size_t)M);
    ctx->yield_g = ctx->yield_c = 0.0;
    ctx->yield_bounces = 0;
    for (auto& m : ctx->maps) { m.built = false; m.n = 0; }
    return PM_OK;
}

int pm_set_bvh_builder(pm_ctx* ctx, int builder) {
    if (!ctx) return PM_ERR_INVALID;
    if (builder != PM_BVH_HOST_SAH && builder != PM_BVH_DEVICE_LBVH)
        return fail(ctx, PM_ERR_INVALID, "bvh builder: PM_BVH_HOST_SAH or PM_BVH_DEVICE_LBVH");
    ctx->bvh_builder = builder;
    return PM_OK;
}

int pm_bvh_info(pm_ctx* ctx, int32_t* out_builder, int64_t* out_nodes, float* out_build_ms) {
    if (!ctx) return PM_ERR_INVALID;
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene");
    if (out_builder) *out_builder = ctx->scene_bvh_builder;
    if (out_nodes) *out_nodes = ctx->bvh_nodes;
    if (out_build_ms) *out_build_ms = ctx->bvh_ms;
    return PM_OK;
}

int pm_scene_aabb(pm_ctx* ctx, float out_aabb[6]) {
    if (!ctx || !out_aabb) return PM_ERR_INVALID;
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene");
    std::memcpy(out_aabb, ctx->aabb, 24);
    return PM_OK;
}

static int prepare_trace(pm_ctx* ctx, const pm_trace_opts* o, int64_t npaths, TraceBatch& B) {
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "pm_set_scene first");
    if (o->max_bounces < 1 || o->max_bounces > 32) return fail(ctx, PM_ERR_INVALID, "max_bounces must be 1..32");
    const size_t stage = (size_t)o->max_bounces * (size_t)npaths * 32;
    ENSURE(ctx->counter, 8);
    ENSURE(ctx->stage, stage);
    ENSURE(ctx->cnt_g, (size_t)npaths * 4);
    ENSURE(ctx->cnt_c, (size_t)npaths * 4);
    ENSURE(ctx->scan_g, (size_t)npaths * 4);
    ENSURE(ctx->scan_c, (size_t)npaths * 4);
    ENSURE(ctx->totals, 16);
    ENSURE(ctx->trace_ws, scan_workspace_bytes(npaths));
    B.S = dev_scene(ctx);
    B.seed = o->seed;
    B.tag = o->stream_tag;
    B.max_bounces = o->max_bounces;
    B.path_counter = P<unsigned long long>(ctx->counter);
    B.stage = P<float4>(ctx->stage);
    B.cnt_g = P<uint32_t>(ctx->cnt_g);
    B.cnt_c = P<uint32_t>(ctx->cnt_c);
    B.scan_g = P<uint32_t>(ctx->scan_g);
    B.scan_c = P<uint32_t>(ctx->scan_c);
    B.totals = P<uint32_t>(ctx->totals);
    B.scan_ws = ctx->trace_ws.p;
    B.status = P<unsigned>(ctx->status);
    B.sm_count = ctx->sm_count;
    B.refill = ctx->trace_refill;
    B.work = ctx->count_work ? P<unsigned long long>(ctx->work) : nullptr;
    return PM_OK;
}

namespace {
// The photon pass; after_launch (when set) is called once, right after the
// first batch's kernels are queued on the context stream and before the host
// waits for them (pm_frame queues its eye pass there).
int trace_photons(pm_ctx* ctx, const pm_trace_opts* o, int64_t* out_paths, const std::function<void()>& after_launch) {
    if (!ctx || !o) return PM_ERR_INVALID;
    ctx->generation++;
    if (o->global_capacity < 0 || o->caustic_capacity < 0) return fail(ctx, PM_ERR_INVALID, "negative capacity");
    CK(cudaSetDevice(ctx->device));
    const int64_t cg = o->global_capacity, cc = o->caustic_capacity;
    const int64_t max_paths = o->max_paths > 0 ? o->max_paths : 64 * std::max<int64_t>(std::max(cg, cc), 1);
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    MapState& C = ctx->maps[PM_MAP_CAUSTIC];
    // the lists and grids are empty from here on: a failed allocation below
    // (ensure releases a buffer before growing it) leaves no map in use
    G.built = C.built = false;
    G.n = C.n = 0;
    G.uniform_pow = C.uniform_pow = false;
    G.has_rec = C.has_rec = false;
    G.lists_pending = C.lists_pending = G.spow_pending = C.spow_pending = false;
    ENSURE(G.rec, std::max<int64_t>(cg, 1) * 32); ENSURE(C.rec, std::max<int64_t>(cc, 1) * 32);
    ENSURE(G.pos, std::max<int64_t>(cg, 1) * 12); ENSURE(G.dir, std::max<int64_t>(cg, 1) * 12); ENSURE(G.pow, std::max<int64_t>(cg, 1) * 12);
    ENSURE(C.pos, std::max<int64_t>(cc, 1) * 12); ENSURE(C.dir, std::max<int64_t>(cc, 1) * 12); ENSURE(C.pow, std::max<int64_t>(cc, 1) * 12);
    G.built = C.built = false;
    G.n = C.n = 0;
    float power[3];
    for (int a = 0; a < 3; a++) power[a] = ctx->light_intensity[a] / (float)cg;
    // Batch sizing: paths are traced in batches until both lists are full; the
    // canonical order makes the result independent of the batch boundaries.
    // The first batch is a pilot unless an earlier call on this scene measured
    // the yield (photons per path); later batches aim at the remaining count.
    const int64_t MAX_BATCH = std::max<int64_t>(4096, std::min<int64_t>((int64_t)1 << 25,
                                                 ((int64_t)12 << 30) / (32 * (int64_t)std::max(o->max_bounces, 1))));
    auto batch_for = [&](double yg, double yc, int64_t need_g, int64_t need_c) -> int64_t {
        double need = 0.0;
        if (need_g > 0) need = std::max(need, yg > 0 ? (double)need_g / yg : (double)MAX_BATCH);
        if (need_c > 0) need = std::max(need, yc > 0 ? (double)need_c / yc : (double)MAX_BATCH);
        // margin: the yield of 10M photons' worth of paths varies by about 3e-4
        // between seeds; a short batch is followed by another one
        return std::min<int64_t>(MAX_BATCH, std::max<int64_t>(4096, (int64_t)(need * 1.002) + 4096));
    };
    int64_t nb;
    if (ctx->yield_bounces == o->max_bounces && (ctx->yield_g > 0 || cg == 0) && (ctx->yield_c > 0 || cc == 0))
        nb = batch_for(ctx->yield_g, ctx->yield_c, cg, cc);
    else
        nb = std::min<int64_t>(std::max<int64_t>(cg + cc, 4096), 262144);
    int64_t fg = 0, fc = 0, p0 = 0;
    double yg = 0.0, yc = 0.0;   // photons per path so far
    int64_t got_g = 0, got_c = 0;
    float k_trace_ms = 0.f;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    while ((fg < cg || fc < cc) && p0 < max_paths) {
        nb = std::min(nb, max_paths - p0);
        TraceBatch B;
        int rc = prepare_trace(ctx, o, nb, B);
        if (rc) return rc;
        B.p0 = p0;
        B.npaths = nb;
        for (int a = 0; a < 3; a++) B.power[a] = power[a];
        B.k_begin = ctx->ev[12];
        B.k_end = ctx->ev[13];
        PhotonList LG{P<float>(G.pos), P<float>(G.dir), P<float>(G.pow), cg, fg, P<float4>(G.rec)};
        PhotonList LC{P<float>(C.pos), P<float>(C.dir), P<float>(C.pow), cc, fc, P<float4>(C.rec)};
        // the direction and power lists are left to fill_pending: the grid
        // reads the records, and a traced map's power is uniform
        LG.lists = LC.lists = false;
        CK(trace_batch(B, LG, LC, ctx->st));
        if (p0 == 0 && after_launch) after_launch();
        ctx->launches += 4;
        CK(cudaMemcpyAsync(ctx->hbuf + 2, B.totals, 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        uint32_t tot[2] = {ctx->hbuf[2], ctx->hbuf[3]};
        if (cc == 0) tot[1] = 0;   // no caustic map: its total was not scanned
        k_trace_ms += elapsed(ctx->ev[12], ctx->ev[13]);
        got_g += tot[0];
        got_c += tot[1];
        fg = std::min(cg, fg + (int64_t)tot[0]);
        fc = std::min(cc, fc + (int64_t)tot[1]);
        p0 += nb;
        yg = (double)got_g / (double)p0;
        yc = (double)got_c / (double)p0;
        nb = batch_for(yg, yc, cg - fg, cc - fc);
    }
    if (p0 > 0) {
        ctx->yield_g = yg;
        ctx->yield_c = yc;
        ctx->yield_bounces = o->max_bounces;
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[1]));
    ctx->stage_ms[0] = elapsed(ctx->ev[0], ctx->ev[1]);
    ctx->stage_ms[5] = k_trace_ms;
    G.n = fg;
    C.n = fc;
    for (MapState* m : {&G, &C}) {   // every photon of a traced map has power intensity / global capacity
        m->uniform_pow = true;
        m->has_rec = true;
        m->lists_pending = true;
        for (int a = 0; a < 3; a++) m->pow_value[a] = power[a];
    }
    if (out_paths) *out_paths = p0;
    int rc = check_status(ctx, "trace");
    if (rc) return rc;
    if (fg < cg || fc < cc) return fail(ctx, PM_ERR_INVALID, "photon maps not filled within max_paths");
    return PM_OK;
}
}  // namespace

int pm_trace_photons(pm_ctx* ctx, const pm_trace_opts* o, int64_t* out_paths) {
    return trace_photons(ctx, o, out_paths, nullptr);
}

int pm_trace_work(pm_ctx* ctx, const pm_trace_opts* o, int64_t* out_paths, uint64_t out_work[3]) {
    if (!ctx || !o || !out_work) return PM_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    ENSURE(ctx->work, 32);
    CK(cudaMemsetAsync(ctx->work.p, 0, 32, ctx->st));
    ctx->count_work = true;
    const int rc = pm_trace_photons(ctx, o, out_paths);
    ctx->count_work = false;
    if (rc) return rc;
    unsigned long long w[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(w, ctx->work.p, 24, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int i = 0; i < 3; i++) out_work[i] = w[i];
    return PM_OK;
}

int pm_trace_paths(pm_ctx* ctx, const pm_trace_opts* o, int64_t p0, int64_t p1, int64_t power_capacity,
                   float* g_pos, float* g_dir, float* c_pos, float* c_dir, uint32_t* counts,
                   int64_t* out_ng, int64_t* out_nc) {
    if (!ctx || !o || p1 <= p0 || !g_pos || !g_dir || !c_pos || !c_dir) return PM_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    const int64_t n = p1 - p0;
    TraceBatch B;
    int rc = prepare_trace(ctx, o, n, B);
    if (rc) return rc;
    B.p0 = p0;
    B.npaths = n;
    for (int a = 0; a < 3; a++) B.power[a] = ctx->light_intensity[a] / (float)power_capacity;
    const int64_t cap = n * o->max_bounces;
    ENSURE(ctx->scratch_pow, (size_t)cap * 24);
    float* pw = P<float>(ctx->scratch_pow);
    PhotonList LG{g_pos, g_dir, pw, cap, 0};
    PhotonList LC{c_pos, c_dir, pw + 3 * cap, cap, 0};
    CK(trace_batch(B, LG, LC, ctx->st));
    ctx->launches += 4;
    if (counts) {
        CK(cudaMemcpy2DAsync(counts, 8, B.cnt_g, 4, 4, (size_t)n, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpy2DAsync(counts + 1, 8, B.cnt_c, 4, 4, (size_t)n, cudaMemcpyDeviceToDevice, ctx->st));
    }
    uint32_t tot[2] = {0, 0};
    CK(cudaMemcpyAsync(tot, B.totals, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (out_ng) *out_ng = tot[0];
    if (out_nc) *out_nc = tot[1];
    return check_status(ctx, "trace_paths");
}

int pm_set_photons(pm_ctx* ctx, int map, int64_t n, const float* pos, const float* power, const float* dir) {
    if (!ctx || n < 0 || (n > 0 && (!pos || !power || !dir))) return PM_ERR_INVALID;
    ctx->generation++;
    if (int rc = valid_map(ctx, map)) return rc;
    CK(cudaSetDevice(ctx->device));
    MapState& m = ctx->maps[map];
    m.n = 0;            // empty until the new list is in place
    m.built = false;
    m.uniform_pow = false;
    m.has_rec = false;
    m.lists_pending = m.spow_pending = false;
    ENSURE(m.pos, std::max<int64_t>(n, 1) * 12);
    ENSURE(m.dir, std::max<int64_t>(n, 1) * 12);
    ENSURE(m.pow, std::max<int64_t>(n, 1) * 12);
    if (n > 0) {
        CK(cudaMemcpyAsync(m.pos.p, pos, (size_t)n * 12, cudaMemcpyDefault, ctx->st));
        CK(cudaMemcpyAsync(m.dir.p, dir, (size_t)n * 12, cudaMemcpyDefault, ctx->st));
        CK(cudaMemcpyAsync(m.pow.p, power, (size_t)n * 12, cudaMemcpyDefault, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    m.n = n;
    m.built = false;
    return PM_OK;
}

namespace {

// A grid build issued on the context stream (grid_issue) and not yet
// recorded in its map (grid_commit).
struct GridIssued {
    GridPlan plan;
    int S = 1;
    float box[6] = {0, 0, 0, 0, 0, 0};
};

// Every launch of a grid build on the context stream (the counting pass's
// read of the fullest cell, which decides the re-grid and the sub-cell split,
// is the one host wait); the map stays unbuilt until grid_commit.  The global
// map's build is timed into ev[2] .. ev[3].
int grid_issue(pm_ctx* ctx, int map, const pm_grid_opts* o, const float* aabb, GridIssued& gi) {
    ctx->generation++;
    if (int rc = valid_map(ctx, map)) return rc;
    pm_grid_opts d = {1000, 5, 5, 0, 0};
    if (!o) o = &d;
    if (o->desired_per_cell < 1 || o->regrid_div < 1 || o->regrid_mult < 1) return fail(ctx, PM_ERR_INVALID, "grid options must be >= 1");
    if (!(o->sub_div == 0 || o->sub_div == 1 || o->sub_div == 2 || o->sub_div == 4 || o->sub_div == 8))
        return fail(ctx, PM_ERR_INVALID, "sub_div must be 0, 1, 2, 4 or 8");
    const float* box = aabb ? aabb : ctx->aabb;
    if (!aabb && !ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene and no aabb");
    CK(cudaSetDevice(ctx->device));
    MapState& m = ctx->maps[map];
    const int64_t n = m.n;
    if (n == 0) return fail(ctx, PM_ERR_INVALID, "map has no photons");
    m.built = false;   // until the new grid is complete (a failed allocation leaves no half grid in use)
    int d1[3], d2[3];
    float c1, c2;
    grid_dims(box, n, o->desired_per_cell, d1, &c1);
    grid_dims(box, n, std::max(o->desired_per_cell / o->regrid_div, 1), d2, &c2);
    const int64_t cells_max = std::max<int64_t>((int64_t)d1[0] * d1[1] * d1[2], (int64_t)d2[0] * d2[1] * d2[2]);
    if (cells_max <= 0 || cells_max > ((int64_t)1 << 26)) return fail(ctx, PM_ERR_INVALID, "grid: cell count out of range");
    ENSURE(m.starts, (size_t)cells_max * 4);
    ENSURE(m.sizes, (size_t)cells_max * 4);
    ENSURE(m.gpos, (size_t)n * 16);
    ENSURE(m.gdir, (size_t)n * 12);
    ENSURE(m.gpow, (size_t)n * 12);
    ENSURE(m.cid, (size_t)n * 4);
    ENSURE(m.keys0, (size_t)n * 4);
    ENSURE(m.keys1, (size_t)n * 4);
    ENSURE(m.vals0, (size_t)n * 4);
    ENSURE(m.vals1, (size_t)n * 4);
    ENSURE(m.small, 64);
    ENSURE(m.counts2, (size_t)((int64_t)d2[0] * d2[1] * d2[2]) * 4);
    GridBuffers B;
    B.pos = P<float>(m.pos); B.dir = P<float>(m.dir); B.pow = P<float>(m.pow); B.n = n;
    B.uniform_pow = m.uniform_pow;
    B.defer_pow = true;   // a uniform sorted power is written by fill_pending when asked for
    B.rec = m.has_rec ? P<float4>(m.rec) : nullptr;
    for (int a = 0; a < 3; a++) B.pow_value[a] = m.pow_value[a];
    B.cell_starts = P<uint32_t>(m.starts); B.cell_sizes = P<uint32_t>(m.sizes);
    B.gpos = P<float4>(m.gpos); B.gdir = P<float>(m.gdir); B.gpow = P<float>(m.gpow);
    B.cid = P<uint32_t>(m.cid);
    B.keys[0] = P<uint32_t>(m.keys0); B.keys[1] = P<uint32_t>(m.keys1);
    B.vals[0] = P<uint32_t>(m.vals0); B.vals[1] = P<uint32_t>(m.vals1);
    B.host_words = ctx->hbuf + 4;
    B.small = P<uint32_t>(m.small);
    B.counts2 = P<uint32_t>(m.counts2);
    B.status = P<unsigned>(ctx->status);
    if (map == PM_MAP_GLOBAL) CK(cudaEventRecord(ctx->ev[2], ctx->st));
    GridPlan& plan = gi.plan;
    CK(grid_count(B, box, o->desired_per_cell, o->regrid_mult, o->regrid_div, &plan, ctx->st));
    const int S = gi.S = o->sub_div > 0 ? o->sub_div : grid_auto_subdiv(plan.max_count, o->k_hint > 0 ? o->k_hint : 64);
    const int64_t keys = plan.cells * S * S * S;
    if (keys > ((int64_t)1 << 31)) return fail(ctx, PM_ERR_INVALID, "grid: too many sub-cells");
    size_t hist_elems = 0, scan_ws = 0;
    grid_scratch_sizes(n, keys, &hist_elems, &scan_ws);
    ENSURE(m.hist, hist_elems * 4);
    ENSURE(m.scan_ws, scan_ws);
    ENSURE(m.key_counts, (size_t)keys * 4);
    ENSURE(m.key_starts, (size_t)(keys + 1) * 4);
    B.hist = P<uint32_t>(m.hist);
    B.scan_ws = m.scan_ws.p;
    B.key_counts = P<uint32_t>(m.key_counts);
    B.key_starts = P<uint32_t>(m.key_starts);
    CK(grid_sort(B, box, plan, S, ctx->st));
    ctx->launches += plan.launches;
    if (map == PM_MAP_GLOBAL) CK(cudaEventRecord(ctx->ev[3], ctx->st));
    std::memcpy(gi.box, box, 24);
    return PM_OK;
}

void grid_commit(pm_ctx* ctx, int map, const GridIssued& gi) {
    MapState& m = ctx->maps[map];
    for (int a = 0; a < 3; a++) m.dims[a] = gi.plan.dims[a];
    m.cell = gi.plan.cell;
    m.cells = gi.plan.cells;
    m.S = gi.S;
    std::memcpy(m.aabb, gi.box, 24);
    m.built = true;
    m.spow_pending = m.uniform_pow;
}

// A traced map's direction and power lists, and its grid's sorted power, are
// not written by the photon pass and the grid build (the grid reads the
// 32-byte records, the estimate the uniform power): they are written here,
// on the context stream, for the calls that hand them out.
int fill_pending(pm_ctx* ctx, MapState& m) {
    if (!m.lists_pending && !m.spow_pending) return PM_OK;
    if (m.lists_pending)
        CK(photon_lists_from_rec(P<float4>(m.rec), m.n, m.pow_value, P<float>(m.dir), P<float>(m.pow), ctx->st));
    if (m.spow_pending && m.built)
        CK(photon_lists_from_rec(nullptr, m.n, m.pow_value, nullptr, P<float>(m.gpow), ctx->st));
    m.lists_pending = m.spow_pending = false;
    CK(cudaStreamSynchronize(ctx->st));
    return PM_OK;
}

}  // namespace

int pm_build_grid(pm_ctx* ctx, int map, const pm_grid_opts* o, const float* aabb) {
    if (!ctx) return PM_ERR_INVALID;
    GridIssued gi;
    if (int rc = grid_issue(ctx, map, o, aabb, gi)) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    if (map == PM_MAP_GLOBAL) ctx->stage_ms[1] = elapsed(ctx->ev[2], ctx->ev[3]);
    if (int rc = check_status(ctx, "grid build")) return rc;
    grid_commit(ctx, map, gi);
    return PM_OK;
}

int pm_get_photons(pm_ctx* ctx, int map, pm_photon_view* out) {
    if (!ctx || !out) return PM_ERR_INVALID;
    if (int rc = valid_map(ctx, map)) return rc;
    MapState& m = ctx->maps[map];
    CK(cudaSetDevice(ctx->device));
    if (int rc = fill_pending(ctx, m)) return rc;
    std::memset(out, 0, sizeof *out);
    out->count = m.n;
    out->list_pos = P<float>(m.pos);
    out->list_dir = P<float>(m.dir);
    out->list_power = P<float>(m.pow);
    if (m.built) {
        out->cells = m.cells;
        for (int a = 0; a < 3; a++) out->dims[a] = m.dims[a];
        out->cell_size = m.cell;
        std::memcpy(out->aabb, m.aabb, 24);
        out->cell_starts = P<uint32_t>(m.starts);
        out->cell_sizes = P<uint32_t>(m.sizes);
        out->sorted_pos = P<float>(m.gpos);
        out->sorted_dir = P<float>(m.gdir);
        out->sorted_power = P<float>(m.gpow);
        out->sub_div = m.S;
        out->key_starts = P<uint32_t>(m.key_starts);
    }
    return PM_OK;
}

int pm_save_photons(pm_ctx* ctx, int map, const char* path) {
    if (!ctx || !path) return PM_ERR_INVALID;
    if (int rc = valid_map(ctx, map)) return rc;
    MapState& m = ctx->maps[map];
    CK(cudaSetDevice(ctx->device));
    if (int rc = fill_pending(ctx, m)) return rc;
    const int64_t n = m.n;
    try {
        std::vector<float> pos(3 * n), pw(3 * n), dir(3 * n);
        if (n > 0) {
            CK(cudaMemcpyAsync(pos.data(), m.pos.p, 12 * n, cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaMemcpyAsync(pw.data(), m.pow.p, 12 * n, cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaMemcpyAsync(dir.data(), m.dir.p, 12 * n, cudaMemcpyDeviceToHost, ctx->st));
        }
        CK(cudaStreamSynchronize(ctx->st));
        FILE* f = fopen(path, "wb");
        if (!f) return fail(ctx, PM_ERR_IO, std::string("cannot open ") + path);
        uint64_t cnt = (uint64_t)n;
        bool ok = fwrite(&cnt, 8, 1, f) == 1;
        std::vector<float> rec(9 * 4096);
        for (int64_t i = 0; ok && i < n; i += 4096) {
            int64_t k = std::min<int64_t>(4096, n - i);
            for (int64_t j = 0; j < k; j++) {
                std::memcpy(&rec[9 * j], &pos[3 * (i + j)], 12);
                std::memcpy(&rec[9 * j + 3], &pw[3 * (i + j)], 12);
                std::memcpy(&rec[9 * j + 6], &dir[3 * (i + j)], 12);
            }
            ok = fwrite(rec.data(), 36, (size_t)k, f) == (size_t)k;
        }
        if (fclose(f) != 0) ok = false;
        return ok ? PM_OK : fail(ctx, PM_ERR_IO, std::string("write failed: ") + path);
    } catch (const std::bad_alloc&) {
        return fail(ctx, PM_ERR_OOM, "pm_save_photons: host memory");
    }
}

// The file is checked against its header before anything is allocated: the
// reference's reader (Initializer.cu:102-141) trusts the count, and a corrupt
// or truncated header must not turn into a huge allocation here.
int pm_load_photons(pm_ctx* ctx, int map, const char* path) {
    if (!ctx || !path) return PM_ERR_INVALID;
    if (int rc = valid_map(ctx, map)) return rc;
    std::unique_ptr<FILE, int (*)(FILE*)> file(fopen(path, "rb"), fclose);
    FILE* f = file.get();
    if (!f) return fail(ctx, PM_ERR_IO, std::string("cannot open ") + path);
    uint64_t cnt = 0;
    long long bytes = -1;
    if (fseek(f, 0, SEEK_END) == 0) bytes = (long long)ftello(f);
    if (bytes < 8 || fseek(f, 0, SEEK_SET) != 0 || fread(&cnt, 8, 1, f) != 1)
        return fail(ctx, PM_ERR_IO, "photon file: no count header");
    if (cnt > ((uint64_t)1 << 32) || (uint64_t)(bytes - 8) / 36 < cnt)
        return fail(ctx, PM_ERR_IO, "photon file: the count header needs " + std::to_string(cnt) +
                                        " records, the file holds " + std::to_string((bytes - 8) / 36));
    try {
        std::vector<float> pos(3 * cnt), pw(3 * cnt), dir(3 * cnt), rec(9 * 4096);
        for (uint64_t i = 0; i < cnt; i += 4096) {
            const size_t k = (size_t)std::min<uint64_t>(4096, cnt - i);
            if (fread(rec.data(), 36, k, f) != k) return fail(ctx, PM_ERR_IO, "truncated photon file");
            for (size_t j = 0; j < k; j++) {
                std::memcpy(&pos[3 * (i + j)], &rec[9 * j], 12);
                std::memcpy(&pw[3 * (i + j)], &rec[9 * j + 3], 12);
                std::memcpy(&dir[3 * (i + j)], &rec[9 * j + 6], 12);
            }
        }
        file.reset();
        return pm_set_photons(ctx, map, (int64_t)cnt, pos.data(), pw.data(), dir.data());
    } catch (const std::bad_alloc&) {
        return fail(ctx, PM_ERR_OOM, "pm_load_photons: host memory");
    }
}


int pm_gather(pm_ctx* ctx, int map, int64_t n, const float* qpos, const float* qnrm, int k, float radius,
              float* out_rad, uint32_t* out_ids, int32_t* out_cnt) {
    if (!ctx || n < 0 || (n > 0 && (!qpos || !qnrm || !out_rad))) return PM_ERR_INVALID;
    if (int rc = valid_map(ctx, map)) return rc;
    if (k < 0 || k > 256) return fail(ctx, PM_ERR_INVALID, "k must be 0..256");
    MapState& m = ctx->maps[map];
    if (!m.built) return fail(ctx, PM_ERR_INVALID, "map grid not built");
    CK(cudaSetDevice(ctx->device));
    GatherQueries Q{};
    Q.n = n; Q.pos3 = qpos; Q.nrm3 = qnrm;
    GatherOut O{out_rad, out_ids, out_cnt, nullptr};
    CK(gather(grid_of(m, m), Q, radius, k, 0, O, P<unsigned>(ctx->status), ctx->st));
    ctx->launches += 1;
    return check_status(ctx, "gather");
}

int pm_camera_setup(const float position[3], const float direction[3], const float upv[3], float fov, int32_t W,
                    int32_t H, pm_camera* out) {
    if (!position || !direction || !upv || !out || W <= 0 || H <= 0) return PM_ERR_INVALID;
    const float pi = 3.141592653589793f;
    float aspect = (float)W / (float)H;
    float theta = fov * pi / 180.0f;
    float h = std::tan(theta / 2);
    out->viewport_h = 2.0f * h;
    out->viewport_w = aspect * out->viewport_h;
    out->focal = 1.0f;
    auto norm_div = [](const float* v, float* o) {
        if (v[0] == 0.f && v[1] == 0.f && v[2] == 0.f) { o[0] = v[0]; o[1] = v[1]; o[2] = v[2]; return; }
        float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        o[0] = v[0] / l; o[1] = v[1] / l; o[2] = v[2] / l;
    };
    auto cross = [](const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = -(a[0] * b[2] - a[2] * b[0]);
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    for (int a = 0; a < 3; a++) out->position[a] = position[a];
    norm_div(direction, out->forward);
    float rc[3];
    cross(out->forward, upv, rc);
    norm_div(rc, out->right);
    cross(out->right, out->forward, out->up);
    out->width = W;
    out->height = H;
    return PM_OK;
}

namespace {

// state of one render between the eye pass and the resolve
struct FrameSetup {
    CameraDev cd;
    Requests R;
    DevScene S;
    int64_t npx = 0, cap = 0, nreq = 0;
    bool caustic = false;
    bool ordered = false;              // the requests' Morton order is already issued (pm_frame)
    const uint32_t* order = nullptr;
};


// buffers and the eye pass on stream st (timed into ev[4] .. ev[5]); with
// y0 < y1 only the pixel blocks that meet rows [y0, y1) run, and every other
// pixel has no requests
int render_eye_launch(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, FrameSetup& F, cudaStream_t st,
                      int y0 = 0, int y1 = 0) {
    MapState& C = ctx->maps[PM_MAP_CAUSTIC];
    F.npx = (int64_t)cam->width * cam->height;
    const int64_t per_px = ((int64_t)1 << std::max(o->max_depth, 1)) - 1;
    F.cap = F.npx * per_px;
    ENSURE(ctx->req_a, (size_t)F.cap * 16);
    ENSURE(ctx->req_b, (size_t)F.cap * 16);
    ENSURE(ctx->req_c, (size_t)F.cap * 16);
    ENSURE(ctx->req_counter, 8);
    ENSURE(ctx->px_base, (size_t)F.npx * 4);
    ENSURE(ctx->px_count, (size_t)F.npx * 4);
    ENSURE(ctx->est_g, (size_t)F.cap * 12);
    F.caustic = C.built;
    if (F.caustic) ENSURE(ctx->est_c, (size_t)F.cap * 12);
    F.S = dev_scene(ctx);
    for (int a = 0; a < 3; a++) {
        F.cd.pos[a] = cam->position[a]; F.cd.fwd[a] = cam->forward[a]; F.cd.right[a] = cam->right[a]; F.cd.up[a] = cam->up[a];
    }
    F.cd.vw = cam->viewport_w; F.cd.vh = cam->viewport_h; F.cd.focal = cam->focal;
    F.cd.W = cam->width; F.cd.H = cam->height;
    Requests& R = F.R;
    R.a = P<float4>(ctx->req_a); R.b = P<float4>(ctx->req_b); R.c = P<float4>(ctx->req_c);
    R.cap = F.cap;
    R.counter = P<unsigned long long>(ctx->req_counter);
    R.px_base = P<uint32_t>(ctx->px_base);
    R.px_count = P<uint32_t>(ctx->px_count);
    if (!ctx->eye_order_valid || std::memcmp(&ctx->eye_order_cam, cam, sizeof *cam) != 0) {
        std::vector<int>& order = ctx->h_eye_order;
        order.clear();
        eye_block_order(ctx, cam, order);
        ENSURE(ctx->eye_order, order.size() * 4);
        CK(cudaMemcpyAsync(ctx->eye_order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st));
        ctx->eye_order_cam = *cam;
        ctx->eye_order_valid = true;
    }
    const int* order = P<int>(ctx->eye_order);
    int64_t nblocks = -1;
    if (y0 < y1) {
        // the band's blocks, in the full order's (slow blocks first)
        const int64_t T = eye_threads(), lo = (int64_t)y0 * cam->width, hi = (int64_t)y1 * cam->width;
        std::vector<int> band;
        for (int b : ctx->h_eye_order)
            if ((int64_t)b * T < hi && ((int64_t)b + 1) * T > lo) band.push_back(b);
        ENSURE(ctx->eye_band, std::max<size_t>(band.size(), 1) * 4);
        if (!band.empty())
            CK(cudaMemcpyAsync(ctx->eye_band.p, band.data(), band.size() * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(ctx->px_count.p, 0, (size_t)F.npx * 4, st));
        order = P<int>(ctx->eye_band);
        nblocks = (int64_t)band.size();
    }
    CK(cudaEventRecord(ctx->ev[4], st));
    CK(eye_pass(F.S, F.cd, o->max_depth, R, P<unsigned>(ctx->status), st, order, nblocks));
    CK(cudaEventRecord(ctx->ev[5], st));
    ctx->launches += 1;
    return PM_OK;
}

// the request count of the eye pass (ordered on ctx->st)
int render_eye_count(pm_ctx* ctx, FrameSetup& F, cudaStream_t st = nullptr) {
    if (!st) st = ctx->st;
    CK(cudaMemcpyAsync(ctx->hbuf + 6, F.R.counter, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    unsigned long long nreq = 0;
    std::memcpy(&nreq, ctx->hbuf + 6, 8);
    F.nreq = (int64_t)std::min<unsigned long long>(nreq, (unsigned long long)F.cap);
    ctx->last_requests = F.nreq;
    ctx->last_pixels = F.npx;
    return PM_OK;
}

// buffers, eye pass and the request count
int render_eye(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, FrameSetup& F) {
    if (int rc = render_eye_launch(ctx, cam, o, F, ctx->st)) return rc;
    return render_eye_count(ctx, F);
}

// caustic gather, resolve (ev[7] .. ev[8]) and the stage times
int render_finish(pm_ctx* ctx, const pm_render_opts* o, FrameSetup& F, uint8_t* out_rgb8, float* out_radiance) {
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    MapState& C = ctx->maps[PM_MAP_CAUSTIC];
    if (F.caustic) {
        GatherQueries Q{};
        Q.n = F.nreq; Q.pos4 = F.R.a; Q.nrm4 = F.R.b; Q.flag_mask = 2u;
        GatherOut OC{P<float>(ctx->est_c), nullptr, nullptr, nullptr};
        CK(gather(grid_of(C, o->faithful_caustic ? G : C), Q, o->r_caustic, o->k_caustic, 1, OC,
                  P<unsigned>(ctx->status), ctx->st));
        ctx->launches += 1;
    }
    CK(cudaEventRecord(ctx->ev[7], ctx->st));
    const float tone_t = (float)std::pow((double)0.6f, -1);
    CK(resolve(F.S, F.cd, F.R, P<float>(ctx->est_g), F.caustic ? P<float>(ctx->est_c) : nullptr, tone_t, out_rgb8,
               out_radiance, ctx->st));
    CK(cudaEventRecord(ctx->ev[8], ctx->st));
    ctx->launches += 1;
    CK(cudaEventSynchronize(ctx->ev[8]));
    ctx->stage_ms[2] = elapsed(ctx->ev[4], ctx->ev[5]);
    ctx->stage_ms[3] = elapsed(ctx->ev[6], ctx->ev[7]);
    ctx->stage_ms[4] = elapsed(ctx->ev[7], ctx->ev[8]);
    return PM_OK;
}

}  // namespace

namespace {

// The gather visits the requests in Morton order of their hit points: 27-bit
// keys in the scene box, sorted by the library's stable radix sort on stream st.
int request_order(pm_ctx* ctx, FrameSetup& F, cudaStream_t st) {
    F.ordered = true;
    F.order = nullptr;
    if (F.nreq <= 0) return PM_OK;
    const int64_t n = F.nreq;
    ENSURE(ctx->rq_keys, (size_t)n * 4);
    ENSURE(ctx->rq_k0, (size_t)n * 4); ENSURE(ctx->rq_k1, (size_t)n * 4);
    ENSURE(ctx->rq_v0, (size_t)n * 4); ENSURE(ctx->rq_v1, (size_t)n * 4);
    ENSURE(ctx->rq_hist, radix_hist_elems(n) * 4);
    ENSURE(ctx->rq_ws, scan_workspace_bytes((int64_t)radix_hist_elems(n)));
    CK(request_keys(F.R.a, n, ctx->aabb, P<uint32_t>(ctx->rq_keys), st));
    RadixBuffers RB{{P<uint32_t>(ctx->rq_k0), P<uint32_t>(ctx->rq_k1)}, {P<uint32_t>(ctx->rq_v0), P<uint32_t>(ctx->rq_v1)},
                    P<uint32_t>(ctx->rq_hist), ctx->rq_ws.p, P<unsigned>(ctx->status)};
    int launches = 0;
    CK(radix_sort_u32(RB, P<uint32_t>(ctx->rq_keys), nullptr, n, REQUEST_KEY_BITS, false, nullptr, &F.order, &launches,
                      st));
    ctx->launches += launches + 1;
    return PM_OK;
}

// global gather, caustic gather, resolve and the status check of a frame whose requests are counted
int render_rest(pm_ctx* ctx, const pm_render_opts* o, FrameSetup& F, uint8_t* out_rgb8, float* out_radiance) {
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    GatherQueries Q{};
    Q.n = F.nreq; Q.pos4 = F.R.a; Q.nrm4 = F.R.b; Q.flag_mask = 1u;
    CK(cudaEventRecord(ctx->ev[6], ctx->st));
    if (!F.ordered)
        if (int rc = request_order(ctx, F, ctx->st)) return rc;
    Q.idx = F.order;
    GatherOut OG{P<float>(ctx->est_g), nullptr, nullptr, nullptr};
    CK(cudaEventRecord(ctx->ev[11], ctx->st));
    CK(gather(grid_of(G, G), Q, o->r_global, o->k_global, 0, OG, P<unsigned>(ctx->status), ctx->st));
    CK(cudaEventRecord(ctx->ev[12], ctx->st));
    ctx->launches += 1;
    if (int rc = render_finish(ctx, o, F, out_rgb8, out_radiance)) return rc;
    ctx->stage_ms[6] = elapsed(ctx->ev[11], ctx->ev[12]);
    return check_status(ctx, "render");
}

}  // namespace

int pm_frame(pm_ctx* ctx, const pm_trace_opts* to, const pm_grid_opts* go, const pm_camera* cam,
             const pm_render_opts* o, uint8_t* out_rgb8, float* out_radiance, int64_t* out_paths) {
    if (!ctx || !to || !go || !cam || !o || !out_rgb8) return PM_ERR_INVALID;
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene");
    if (o->max_depth < 0 || o->max_depth > RENDER_MAX_DEPTH) return fail(ctx, PM_ERR_INVALID, "max_depth must be 0..5");
    if (o->k_global < 0 || o->k_global > 256 || o->k_caustic < 0 || o->k_caustic > 256)
        return fail(ctx, PM_ERR_INVALID, "k must be 0..256");
    if (cam->width <= 0 || cam->height <= 0) return fail(ctx, PM_ERR_INVALID, "bad camera size");
    CK(cudaSetDevice(ctx->device));
    // The eye pass needs neither the photons nor the grid: it is queued on the
    // frame stream right after the photon pass's kernels, so its blocks take
    // the SMs the persistent tracer leaves as its last paths end (and the
    // grid build then runs with the GPU to itself: step 8.40 -> 8.23 ms); the
    // request count and the requests' Morton order follow on the same stream
    // beside the grid build, and the gather waits for both streams.
    if (!ctx->frame_st) {
        CK(cudaStreamCreateWithFlags(&ctx->frame_st, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->frame_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->frame_done, cudaEventDisableTiming));
    }
    CK(cudaEventRecord(ctx->frame_fork, ctx->st));   // the previous frame's reads of the eye buffers are done
    CK(cudaStreamWaitEvent(ctx->frame_st, ctx->frame_fork, 0));
    FrameSetup F;
    int erc = PM_OK;
    bool eye_queued = false;
    const int trc = trace_photons(ctx, to, out_paths, [&]() {
        erc = render_eye_launch(ctx, cam, o, F, ctx->frame_st);
        eye_queued = true;
    });
    if (trc) {
        if (eye_queued) cudaStreamSynchronize(ctx->frame_st);   // its buffers stay in use until it ends
        return trc;
    }
    const bool caustic = to->caustic_capacity > 0 && o->k_caustic > 0;
    GridIssued gg, gc;
    int rc = eye_queued ? erc : render_eye_launch(ctx, cam, o, F, ctx->frame_st);
    if (rc == PM_OK) rc = grid_issue(ctx, PM_MAP_GLOBAL, go, nullptr, gg);
    if (rc == PM_OK && caustic) rc = grid_issue(ctx, PM_MAP_CAUSTIC, go, nullptr, gc);
    if (rc == PM_OK) rc = render_eye_count(ctx, F, ctx->frame_st);
    if (rc == PM_OK) rc = request_order(ctx, F, ctx->frame_st);
    if (rc == PM_OK && cudaEventRecord(ctx->frame_done, ctx->frame_st) != cudaSuccess)
        rc = cuda_fail(ctx, cudaErrorUnknown, "frame event");
    if (rc == PM_OK && cudaStreamWaitEvent(ctx->st, ctx->frame_done, 0) != cudaSuccess)
        rc = cuda_fail(ctx, cudaErrorUnknown, "frame join");
    if (rc != PM_OK) {
        // the frame stream's buffers stay in use until it ends
        cudaStreamSynchronize(ctx->frame_st);
        cudaStreamSynchronize(ctx->st);
        return rc;
    }
    // the grids are complete in stream order before the gather reads them;
    // their device status is checked with the frame's
    grid_commit(ctx, PM_MAP_GLOBAL, gg);
    if (caustic) grid_commit(ctx, PM_MAP_CAUSTIC, gc);
    if (int rc2 = render_checks(ctx, cam, o)) return rc2;
    F.caustic = ctx->maps[PM_MAP_CAUSTIC].built;
    if (F.caustic) ENSURE(ctx->est_c, (size_t)F.cap * 12);
    rc = render_rest(ctx, o, F, out_rgb8, out_radiance);
    if (rc == PM_OK) ctx->stage_ms[1] = elapsed(ctx->ev[2], ctx->ev[3]);
    else ctx->maps[PM_MAP_GLOBAL].built = ctx->maps[PM_MAP_CAUSTIC].built = false;
    return rc;
}

int pm_render(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, uint8_t* out_rgb8, float* out_radiance) {
    if (!ctx || !cam || !o || !out_rgb8) return PM_ERR_INVALID;
    if (int rc = render_checks(ctx, cam, o)) return rc;
    CK(cudaSetDevice(ctx->device));
    FrameSetup F;
    if (int rc = render_eye(ctx, cam, o, F)) return rc;
    return render_rest(ctx, o, F, out_rgb8, out_radiance);
}

int pm_render_rows(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, int32_t y0, int32_t y1,
                   uint8_t* out_rgb8, float* out_radiance) {
    if (!ctx || !cam || !o || !out_rgb8) return PM_ERR_INVALID;
    if (int rc = render_checks(ctx, cam, o)) return rc;
    if (y0 < 0 || y1 > cam->height || y0 >= y1) return fail(ctx, PM_ERR_INVALID, "rows: 0 <= y0 < y1 <= height");
    CK(cudaSetDevice(ctx->device));
    FrameSetup F;
    if (int rc = render_eye_launch(ctx, cam, o, F, ctx->st, y0, y1)) return rc;
    if (int rc = render_eye_count(ctx, F)) return rc;
    return render_rest(ctx, o, F, out_rgb8, out_radiance);
}

int pm_render_learned(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, const pm_learned_opts* lo,
                      uint8_t* out_rgb8, float* out_radiance, pm_learned_stats* out_stats) {
    if (!ctx || !cam || !o || !lo || !out_rgb8) return PM_ERR_INVALID;
    if (int rc = learned_checks(ctx, lo)) return rc;
    if (int rc = render_checks(ctx, cam, o)) return rc;
    CK(cudaSetDevice(ctx->device));
    FrameSetup F;
    if (int rc = render_eye(ctx, cam, o, F)) return rc;
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    const int T = lo->tile, Pn = lo->probes;
    const int64_t ntiles = (int64_t)((cam->width + T - 1) / T) * ((cam->height + T - 1) / T);
    const int64_t nprobe = ntiles * Pn;
    ENSURE(ctx->est_mlp, (size_t)F.cap * 12);
    ENSURE(ctx->est_fb, (size_t)F.cap * 12);
    ENSURE(ctx->probe_pos, (size_t)nprobe * 16);
    ENSURE(ctx->probe_nrm, (size_t)nprobe * 16);
    ENSURE(ctx->probe_req, (size_t)nprobe * 4);
    ENSURE(ctx->probe_est, (size_t)nprobe * 12);
    ENSURE(ctx->tile_flag, (size_t)ntiles);
    ENSURE(ctx->learned_counts, 32);   // flagged tiles, fallback requests, gather work counter
    ENSURE(ctx->fallback_list, (size_t)std::max<int64_t>(F.nreq, 1) * 4);
    CK(cudaEventRecord(ctx->ev[6], ctx->st));
    // the cache answers every global request (after training still queued)
    if (int rc = cache_fence(ctx)) return rc;
    MlpInputs in{};
    in.n = F.nreq; in.rec_pos = F.R.a; in.rec_nrm = F.R.b; in.flag_mask = 1u;
    CK(mlp_infer(cache_net(ctx), in, P<float>(ctx->est_mlp), P<unsigned>(ctx->status), ctx->sm_count, ctx->st));
    // exact gathers at the probes (their pixels' primary hits, traced from the
    // camera); tiles whose cache error is too large fall back
    CK(probe_hits(dev_scene(ctx), F.cd, T, Pn, P<float4>(ctx->probe_pos), P<float4>(ctx->probe_nrm), ctx->st));
    GatherQueries PQ{};
    PQ.n = nprobe; PQ.pos4 = P<float4>(ctx->probe_pos); PQ.nrm4 = P<float4>(ctx->probe_nrm); PQ.flag_mask = 1u;
    GatherOut PO{P<float>(ctx->probe_est), nullptr, nullptr, nullptr};
    CK(gather(grid_of(G, G), PQ, o->r_global, o->k_global, 0, PO, P<unsigned>(ctx->status), ctx->st));
    CK(learned_probe_req(F.cd, F.R, T, Pn, P<float4>(ctx->probe_pos), P<float4>(ctx->probe_nrm),
                         P<uint32_t>(ctx->probe_req), P<unsigned>(ctx->status), ctx->st));
    CK(cudaMemsetAsync(ctx->learned_counts.p, 0, 32, ctx->st));
    CK(learned_select(F.cd, F.R, F.nreq, nullptr, T, Pn, P<uint32_t>(ctx->probe_req), P<float>(ctx->probe_est),
                      P<float>(ctx->est_mlp), lo->max_rel_err, lo->noise_z, P<uint8_t>(ctx->tile_flag),
                      P<unsigned long long>(ctx->learned_counts), P<uint32_t>(ctx->fallback_list), ctx->sm_count,
                      ctx->st));
    // the exact gather for the listed fallback requests only (count read on the device)
    GatherQueries Q{};
    Q.n = F.nreq; Q.pos4 = F.R.a; Q.nrm4 = F.R.b; Q.flag_mask = LEARNED_FALLBACK;
    Q.idx = P<uint32_t>(ctx->fallback_list);
    GatherOut OF{P<float>(ctx->est_fb), nullptr, nullptr, nullptr};
    unsigned long long* counts = P<unsigned long long>(ctx->learned_counts);
    CK(gather_listed(grid_of(G, G), Q, counts + 1, counts + 2, o->r_global, o->k_global, OF, ctx->sm_count, ctx->st));
    CK(learned_merge(F.R, F.nreq, nullptr, P<float>(ctx->est_mlp), P<float>(ctx->est_fb), P<float>(ctx->est_g),
                     ctx->sm_count, ctx->st));
    ctx->launches += (F.nreq > 0 ? 1 : 0) + 1 + 1 + 1 + 1 + (F.nreq > 0 ? 1 : 0) + 1 + (F.nreq > 0 ? 1 : 0);
    if (int rc = render_finish(ctx, o, F, out_rgb8, out_radiance)) return rc;
    if (out_stats) {
        unsigned long long cnt[2] = {0, 0};
        CK(cudaMemcpyAsync(cnt, ctx->learned_counts.p, 16, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        out_stats->tiles = ntiles;
        out_stats->fallback_tiles = (int64_t)cnt[0];
        out_stats->requests = F.nreq;
        out_stats->fallback_requests = (int64_t)cnt[1];
    }
    return check_status(ctx, "learned render");
}

int pm_cache_sample_points(pm_ctx* ctx, const pm_camera* cam, int64_t n, uint64_t seed, float* out_pos, float* out_nrm,
                           float* out_weight) {
    if (!ctx || !cam) return PM_ERR_INVALID;
    if (!ctx->has_scene) return fail(ctx, PM_ERR_INVALID, "no scene");
    if (n < 0 || (n > 0 && (!out_pos || !out_nrm || !out_weight))) return fail(ctx, PM_ERR_INVALID, "sample points: bad arguments");
    if (cam->width <= 0 || cam->height <= 0) return fail(ctx, PM_ERR_INVALID, "bad camera size");
    CK(cudaSetDevice(ctx->device));
    CameraDev cd;
    for (int a = 0; a < 3; a++) {
        cd.pos[a] = cam->position[a]; cd.fwd[a] = cam->forward[a]; cd.right[a] = cam->right[a]; cd.up[a] = cam->up[a];
    }
    cd.vw = cam->viewport_w; cd.vh = cam->viewport_h; cd.focal = cam->focal;
    cd.W = cam->width; cd.H = cam->height;
    CK(sample_primary_hits(dev_scene(ctx), cd, n, seed, out_pos, out_nrm, out_weight, ctx->st));
    if (n > 0) ctx->launches += 1;
    return check_status(ctx, "sample points");
}

int pm_scan_u32(pm_ctx* ctx, const uint32_t* in, uint32_t* out, int64_t n, int inclusive) {
    if (!ctx || n < 0 || (n > 0 && (!in || !out))) return PM_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    ENSURE(ctx->gws, scan_workspace_bytes(n));
    CK(scan_u32(in, out, n, inclusive, nullptr, ctx->gws.p, P<unsigned>(ctx->status), ctx->st));
    ctx->launches += 1;
    return check_status(ctx, "scan");
}

int pm_debug_scan_stall(pm_ctx* ctx, const uint32_t* in, uint32_t* out, int64_t n, int64_t spin_limit,
                        int32_t silent_tile) {
    if (!ctx || n <= 0 || !in || !out || spin_limit < 1 || spin_limit > SCAN_SPIN_LIMIT || silent_tile < -1)
        return PM_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    ENSURE(ctx->gws, scan_workspace_bytes(n));
    CK(scan_u32(in, out, n, 1, nullptr, ctx->gws.p, P<unsigned>(ctx->status), ctx->st, (long long)spin_limit,
                silent_tile));
    ctx->launches += 1;
    return check_status(ctx, "scan (stall test)");
}

}  // extern "C"
