// pm_learned_graph.cu -- the learned frame (online training + learned render)
// captured once and replayed as one CUDA graph.
//
// One frame = `steps` Adam steps on consecutive batches of a training pool
// and the learned render of pm_render_learned (eye pass, cache inference,
// exact probes, tile check, listed fallback gather, merge, resolve); the
// training, then the cache inference (once the eye pass is done) run on a
// second stream beside the eye pass and the probe gathers.  Every
// size that the host-driven path reads back between launches lives on the
// device here: the eye pass's request count drives inference, the fallback
// marking, the listed gather and the merge (persistent or grid-stride
// launches over the request capacity); the pool offset and the Adam step
// number advance on the device.  So a frame is one graph launch and one status
// check, with no host round trip inside it.  The graph owns its request and
// estimate buffers; it reads the context's scene, photon map and cache, and
// must be created again after any of those is rebuilt or re-initialised
// (pm_set_scene, pm_set_photons / pm_load_photons, pm_trace_photons,
// pm_build_grid, pm_frame, pm_cache_init): their device addresses, the grid's
// dimensions and the cache's encoding box are part of the captured launches.
// The graph records the context's generation and the addresses and sizes of
// the context buffers its launches read (scene, both maps, cache, status word)
// when it is made; pm_learned_graph_run refuses to launch (PM_ERR_INVALID)
// when either has changed since.
#include <algorithm>
#include <cmath>
#include "pm_context.cuh"
#include "pm_learned.cuh"
#include "pm_mlp.cuh"
#include "pm_render.cuh"

using namespace pm;

struct pm_learned_graph {
    pm_ctx* ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // frame
    CameraDev cd{};
    pm_render_opts ro{};
    pm_learned_opts lo{};
    int64_t npx = 0, cap = 0, ntiles = 0, nprobe = 0;
    uint8_t* out_rgb8 = nullptr;
    float* out_radiance = nullptr;
    // training
    const float* pool_pos = nullptr;
    const float* pool_nrm = nullptr;
    const float* pool_target = nullptr;
    int64_t pool_n = 0, batch = 0;
    int steps = 0;
    bool overlap = false;       // inference reads w16_snap (the cache before this frame's training)
    // device buffers owned by the graph
    DevBuf req_a, req_b, req_c, counter, px_base, px_count, est_mlp, est_fb, est_g;
    DevBuf probe_pos, probe_nrm, probe_req, probe_est, tile_flag, counts, fb_list, state, eye_order, w16_snap;
    int launches_per_frame = 0;
    // the context as the captured launches saw it
    uint64_t generation = 0, buffers = 0;
    // training runs on a second stream beside the eye pass (it needs neither;
    // inference waits for it); the probes' own primary hits and exact gathers
    // run on a third, beside the eye pass's tail
    cudaStream_t side = nullptr, inf = nullptr, probe = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, eye_done = nullptr, inf_done = nullptr, probe_done = nullptr;
};

namespace {

// after a training step: the pool offset past the batch it read (which
// started at 0 where the stored offset would have run past n: the wrap the
// training kernel applies) and the Adam step number the step's update uses
__global__ void k_pool_step(int64_t* off, int64_t n, int64_t b, int* step) {
    int64_t o = *off;
    if (o + b > n) o = 0;
    *off = o + b;
    *step += 1;
}

int64_t* state_offset(pm_learned_graph* g) { return P<int64_t>(g->state); }
int* state_step(pm_learned_graph* g) { return reinterpret_cast<int*>(P<int64_t>(g->state) + 1); }

Requests requests_of(pm_learned_graph* g) {
    Requests R;
    R.a = P<float4>(g->req_a); R.b = P<float4>(g->req_b); R.c = P<float4>(g->req_c);
    R.cap = g->cap;
    R.counter = P<unsigned long long>(g->counter);
    R.px_base = P<uint32_t>(g->px_base);
    R.px_count = P<uint32_t>(g->px_count);
    return R;
}

// the context buffers the captured launches read
uint64_t read_set(pm_ctx* ctx) {
    std::vector<DevBuf*> v = {&ctx->tri, &ctx->tri_pos, &ctx->tri_nrm, &ctx->tri_diffuse, &ctx->nodes, &ctx->prim,
                              &ctx->maabb, &ctx->mats, &ctx->ca, &ctx->tri_leaf, &ctx->status, &ctx->cache_w32,
                              &ctx->cache_w16, &ctx->cache_m, &ctx->cache_v, &ctx->cache_grad, &ctx->cache_loss};
    for (auto& m : ctx->maps)
        for (DevBuf* b : {&m.pos, &m.dir, &m.pow, &m.starts, &m.sizes, &m.gpos, &m.gdir, &m.gpow, &m.cid, &m.keys0,
                          &m.keys1, &m.vals0, &m.vals1, &m.hist, &m.scan_ws, &m.small, &m.key_counts,
                          &m.key_starts, &m.counts2})
            v.push_back(b);
    return buffer_fingerprint(v);
}

// every launch of one frame, on ctx->st (captured or eager)
int enqueue_frame(pm_learned_graph* g) {
    pm_ctx* ctx = g->ctx;
    const cudaStream_t main_st = ctx->st;
    unsigned* status = P<unsigned>(ctx->status);
    const MlpNet net = cache_net(ctx);
    MlpNet net_infer = net;
    const pm_cache_opts& co = ctx->cache_opts;
    int launches = 0;
    if (g->overlap) {   // the cache as the previous frames trained it, for this frame's inference
        CK(cudaMemcpyAsync(g->w16_snap.p, ctx->cache_w16.p, (size_t)PM_CACHE_PARAMS * 2, cudaMemcpyDeviceToDevice,
                           main_st));
        net_infer.w = P<__nv_bfloat16>(g->w16_snap);
    }
    // online training on the pool, on the side stream: the eye pass leaves
    // most SMs idle while its slowest pixels finish, and training fills them
    CK(cudaEventRecord(g->fork, main_st));
    CK(cudaStreamWaitEvent(g->side, g->fork, 0));
    // the probes: their pixels' primary hits traced from the camera and
    // gathered exactly, on their own stream beside the eye pass
    {
        const DevScene S = dev_scene(ctx);
        MapState& G = ctx->maps[PM_MAP_GLOBAL];
        CK(cudaStreamWaitEvent(g->probe, g->fork, 0));
        CK(probe_hits(S, g->cd, g->lo.tile, g->lo.probes, P<float4>(g->probe_pos), P<float4>(g->probe_nrm), g->probe));
        GatherQueries PQ{};
        PQ.n = g->nprobe;
        PQ.pos4 = P<float4>(g->probe_pos);
        PQ.nrm4 = P<float4>(g->probe_nrm);
        PQ.flag_mask = 1u;
        GatherOut PO{P<float>(g->probe_est), nullptr, nullptr, nullptr};
        CK(gather(grid_of(G, G), PQ, g->ro.r_global, g->ro.k_global, 0, PO, status, g->probe));
        CK(cudaEventRecord(g->probe_done, g->probe));
        launches += 2;
    }
    cudaStream_t st = g->side;
    if (g->steps > 0) {
        // the gradient starts at zero (each Adam step zeroes it after use); the
        // loss is not read back by a replayed frame
        CK(cudaMemsetAsync(ctx->cache_grad.p, 0, (size_t)PM_CACHE_PARAMS * 4, st));
        CK(cudaMemsetAsync(ctx->cache_loss.p, 0, 4, st));
    }
    for (int s = 0; s < g->steps; s++) {
        MlpInputs in{};
        in.n = g->batch;
        in.pos3 = g->pool_pos;
        in.nrm3 = g->pool_nrm;
        in.base_dev = state_offset(g);
        in.base_wrap = g->pool_n;
        CK(mlp_train(net, in, g->pool_target, nullptr, 2.f / (3.f * (float)g->batch), P<float>(ctx->cache_grad),
                     P<float>(ctx->cache_loss), status, ctx->sm_count, st));
        k_pool_step<<<1, 1, 0, st>>>(state_offset(g), g->pool_n, g->batch, state_step(g));
        CK(cudaGetLastError());
        CK(mlp_adam_dev(P<float>(ctx->cache_w32), P<__nv_bfloat16>(ctx->cache_w16), P<float>(ctx->cache_grad),
                        P<float>(ctx->cache_m), P<float>(ctx->cache_v), state_step(g), co.lr, co.beta1, co.beta2,
                        co.eps, st, false));
        launches += 3;
    }
    // the learned render: eye pass, then the probe gathers here while the side
    // stream (after its training) answers every request with the cache
    st = main_st;
    const DevScene S = dev_scene(ctx);
    MapState& G = ctx->maps[PM_MAP_GLOBAL];
    const Requests R = requests_of(g);
    CK(eye_pass(S, g->cd, g->ro.max_depth, R, status, st, P<int>(g->eye_order)));
    CK(cudaEventRecord(g->eye_done, st));
    // inference: after the training on the side stream, or (overlap) on its
    // own stream with the frame-start copy while the training goes on
    const cudaStream_t ist = g->overlap ? g->inf : g->side;
    CK(cudaStreamWaitEvent(ist, g->eye_done, 0));
    MlpInputs in{};
    in.n = g->cap;
    in.rec_pos = R.a;
    in.rec_nrm = R.b;
    in.flag_mask = 1u;
    in.n_dev = R.counter;
    CK(mlp_infer(net_infer, in, P<float>(g->est_mlp), status, ctx->sm_count, ist));
    CK(cudaEventRecord(g->overlap ? g->inf_done : g->join, ist));
    if (g->overlap) CK(cudaEventRecord(g->join, g->side));   // the training, joined at the frame's end
    const int T = g->lo.tile, Pn = g->lo.probes;
    CK(cudaStreamWaitEvent(st, g->probe_done, 0));   // the probes' records and exact estimates
    CK(learned_probe_req(g->cd, R, T, Pn, P<float4>(g->probe_pos), P<float4>(g->probe_nrm), P<uint32_t>(g->probe_req),
                         status, st));
    CK(cudaStreamWaitEvent(st, g->overlap ? g->inf_done : g->join, 0));   // the cache's answers
    unsigned long long* counts = P<unsigned long long>(g->counts);
    CK(cudaMemsetAsync(counts, 0, 32, st));
    CK(learned_select(g->cd, R, g->cap, R.counter, T, Pn, P<uint32_t>(g->probe_req), P<float>(g->probe_est),
                      P<float>(g->est_mlp), g->lo.max_rel_err, g->lo.noise_z, P<uint8_t>(g->tile_flag), counts,
                      P<uint32_t>(g->fb_list), ctx->sm_count, st));
    GatherQueries Q{};
    Q.n = g->cap;
    Q.pos4 = R.a;
    Q.nrm4 = R.b;
    Q.flag_mask = LEARNED_FALLBACK;
    Q.idx = P<uint32_t>(g->fb_list);
    GatherOut OF{P<float>(g->est_fb), nullptr, nullptr, nullptr};
    CK(gather_listed(grid_of(G, G), Q, counts + 1, counts + 2, g->ro.r_global, g->ro.k_global, OF, ctx->sm_count, st));
    CK(learned_merge(R, g->cap, R.counter, P<float>(g->est_mlp), P<float>(g->est_fb), P<float>(g->est_g), ctx->sm_count,
                     st));
    const float tone_t = (float)std::pow((double)0.6f, -1);
    CK(resolve(S, g->cd, R, P<float>(g->est_g), nullptr, tone_t, g->out_rgb8, g->out_radiance, st));
    if (g->overlap) CK(cudaStreamWaitEvent(st, g->join, 0));   // the next frame's copy sees this frame's training
    launches += 9;   // eye, inference, probe requests, counts reset, tile flags, marks, fallback gather, merge, resolve
    g->launches_per_frame = launches;
    return PM_OK;
}

void free_graph(pm_learned_graph* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->fork) cudaEventDestroy(g->fork);
    if (g->join) cudaEventDestroy(g->join);
    if (g->eye_done) cudaEventDestroy(g->eye_done);
    if (g->inf_done) cudaEventDestroy(g->inf_done);
    if (g->probe_done) cudaEventDestroy(g->probe_done);
    if (g->probe) cudaStreamDestroy(g->probe);
    if (g->side) cudaStreamDestroy(g->side);
    if (g->inf) cudaStreamDestroy(g->inf);
    DevBuf* bufs[] = {&g->req_a, &g->req_b, &g->req_c, &g->counter, &g->px_base, &g->px_count, &g->est_mlp, &g->est_fb,
                      &g->est_g, &g->probe_pos, &g->probe_nrm, &g->probe_req, &g->probe_est, &g->tile_flag,
                      &g->counts, &g->fb_list, &g->state, &g->eye_order, &g->w16_snap};
    for (DevBuf* b : bufs) release(*b);
    delete g;
}

// the context's FP32 weights, BF16 copies and Adam moments (saved around the warm-up frame)
struct CacheSnapshot {
    DevBuf w32, w16, m, v;
};

}  // namespace

extern "C" {

int pm_learned_graph_create(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* o, const pm_learned_opts* lo,
                            const float* pool_pos, const float* pool_nrm, const float* pool_target, int64_t pool_n,
                            int64_t batch, int32_t steps, int64_t pool_offset, int32_t overlap_training,
                            uint8_t* out_rgb8, float* out_radiance, pm_learned_graph** out) {
    if (!ctx || !cam || !o || !lo || !out_rgb8 || !out) return PM_ERR_INVALID;
    *out = nullptr;
    if (int rc = learned_checks(ctx, lo)) return rc;
    if (int rc = render_checks(ctx, cam, o)) return rc;
    if (ctx->maps[PM_MAP_CAUSTIC].built && o->k_caustic > 0)
        return fail(ctx, PM_ERR_INVALID, "learned graph: the caustic estimate is not part of the graph (k_caustic 0)");
    if (steps < 0 || (steps > 0 && (!pool_pos || !pool_nrm || !pool_target || pool_n <= 0 || batch <= 0)))
        return fail(ctx, PM_ERR_INVALID, "learned graph: steps >= 0; with steps, a pool (n > 0) and batch > 0");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    pm_learned_graph* g = new pm_learned_graph();
    g->ctx = ctx;
    g->ro = *o;
    g->lo = *lo;
    for (int a = 0; a < 3; a++) {
        g->cd.pos[a] = cam->position[a]; g->cd.fwd[a] = cam->forward[a]; g->cd.right[a] = cam->right[a];
        g->cd.up[a] = cam->up[a];
    }
    g->cd.vw = cam->viewport_w; g->cd.vh = cam->viewport_h; g->cd.focal = cam->focal;
    g->cd.W = cam->width; g->cd.H = cam->height;
    g->npx = (int64_t)cam->width * cam->height;
    g->cap = g->npx * (((int64_t)1 << std::max(o->max_depth, 1)) - 1);
    g->ntiles = (int64_t)((cam->width + lo->tile - 1) / lo->tile) * ((cam->height + lo->tile - 1) / lo->tile);
    g->nprobe = g->ntiles * lo->probes;
    g->out_rgb8 = out_rgb8;
    g->out_radiance = out_radiance;
    g->pool_pos = pool_pos; g->pool_nrm = pool_nrm; g->pool_target = pool_target;
    g->pool_n = pool_n;
    g->batch = std::min(batch, std::max<int64_t>(pool_n, 1));
    g->steps = steps;
    g->overlap = overlap_training != 0;
    auto bail = [&](int rc) { free_graph(g); return rc; };
    auto need = [&](DevBuf& b, size_t bytes) { return ensure(b, std::max<size_t>(bytes, 16)); };
    cudaError_t e = cudaSuccess;
    const struct { DevBuf* b; size_t bytes; } allocs[] = {
        {&g->req_a, (size_t)g->cap * 16}, {&g->req_b, (size_t)g->cap * 16}, {&g->req_c, (size_t)g->cap * 16},
        {&g->counter, 8}, {&g->px_base, (size_t)g->npx * 4}, {&g->px_count, (size_t)g->npx * 4},
        {&g->est_mlp, (size_t)g->cap * 12}, {&g->est_fb, (size_t)g->cap * 12}, {&g->est_g, (size_t)g->cap * 12},
        {&g->probe_pos, (size_t)g->nprobe * 16}, {&g->probe_nrm, (size_t)g->nprobe * 16},
        {&g->probe_req, (size_t)g->nprobe * 4}, {&g->probe_est, (size_t)g->nprobe * 12},
        {&g->tile_flag, (size_t)g->ntiles}, {&g->counts, 32}, {&g->fb_list, (size_t)g->cap * 4}, {&g->state, 16},
        {&g->w16_snap, (size_t)PM_CACHE_PARAMS * 2}};
    for (const auto& a : allocs)
        if ((e = need(*a.b, a.bytes)) != cudaSuccess) return bail(cuda_fail(ctx, e, "learned graph buffers"));
    if ((e = cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&g->inf, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&g->probe, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g->probe_done, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g->inf_done, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g->join, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g->eye_done, cudaEventDisableTiming)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "learned graph streams"));
    // the eye pass's block order (slow blocks first), fixed with the camera
    std::vector<int> order;
    eye_block_order(ctx, cam, order);
    if ((e = need(g->eye_order, order.size() * 4)) != cudaSuccess ||
        (e = cudaMemcpyAsync(g->eye_order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, ctx->st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->st)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "learned graph eye order"));
    // training state: the pool offset and the Adam step number
    const int64_t st_host[2] = {std::max<int64_t>(pool_offset, 0), 0};
    if ((e = cudaMemcpyAsync(g->state.p, st_host, 16, cudaMemcpyHostToDevice, ctx->st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(state_step(g), &ctx->cache_step, 4, cudaMemcpyHostToDevice, ctx->st)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "learned graph state"));
    // one eager frame loads every kernel before the capture; the cache is
    // restored afterwards, so creating the graph leaves the weights as they were
    CacheSnapshot snap;
    DevBuf* src[] = {&ctx->cache_w32, &ctx->cache_w16, &ctx->cache_m, &ctx->cache_v};
    DevBuf* dst[] = {&snap.w32, &snap.w16, &snap.m, &snap.v};
    auto drop_snapshot = [&]() { for (DevBuf* b : dst) release(*b); };
    for (int i = 0; i < 4; i++) {
        if ((e = ensure(*dst[i], src[i]->bytes)) != cudaSuccess ||
            (e = cudaMemcpyAsync(dst[i]->p, src[i]->p, src[i]->bytes, cudaMemcpyDeviceToDevice, ctx->st)) != cudaSuccess) {
            drop_snapshot();
            return bail(cuda_fail(ctx, e, "learned graph cache snapshot"));
        }
    }
    int rc = enqueue_frame(g);
    if (rc == PM_OK) rc = check_status(ctx, "learned graph warm-up frame");
    for (int i = 0; i < 4 && rc == PM_OK; i++)
        if ((e = cudaMemcpyAsync(src[i]->p, dst[i]->p, src[i]->bytes, cudaMemcpyDeviceToDevice, ctx->st)) != cudaSuccess)
            rc = cuda_fail(ctx, e, "learned graph cache restore");
    if (rc == PM_OK &&
        ((e = cudaMemcpyAsync(g->state.p, st_host, 16, cudaMemcpyHostToDevice, ctx->st)) != cudaSuccess ||
         (e = cudaStreamSynchronize(ctx->st)) != cudaSuccess))
        rc = cuda_fail(ctx, e, "learned graph state");
    drop_snapshot();
    if (rc != PM_OK) return bail(rc);
    // capture
    if ((e = cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "learned graph: begin capture (the context's stream must not be the legacy default stream)"));
    rc = enqueue_frame(g);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(ctx->st, &graph);
    g->graph = graph;
    if (rc != PM_OK) return bail(rc);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "learned graph: end capture"));
    if ((e = cudaGraphInstantiate(&g->exec, g->graph, 0)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "learned graph: instantiate"));
    g->generation = ctx->generation;
    g->buffers = read_set(ctx);
    *out = g;
    return PM_OK;
}

int pm_learned_graph_run(pm_learned_graph* g, pm_learned_stats* out_stats) {
    if (!g) return PM_ERR_INVALID;
    pm_ctx* ctx = g->ctx;
    if (g->generation != ctx->generation || g->buffers != read_set(ctx))
        return fail(ctx, PM_ERR_INVALID, "learned graph: the scene, a photon map or the cache was rebuilt or "
                                         "re-initialised since the graph was made; make it again");
    CK(cudaSetDevice(ctx->device));
    if (int rc = cache_fence(ctx)) return rc;
    // the step number follows the context's (training calls between frames count too)
    CK(cudaMemcpyAsync(state_step(g), &ctx->cache_step, 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaGraphLaunch(g->exec, ctx->st));
    ctx->launches += g->launches_per_frame;
    ctx->cache_step += g->steps;
    if (int rc = check_status(ctx, "learned graph frame")) return rc;
    if (out_stats) {
        unsigned long long cnt[2] = {0, 0}, nreq = 0;
        CK(cudaMemcpyAsync(cnt, g->counts.p, 16, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(&nreq, g->counter.p, 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        out_stats->tiles = g->ntiles;
        out_stats->fallback_tiles = (int64_t)cnt[0];
        out_stats->requests = (int64_t)std::min<unsigned long long>(nreq, (unsigned long long)g->cap);
        out_stats->fallback_requests = (int64_t)cnt[1];
    }
    return PM_OK;
}

int pm_learned_graph_offset(pm_learned_graph* g, int64_t* out_offset) {
    if (!g || !out_offset) return PM_ERR_INVALID;
    pm_ctx* ctx = g->ctx;
    CK(cudaMemcpyAsync(out_offset, state_offset(g), 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return PM_OK;
}

void pm_learned_graph_destroy(pm_learned_graph* g) {
    if (!g) return;
    cudaSetDevice(g->ctx->device);
    free_graph(g);
}

}  // extern "C"
