// pm_batch.cu -- the batched form: many scene instances per frame, one work
// queue per stage, the frame captured once into a CUDA graph.
//
// Per frame (no host round trip):
//   trace_multi     one persistent launch over the concatenated path ranges of
//                   all instances (each lane takes the next path, looks up its
//                   instance, traces it in that instance's scene and stream);
//                   one scan; one canonical-order compaction into per-instance
//                   photon slots cut at each capacity
//   grid_multi      one key space over all instances (instance key base + the
//                   sub-cell key in the instance's grid), one count, one scan,
//                   one stable radix sort, one record gather
//   eye_pass_multi  one launch over all pixels of all instances
//   gather_multi    persistent warps over one request queue (the request count
//                   stays on the device), each request answered with its
//                   instance's grid, k and radius
//   resolve_multi   one launch over all pixels
//
// Everything that needs the host is decided at creation: the paths each
// instance traces (a single-instance calibration trace of the same streams,
// plus a margin), each instance's grid (cell size, dims, sub-cell split; the
// reference's sizing, or the autotuner's choice), buffer sizes, block shapes.
// The autotuner times candidate frames: grid sizing (photons per cell),
// gather block shape (warps per block) and the tracer's lane-refill
// threshold, each stage on its own.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "pm_context.cuh"
#include "pm_gather.cuh"
#include "pm_grid.cuh"
#include "pm_render.cuh"
#include "pm_scan.cuh"
#include "pm_trace.cuh"

using namespace pm;

struct pm_batch {
    int device = 0;
    cudaStream_t st = nullptr;
    std::string err;
    int sm_count = 148;
    int n = 0;
    std::vector<pm_ctx*> ctx;                 // one per instance: scene, calibration, grid plans
    std::vector<pm_batch_instance> inst;
    std::vector<int64_t> paths, path_off, ph_off, key_off, cell_off, px_off;
    std::vector<TraceInst> trace_host;
    int64_t total_paths = 0, total_slots = 0, total_keys = 0, total_cells = 0, total_px = 0, req_cap = 0;
    int64_t req_split = 0;    // requests of gather class 0 in [0, req_split), class 1 in [req_split, req_cap)
    int max_bounces = 1;
    // device tables
    DevBuf t_trace, t_outs, t_path_off, t_grid, t_ph_off, t_cell_off, t_render, t_px_off, t_gather;
    // trace
    DevBuf counter, stage, cnt_g, cnt_c, scan_g, totals, trace_ws, inst_total;
    DevBuf pos, dir, pow;
    // grid
    DevBuf cid, keys0, keys1, vals0, vals1, hist, grid_ws, key_counts, key_starts, cstarts, csizes, gpos, gdir, gpow;
    // render
    DevBuf req_a, req_b, req_c, req_counter, px_base, px_count, est_g, queues, rgb8, status;
    // choices
    int desired = 1000, gather_warps = 8, refill = 8;
    float guess = GATHER_GUESS;   // the gather walk's first-ring guess (photons within it, in units of k)
    float khint = 0.f;            // sub-cell split: 0 = the library default (sized for k 64), else the
                                  // automatic rule for khint x the instance's k
    // graph
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t seeded_frame = 0;
    float ms_last = 0.f;
    int64_t photons_last = 0, requests_last = 0;
    std::vector<int64_t> stored_last;   // photons each instance stored in the last frame
    int underfilled = 0;
    float stage_ms[5] = {0, 0, 0, 0, 0};
};

namespace {

int bfail(pm_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

#define BCK(expr)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (expr);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? PM_ERR_OOM : PM_ERR_CUDA,            \
                         std::string(#expr) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

template <class T>
cudaError_t upload(DevBuf& d, const std::vector<T>& h, cudaStream_t st) {
    cudaError_t e = ensure(d, std::max<size_t>(h.size() * sizeof(T), 16));
    if (e != cudaSuccess || h.empty()) return e;
    e = cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

std::vector<int64_t> offsets(const std::vector<int64_t>& sizes) {
    std::vector<int64_t> o(sizes.size() + 1, 0);
    for (size_t i = 0; i < sizes.size(); i++) o[i + 1] = o[i] + sizes[i];
    return o;
}

// Per-instance grids for the given sizing, from each instance's calibration
// map (pm_build_grid on the instance context: the reference's re-grid rule and
// the automatic sub-cell split), and the tables that depend on them.
int plan_grids(pm_batch* b, int desired) {
    std::vector<GridInstDev> g((size_t)b->n);
    std::vector<int64_t> keys((size_t)b->n), cells((size_t)b->n);
    for (int i = 0; i < b->n; i++) {
        pm_ctx* c = b->ctx[(size_t)i];
        const int kh = b->khint > 0.f ? std::max(1, (int)std::lround(b->khint * (float)b->inst[(size_t)i].k)) : 0;
        pm_grid_opts go = {desired, 5, 5, 0, kh};
        if (int rc = pm_build_grid(c, PM_MAP_GLOBAL, &go, nullptr)) return bfail(b, rc, pm_last_error(c));
        const MapState& m = c->maps[PM_MAP_GLOBAL];
        GridInstDev& t = g[(size_t)i];
        for (int a = 0; a < 3; a++) t.mn[a] = m.aabb[a];
        t.gx = m.dims[0]; t.gy = m.dims[1]; t.gz = m.dims[2];
        t.cell = m.cell;
        t.S = m.S;
        cells[(size_t)i] = m.cells;
        keys[(size_t)i] = m.cells * (int64_t)m.S * m.S * m.S;
    }
    b->key_off = offsets(keys);
    b->cell_off = offsets(cells);
    b->total_keys = b->key_off.back();
    b->total_cells = b->cell_off.back();
    if (b->total_keys + 2 >= ((int64_t)1 << 32)) return bfail(b, PM_ERR_INVALID, "batch: too many sub-cells");
    for (int i = 0; i < b->n; i++) {
        GridInstDev& t = g[(size_t)i];
        t.key0 = b->key_off[(size_t)i];
        t.cell0 = b->cell_off[(size_t)i];
        t.ph0 = b->ph_off[(size_t)i];
        t.cap = b->inst[(size_t)i].photons;
    }
    BCK(upload(b->t_grid, g, b->st));
    BCK(upload(b->t_cell_off, b->cell_off, b->st));
    BCK(ensure(b->key_counts, (size_t)(b->total_keys + 1) * 4));
    BCK(ensure(b->key_starts, (size_t)(b->total_keys + 2) * 4));
    BCK(ensure(b->cstarts, (size_t)std::max<int64_t>(b->total_cells, 1) * 4));
    BCK(ensure(b->csizes, (size_t)std::max<int64_t>(b->total_cells, 1) * 4));
    size_t hist_elems = 0, ws = 0;
    grid_scratch_sizes(b->total_slots, b->total_keys + 1, &hist_elems, &ws);
    BCK(ensure(b->hist, hist_elems * 4));
    BCK(ensure(b->grid_ws, ws));
    // gather table: each instance's view of the shared sorted arrays
    std::vector<GatherInstDev> gt((size_t)b->n);
    for (int i = 0; i < b->n; i++) {
        GatherInstDev& t = gt[(size_t)i];
        const GridInstDev& q = g[(size_t)i];
        t.G.gpos = P<float4>(b->gpos);
        t.G.gdir = P<float>(b->gdir);
        t.G.gpow = P<float>(b->gpow);
        t.G.key_starts = P<uint32_t>(b->key_starts) + q.key0;
        for (int a = 0; a < 3; a++) t.G.mn[a] = q.mn[a];
        t.G.gx = q.gx; t.G.gy = q.gy; t.G.gz = q.gz;
        t.G.cell = q.cell;
        t.G.S = q.S;
        t.G.guess = b->guess;
        t.r = b->inst[(size_t)i].radius;
        t.k = b->inst[(size_t)i].k;
        t.cls = gather_class(t.k);
    }
    BCK(upload(b->t_gather, gt, b->st));
    b->desired = desired;
    return PM_OK;
}

TraceMulti trace_args(pm_batch* b) {
    TraceMulti M{};
    M.ninst = b->n;
    M.total = b->total_paths;
    M.path_off = P<int64_t>(b->t_path_off);
    M.table = b->t_trace.p;
    M.outs = P<TraceInstOut>(b->t_outs);
    M.path_counter = P<unsigned long long>(b->counter);
    M.stage = P<float4>(b->stage);
    M.cnt_g = P<uint32_t>(b->cnt_g);
    M.cnt_c = P<uint32_t>(b->cnt_c);
    M.scan_g = P<uint32_t>(b->scan_g);
    M.totals = P<uint32_t>(b->totals);
    M.scan_ws = b->trace_ws.p;
    M.pos = P<float>(b->pos);
    M.dir = P<float>(b->dir);
    M.pow = P<float>(b->pow);
    M.inst_total = P<int64_t>(b->inst_total);
    M.status = P<unsigned>(b->status);
    M.sm_count = b->sm_count;
    M.refill = b->refill;
    return M;
}

// per-frame photon seeds in the trace table
int seed_frame(pm_batch* b, uint64_t frame) {
    for (int i = 0; i < b->n; i++) b->trace_host[(size_t)i].seed = b->inst[(size_t)i].seed + frame;
    const TraceMulti M = trace_args(b);
    BCK(trace_multi_tables(M, b->trace_host.data(), b->st));
    b->seeded_frame = frame;
    return PM_OK;
}

Requests request_args(pm_batch* b) {
    Requests R;
    R.a = P<float4>(b->req_a);
    R.b = P<float4>(b->req_b);
    R.c = P<float4>(b->req_c);
    R.cap = b->req_cap;
    R.counter = P<unsigned long long>(b->req_counter);
    R.px_base = P<uint32_t>(b->px_base);
    R.px_count = P<uint32_t>(b->px_count);
    return R;
}

// The stages of one frame on b->st; stage < 0: all, else only that stage
// (0 trace, 1 grid, 2 eye, 3 gather, 4 resolve), for the autotuner.
int launch_stages(pm_batch* b, int stage, int* launches) {
    int L = 0;
    if (stage < 0 || stage == 0) {
        const TraceMulti M = trace_args(b);
        BCK(trace_multi(M, b->st));
        L += 3;
    }
    if (stage < 0 || stage == 1) {
        GridBuffers B{};
        B.pos = P<float>(b->pos); B.dir = P<float>(b->dir); B.pow = P<float>(b->pow);
        B.n = b->total_slots;
        B.cell_starts = P<uint32_t>(b->cstarts); B.cell_sizes = P<uint32_t>(b->csizes);
        B.gpos = P<float4>(b->gpos); B.gdir = P<float>(b->gdir); B.gpow = P<float>(b->gpow);
        B.key_counts = P<uint32_t>(b->key_counts); B.key_starts = P<uint32_t>(b->key_starts);
        B.cid = P<uint32_t>(b->cid);
        B.keys[0] = P<uint32_t>(b->keys0); B.keys[1] = P<uint32_t>(b->keys1);
        B.vals[0] = P<uint32_t>(b->vals0); B.vals[1] = P<uint32_t>(b->vals1);
        B.hist = P<uint32_t>(b->hist);
        B.scan_ws = b->grid_ws.p;
        B.status = P<unsigned>(b->status);
        GridMulti G{};
        G.ninst = b->n;
        G.tab = P<GridInstDev>(b->t_grid);
        G.ph_off = P<int64_t>(b->t_ph_off);
        G.cell_off = P<int64_t>(b->t_cell_off);
        G.filled = P<int64_t>(b->inst_total);
        G.total_keys = b->total_keys;
        G.total_cells = b->total_cells;
        BCK(grid_multi(B, G, &L, b->st));
    }
    Requests R = request_args(b);
    if (stage < 0 || stage == 2) {
        BCK(eye_pass_multi(P<RenderInstDev>(b->t_render), P<int64_t>(b->t_px_off), b->n, b->total_px, R,
                           b->req_split, P<unsigned>(b->status), b->st));
        L += 1;
    }
    if (stage < 0 || stage == 3) {
        GatherQueries Q{};
        Q.n = b->req_cap; Q.pos4 = R.a; Q.nrm4 = R.b; Q.flag_mask = 1u;
        GatherOut O{P<float>(b->est_g), nullptr, nullptr, nullptr};
        BCK(gather_multi(P<GatherInstDev>(b->t_gather), P<int64_t>(b->t_px_off), b->n, Q, R.c, R.counter,
                         b->req_split, P<unsigned long long>(b->queues), O, b->gather_warps, b->sm_count, b->st));
        L += (b->req_split > 0 ? 1 : 0) + (b->req_split < b->req_cap ? 1 : 0);
    }
    if (stage < 0 || stage == 4) {
        const float tone_t = (float)std::pow((double)0.6f, -1);
        BCK(resolve_multi(P<RenderInstDev>(b->t_render), P<int64_t>(b->t_px_off), b->n, b->total_px, R,
                          P<float>(b->est_g), tone_t, P<uint8_t>(b->rgb8), nullptr, b->st));
        L += 1;
    }
    if (launches) *launches = L;
    return PM_OK;
}

int check_batch_status(pm_batch* b) {
    uint32_t bits = 0;
    BCK(cudaMemcpyAsync(&bits, b->status.p, 4, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    if (bits) {
        BCK(cudaMemsetAsync(b->status.p, 0, 4, b->st));
        char buf[128];
        snprintf(buf, sizeof buf, "batch frame: device status 0x%x (1 timeout, 2 overflow, 4 stack, 8 bad input)", bits);
        return bfail(b, (bits & ST_TIMEOUT) ? PM_ERR_TIMEOUT : PM_ERR_OVERFLOW, buf);
    }
    return PM_OK;
}

// device time of one stage (eager) averaged over reps, after a warm-up
int time_stage(pm_batch* b, int stage, int reps, float* ms) {
    if (int rc = launch_stages(b, stage, nullptr)) return rc;
    BCK(cudaEventRecord(b->ev0, b->st));
    for (int r = 0; r < reps; r++)
        if (int rc = launch_stages(b, stage, nullptr)) return rc;
    BCK(cudaEventRecord(b->ev1, b->st));
    BCK(cudaEventSynchronize(b->ev1));
    *ms = elapsed(b->ev0, b->ev1) / (float)reps;
    return check_batch_status(b);
}

// Times each stage's candidates on frame 0 and keeps the fastest: the
// tracer's refill threshold; the grid sizing together with the gather block
// shape (grid build + eye pass + gather of that grid); the sub-cell split (the
// library default, or the automatic rule for 1/4, 1 or 4 x each instance's
// own k: one power of two finer, the rule's, one coarser); then the gather
// walk's first-ring guess (no guess, or a bound expected to hold 1.5, 2 or
// 3 x k photons) on the chosen grid.  No candidate changes an answer.
int autotune(pm_batch* b) {
    if (int rc = launch_stages(b, -1, nullptr)) return rc;   // one full frame fills every stage's inputs
    BCK(cudaStreamSynchronize(b->st));
    float best = 1e30f, ms = 0.f;
    int best_refill = b->refill;
    for (int refill : {4, 8, 16}) {
        b->refill = refill;
        if (int rc = time_stage(b, 0, 2, &ms)) return rc;
        if (ms < best) { best = ms; best_refill = refill; }
    }
    b->refill = best_refill;
    if (int rc = launch_stages(b, 0, nullptr)) return rc;   // frame 0's photons for the grid candidates
    best = 1e30f;
    int best_desired = b->desired, best_warps = b->gather_warps;
    for (int desired : {125, 250, 500, 1000, 2000}) {
        if (int rc = plan_grids(b, desired)) return rc;
        for (int warps : {4, 8}) {
            b->gather_warps = warps;
            float tg = 0.f, te = 0.f, tq = 0.f;
            if (int rc = time_stage(b, 1, 1, &tg)) return rc;
            if (int rc = time_stage(b, 2, 1, &te)) return rc;
            if (int rc = time_stage(b, 3, 2, &tq)) return rc;
            if (tg + tq < best) { best = tg + tq; best_desired = desired; best_warps = warps; }
        }
    }
    b->gather_warps = best_warps;
    float best_khint = b->khint;
    best = 1e30f;
    for (float kh : {0.f, 0.25f, 1.f, 4.f}) {
        b->khint = kh;
        if (int rc = plan_grids(b, best_desired)) return rc;
        float tg = 0.f, te = 0.f, tq = 0.f;
        if (int rc = time_stage(b, 1, 1, &tg)) return rc;
        if (int rc = time_stage(b, 2, 1, &te)) return rc;
        if (int rc = time_stage(b, 3, 2, &tq)) return rc;
        if (tg + tq < best) { best = tg + tq; best_khint = kh; }
    }
    b->khint = best_khint;
    float best_guess = b->guess;
    best = 1e30f;
    for (float guess : {0.f, 1.5f, 2.f, 3.f}) {
        b->guess = guess;
        if (int rc = plan_grids(b, best_desired)) return rc;
        float tg = 0.f, te = 0.f, tq = 0.f;
        if (int rc = time_stage(b, 1, 1, &tg)) return rc;
        if (int rc = time_stage(b, 2, 1, &te)) return rc;
        if (int rc = time_stage(b, 3, 2, &tq)) return rc;
        if (tq < best) { best = tq; best_guess = guess; }
    }
    b->guess = best_guess;
    return plan_grids(b, best_desired);
}

int capture(pm_batch* b) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    const int rc = launch_stages(b, -1, &launches);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    BCK(e);
    b->graph = g;
    BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->launches = launches;
    return PM_OK;
}

int create(pm_batch* b, const pm_batch_instance* in, int32_t n, const pm_batch_opts* opts) {
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    BCK(cudaEventCreate(&b->ev0));
    BCK(cudaEventCreate(&b->ev1));
    cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device);
    b->n = n;
    b->inst.assign(in, in + n);
    std::vector<int64_t> npx((size_t)n), caps((size_t)n), req((size_t)n);
    b->paths.assign((size_t)n, 0);
    b->trace_host.resize((size_t)n);
    std::vector<TraceInstOut> outs((size_t)n);
    std::vector<RenderInstDev> rt((size_t)n);
    for (int i = 0; i < n; i++) {
        const pm_batch_instance& I = in[i];
        if (!I.scene || I.photons <= 0 || I.max_bounces < 1 || I.max_bounces > 32 || I.k < 1 || I.k > 256 ||
            !(I.radius > 0.f) || I.max_depth < 0 || I.max_depth > RENDER_MAX_DEPTH || I.camera.width <= 0 ||
            I.camera.height <= 0)
            return bfail(b, PM_ERR_INVALID, "batch: instance " + std::to_string(i) + " has invalid parameters");
        pm_ctx* c = nullptr;
        pm_device_opts d = {b->device, (void*)b->st};
        if (int rc = pm_create(&c, &d)) return bfail(b, rc, "batch: context creation failed");
        b->ctx.push_back(c);
        if (int rc = pm_set_scene(c, I.scene)) return bfail(b, rc, std::string("batch: ") + pm_last_error(c));
        // calibration: the instance's own streams, traced single-instance, fix its path count
        pm_trace_opts to = {};
        to.seed = I.seed; to.stream_tag = 0; to.max_bounces = I.max_bounces;
        to.global_capacity = I.photons; to.caustic_capacity = 0; to.max_paths = 0;
        int64_t used = 0;
        if (int rc = pm_trace_photons(c, &to, &used)) return bfail(b, rc, std::string("batch: ") + pm_last_error(c));
        b->paths[(size_t)i] = used + used / 50 + 256;   // margin for other frames' streams
        caps[(size_t)i] = I.photons;
        npx[(size_t)i] = (int64_t)I.camera.width * I.camera.height;
        req[(size_t)i] = npx[(size_t)i] * (((int64_t)1 << std::max(I.max_depth, 1)) - 1);
        TraceInst& T = b->trace_host[(size_t)i];
        T.S = dev_scene(c);
        T.seed = I.seed;
        T.tag = 0;
        T.max_bounces = I.max_bounces;
        T.p0 = 0;
        for (int a = 0; a < 3; a++) T.power[a] = c->light_intensity[a] / (float)I.photons;
        b->max_bounces = std::max(b->max_bounces, I.max_bounces);
        RenderInstDev& R = rt[(size_t)i];
        R.S = T.S;
        for (int a = 0; a < 3; a++) {
            R.cam.pos[a] = I.camera.position[a]; R.cam.fwd[a] = I.camera.forward[a];
            R.cam.right[a] = I.camera.right[a]; R.cam.up[a] = I.camera.up[a];
        }
        R.cam.vw = I.camera.viewport_w; R.cam.vh = I.camera.viewport_h; R.cam.focal = I.camera.focal;
        R.cam.W = I.camera.width; R.cam.H = I.camera.height;
        R.max_depth = I.max_depth;
        R.cls = gather_class(I.k);
    }
    b->path_off = offsets(b->paths);
    b->ph_off = offsets(caps);
    b->px_off = offsets(npx);
    b->total_paths = b->path_off.back();
    b->total_slots = b->ph_off.back();
    b->total_px = b->px_off.back();
    b->req_cap = offsets(req).back();
    b->req_split = 0;
    for (int i = 0; i < n; i++)
        if (rt[(size_t)i].cls == 0) b->req_split += req[(size_t)i];
    if (b->total_slots >= ((int64_t)1 << 32) || b->total_paths >= ((int64_t)1 << 32) ||
        b->req_cap >= ((int64_t)1 << 32) || b->total_px >= ((int64_t)1 << 32))
        return bfail(b, PM_ERR_INVALID, "batch: more than 2^32 paths, photons, pixels or requests");
    for (int i = 0; i < n; i++) {
        outs[(size_t)i].ph0 = b->ph_off[(size_t)i];
        outs[(size_t)i].cap = caps[(size_t)i];
        for (int a = 0; a < 3; a++) outs[(size_t)i].power[a] = b->trace_host[(size_t)i].power[a];
    }
    const int64_t TP = b->total_paths, NS = b->total_slots, NP = b->total_px, RC = b->req_cap;
    const size_t MB = (size_t)b->max_bounces;
    BCK(ensure(b->counter, 16));
    BCK(ensure(b->stage, MB * TP * 32));
    BCK(ensure(b->cnt_g, TP * 4));
    BCK(ensure(b->cnt_c, TP * 4));
    BCK(ensure(b->scan_g, TP * 4));
    BCK(ensure(b->totals, 16));
    BCK(ensure(b->trace_ws, scan_workspace_bytes(TP)));
    BCK(ensure(b->inst_total, (size_t)n * 8));
    BCK(ensure(b->pos, NS * 12));
    BCK(ensure(b->dir, NS * 12));
    BCK(ensure(b->pow, NS * 12));
    BCK(ensure(b->cid, NS * 4));
    BCK(ensure(b->keys0, NS * 4));
    BCK(ensure(b->keys1, NS * 4));
    BCK(ensure(b->vals0, NS * 4));
    BCK(ensure(b->vals1, NS * 4));
    BCK(ensure(b->gpos, NS * 16));
    BCK(ensure(b->gdir, NS * 12));
    BCK(ensure(b->gpow, NS * 12));
    BCK(ensure(b->req_a, RC * 16));
    BCK(ensure(b->req_b, RC * 16));
    BCK(ensure(b->req_c, RC * 16));
    BCK(ensure(b->req_counter, 16));
    BCK(ensure(b->px_base, NP * 4));
    BCK(ensure(b->px_count, NP * 4));
    BCK(ensure(b->est_g, RC * 12));
    BCK(ensure(b->queues, 16));
    BCK(ensure(b->rgb8, NP * 3));
    BCK(ensure(b->status, 16));
    BCK(cudaMemsetAsync(b->status.p, 0, 16, b->st));
    BCK(cudaMemsetAsync(b->pos.p, 0, (size_t)NS * 12, b->st));
    BCK(upload(b->t_path_off, b->path_off, b->st));
    BCK(upload(b->t_ph_off, b->ph_off, b->st));
    BCK(upload(b->t_px_off, b->px_off, b->st));
    BCK(upload(b->t_outs, outs, b->st));
    BCK(upload(b->t_render, rt, b->st));
    BCK(ensure(b->t_trace, trace_multi_table_bytes(n)));
    if (int rc = seed_frame(b, 0)) return rc;
    if (int rc = plan_grids(b, 1000)) return rc;
    if (opts && opts->autotune)
        if (int rc = autotune(b)) return rc;
    // per-stage device times of the chosen configuration (frame 0, eager)
    if (int rc = launch_stages(b, -1, nullptr)) return rc;
    for (int stage = 0; stage < 5; stage++)
        if (int rc = time_stage(b, stage, 1, &b->stage_ms[stage])) return rc;
    if (b->use_graph)
        if (int rc = capture(b)) return rc;
    return PM_OK;
}

}  // namespace

extern "C" {

int pm_batch_create(pm_batch** out, const pm_batch_instance* in, int32_t n, const pm_batch_opts* opts) {
    if (!out || !in || n <= 0) return PM_ERR_INVALID;
    pm_batch* b = new pm_batch();
    b->device = opts ? opts->device : 0;
    b->use_graph = opts ? opts->use_graph != 0 : true;
    *out = b;   // on failure too: the caller reads pm_batch_last_error, then destroys
    return create(b, in, n, opts);
}

void pm_batch_destroy(pm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (pm_ctx* c : b->ctx) pm_destroy(c);
    DevBuf* bufs[] = {&b->t_trace, &b->t_outs, &b->t_path_off, &b->t_grid, &b->t_ph_off, &b->t_cell_off, &b->t_render,
                      &b->t_px_off, &b->t_gather, &b->counter, &b->stage, &b->cnt_g, &b->cnt_c,
                      &b->scan_g, &b->totals, &b->trace_ws, &b->inst_total, &b->pos, &b->dir, &b->pow, &b->cid,
                      &b->keys0, &b->keys1, &b->vals0, &b->vals1, &b->hist, &b->grid_ws, &b->key_counts,
                      &b->key_starts, &b->cstarts, &b->csizes, &b->gpos, &b->gdir, &b->gpow, &b->req_a, &b->req_b,
                      &b->req_c, &b->req_counter, &b->px_base, &b->px_count, &b->est_g, &b->queues, &b->rgb8,
                      &b->status};
    for (DevBuf* d : bufs) release(*d);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

const char* pm_batch_last_error(const pm_batch* b) { return b ? b->err.c_str() : "null batch"; }

int pm_batch_frame(pm_batch* b, uint64_t frame) {
    if (!b) return PM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    if (frame != b->seeded_frame)
        if (int rc = seed_frame(b, frame)) return rc;
    BCK(cudaEventRecord(b->ev0, b->st));
    if (b->exec) {
        BCK(cudaGraphLaunch(b->exec, b->st));
    } else {
        int launches = 0;
        if (int rc = launch_stages(b, -1, &launches)) return rc;
        b->launches = launches;
    }
    BCK(cudaEventRecord(b->ev1, b->st));
    std::vector<int64_t> tot((size_t)b->n);
    unsigned long long nreq_cls[2] = {0, 0};   // requests of the two gather classes
    BCK(cudaMemcpyAsync(tot.data(), b->inst_total.p, (size_t)b->n * 8, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaMemcpyAsync(nreq_cls, b->req_counter.p, 16, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    b->ms_last = elapsed(b->ev0, b->ev1);
    b->photons_last = 0;
    b->underfilled = 0;
    b->stored_last.assign((size_t)b->n, 0);
    for (int i = 0; i < b->n; i++) {
        const int64_t cap = b->inst[(size_t)i].photons;
        b->stored_last[(size_t)i] = std::min(cap, tot[(size_t)i]);
        b->photons_last += b->stored_last[(size_t)i];
        if (tot[(size_t)i] < cap) b->underfilled++;
    }
    b->requests_last = (int64_t)(nreq_cls[0] + nreq_cls[1]);
    return check_batch_status(b);
}

int pm_batch_image(pm_batch* b, int32_t i, const uint8_t** out, int32_t* w, int32_t* h) {
    if (!b || !out || i < 0 || i >= b->n || !b->rgb8.p) return PM_ERR_INVALID;
    *out = P<uint8_t>(b->rgb8) + 3 * b->px_off[(size_t)i];
    if (w) *w = b->inst[(size_t)i].camera.width;
    if (h) *h = b->inst[(size_t)i].camera.height;
    return PM_OK;
}

int pm_batch_photons(pm_batch* b, int32_t i, const float** pos, const float** power, const float** dir,
                     int64_t* count) {
    if (!b || i < 0 || i >= b->n || b->stored_last.size() != (size_t)b->n) return PM_ERR_INVALID;
    const int64_t o = 3 * b->ph_off[(size_t)i];
    if (pos) *pos = P<float>(b->pos) + o;
    if (power) *power = P<float>(b->pow) + o;
    if (dir) *dir = P<float>(b->dir) + o;
    if (count) *count = b->stored_last[(size_t)i];
    return PM_OK;
}

int pm_batch_get_info(pm_batch* b, pm_batch_info* o) {
    if (!b || !o) return PM_ERR_INVALID;
    std::memset(o, 0, sizeof *o);
    o->instances = b->n;
    o->paths = b->total_paths;
    o->photon_slots = b->total_slots;
    o->keys = b->total_keys;
    o->pixels = b->total_px;
    o->request_capacity = b->req_cap;
    o->desired_per_cell = b->desired;
    o->gather_warps = b->gather_warps;
    o->gather_guess = b->guess;
    o->subcell_khint = b->khint;
    o->trace_refill = b->refill;
    o->graph = b->exec ? 1 : 0;
    o->launches_per_frame = b->launches;
    o->ms_last_frame = b->ms_last;
    o->photons_last_frame = b->photons_last;
    o->requests_last_frame = b->requests_last;
    o->underfilled = b->underfilled;
    for (int i = 0; i < 5; i++) o->stage_ms[i] = b->stage_ms[i];
    return PM_OK;
}

}  // extern "C"
