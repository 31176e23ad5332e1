/* pm_api.h -- C ABI of the B200 photon-mapping core (libpm_b200.so).
 *
 * The reference (Alator-ux/Cuda-Photon-Mapping, paths relative to its
 * CudaPhotonMapping/ directory) has no formal plugin API; its host calls C++
 * functions at three seams.  Each entry point below names the seam it replaces.
 *
 * Conventions
 *  - Every function returns PM_OK (0) or a negative PM_ERR_* code; the message
 *    of the last failure is available from pm_last_error().  The library never
 *    exits the process and never resets the device (the reference's check_cuda
 *    does both, CudaUtils.cu:6-14).
 *  - A pm_ctx belongs to one host thread at a time.  All device work is issued
 *    on the context's stream; entry points that return host-visible results
 *    synchronise that stream before returning.
 *  - Device buffers the context allocates are owned by it and freed by
 *    pm_destroy.  Output buffers passed in by the caller stay the caller's.
 *  - Pointers documented as "device" must be device (or managed) memory of the
 *    context's device; "host" pointers are read during the call only.
 */
#ifndef PM_API_H
#define PM_API_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PM_OK 0
#define PM_ERR_INVALID (-1)   /* bad argument or call order */
#define PM_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define PM_ERR_OOM (-3)       /* device allocation failed */
#define PM_ERR_TIMEOUT (-4)   /* a bounded device wait gave up (status word) */
#define PM_ERR_OVERFLOW (-5)  /* a fixed-capacity device buffer would have overflowed */
#define PM_ERR_IO (-6)        /* file read / write failed */

#define PM_MAP_GLOBAL 0       /* the reference's diffuse_grid  */
#define PM_MAP_CAUSTIC 1      /* the reference's specular_grid */

typedef struct pm_ctx pm_ctx;

typedef struct {
    int device;        /* CUDA device ordinal */
    void* stream;      /* cudaStream_t to issue work on; NULL: the context creates one */
} pm_device_opts;

/* Triangle soup sorted by model (tri_model non-decreasing).  materials: 12
 * floats per model = diffuse[3] specular[3] emission[3] ior opaque shininess
 * (Material.cuh:4-31).  tri_diffuse (optional, 3 floats per triangle)
 * overrides the model's diffuse albedo per triangle.  Host pointers. */
typedef struct {
    int32_t ntri;
    const float* tri_pos;       /* 9 floats per triangle: v0 v1 v2 */
    const float* tri_nrm;       /* 9 floats per triangle: vertex normals */
    const int32_t* tri_model;
    const float* tri_diffuse;   /* may be NULL */
    int32_t nmodel;
    const float* materials;
    int32_t light_model;        /* the model photons are emitted from (Initializer.cu:62-100) */
    float light_intensity[3];   /* LightSource::intensity (Light.cuh:8) */
    float default_ior;          /* GlobalParams::default_refractive_index */
} pm_scene_desc;

typedef struct {
    uint64_t seed;              /* key of the per-path Philox streams */
    uint32_t stream_tag;        /* fourth counter word (0 for photon paths) */
    int32_t max_bounces;        /* PHOTON_BOUNCE_NUM (PhotonTracing.cu:20); 1..32 */
    int64_t global_capacity;    /* diffuse_num of trace_photons */
    int64_t caustic_capacity;   /* specular_num of trace_photons (0: no caustic map) */
    int64_t max_paths;          /* give up (PM_ERR_INVALID) after this many paths; 0: 64 x capacity */
} pm_trace_opts;

typedef struct {
    int32_t desired_per_cell;   /* 1000 in PhotonGrid::build */
    int32_t regrid_mult;        /* re-grid when a cell holds > regrid_mult * desired (5) */
    int32_t regrid_div;         /* ... at desired / regrid_div photons per cell (5) */
    int32_t sub_div;            /* photons inside a cell are ordered by sub-cell, each cell split
                                   sub_div^3 ways (1, 2, 4 or 8; 0 = chosen from the fullest cell);
                                   the gather walks sub-cells.  The cells are the reference's. */
    int32_t k_hint;             /* expected kNN k for the automatic sub_div (0 = 64) */
} pm_grid_opts;

/* The reference Camera's fields (Camera.cuh:11-33); pm_camera_setup fills them
 * like Camera's constructor (Camera.cuh:43-65). */
typedef struct {
    float position[3], forward[3], right[3], up[3];
    float viewport_w, viewport_h, focal;
    int32_t width, height;
} pm_camera;

typedef struct {
    int32_t max_depth;          /* GlobalParams::max_depth (kernel.cu:23): 0..5 */
    int32_t k_global;           /* GlobalParams::global_photon_num: kNN k of the global map (<= 256) */
    float r_global;             /* 0.1 in render_trace (Raytracer.cuh:187) */
    int32_t k_caustic;          /* GlobalParams::caustic_photon_num (<= 256) */
    float r_caustic;            /* 0.2 (Raytracer.cuh:200) */
    int32_t faithful_caustic;   /* 1: the caustic estimate reads the global map's direction / power
                                   arrays with caustic indices, as Raytracer.cuh:203-204 does */
} pm_render_opts;

/* Read-only device view of one photon map (valid until the map is rebuilt). */
typedef struct {
    int64_t count;              /* photons in the map */
    int64_t cells;
    int32_t dims[3];
    float cell_size;
    float aabb[6];
    const uint32_t* cell_starts;    /* device, cells entries (exclusive scan of cell_sizes) */
    const uint32_t* cell_sizes;     /* device, cells entries */
    const float* sorted_pos;        /* device, 4 floats per photon: xyz + source index bits */
    const float* sorted_dir;        /* device, 3 floats per photon */
    const float* sorted_power;      /* device, 3 floats per photon */
    const float* list_pos;          /* device, traced order (before the grid build), 3 floats */
    const float* list_dir;
    const float* list_power;
    int32_t sub_div;                /* sub-cells per cell axis of the sorted order */
    const uint32_t* key_starts;     /* device, cells * sub_div^3 + 1 entries: photons of sub-cell
                                       key (cell * sub_div^3 + sx + sub_div * (sy + sub_div * sz))
                                       are sorted slots [key_starts[key], key_starts[key + 1]) */
} pm_photon_view;

/* ------------------------------------------------------------- lifetime -- */
int pm_create(pm_ctx** out, const pm_device_opts* opts);
void pm_destroy(pm_ctx* ctx);
const char* pm_last_error(const pm_ctx* ctx);
int pm_sync(pm_ctx* ctx);

/* Scene upload + BVH build.  Replaces the device half of
 * initialize_scene_and_photon_maps (Initializer.cu:180-205): models, lights,
 * scene AABB, critical-angle table (PhotonTracing.cu:79-125). */
int pm_set_scene(pm_ctx* ctx, const pm_scene_desc* scene);

/* OBJ / MTL import (host only, no context).  Replaces loadOBJ
 * (ObjLoader.cpp:18-320) with the light convention of
 * initialize_light_sources (Initializer.cu:62-100): models are runs of
 * consecutive face lines named by the last g / o line, materials come from
 * usemtl + the mtllib file (Material() defaults for what it omits), quads
 * split as (v0 v1 v3), (v1 v2 v3), the model named "light" emits.  Errors:
 * PM_ERR_IO (file), PM_ERR_INVALID (syntax, indices), message in err. */
typedef struct pm_obj_scene pm_obj_scene;
int pm_obj_load(const char* dir, const char* file, pm_obj_scene** out, char* err, int err_len);
/* A pm_scene_desc pointing into s (valid while s lives): light intensity 1,
 * the given default refractive index.  PM_ERR_INVALID if no model is named "light". */
int pm_obj_desc(const pm_obj_scene* s, float default_ior, pm_scene_desc* out);
int32_t pm_obj_model_count(const pm_obj_scene* s);
const char* pm_obj_model_name(const pm_obj_scene* s, int32_t model);
int32_t pm_obj_light_model(const pm_obj_scene* s);   /* -1: none */
void pm_obj_free(pm_obj_scene* s);
int pm_scene_aabb(pm_ctx* ctx, float out_aabb[6]);

/* BVH builder used by the next pm_set_scene (the closest-hit answers, and so
 * every photon map and image, are the same with either; only speed differs). */
#define PM_BVH_HOST_SAH 0     /* binned SAH on the host (default): the faster tree to trace */
#define PM_BVH_DEVICE_LBVH 1  /* linear BVH over Morton codes, built on the device in ~1 ms */
int pm_set_bvh_builder(pm_ctx* ctx, int builder);

/* The current scene's BVH: its builder, interior nodes, build time in ms. */
int pm_bvh_info(pm_ctx* ctx, int32_t* out_builder, int64_t* out_nodes, float* out_build_ms);

/* Photon pass.  Replaces trace_photons(gpu_scene, cpu_scene, diffuse_num,
 * specular_num) (PhotonTracing.cu:379-422): fills both maps' photon lists to
 * capacity in canonical order (path index, then bounce). out_paths (optional)
 * receives the number of paths traced. */
int pm_trace_photons(pm_ctx* ctx, const pm_trace_opts* opts, int64_t* out_paths);

/* The photon pass of pm_trace_photons (the same photons, lists and grids
 * untouched otherwise) with the tracer's work counted, for the flop roofline
 * of the photon tracer (no counterpart in the reference, which estimates 86
 * flop per triangle test, Model.cuh:65-67): out_work[0] = rays traced (a ray
 * whose nearest hit sits at t = 0 in an earlier model counts once),
 * [1] BVH interior nodes visited (each visit tests both children's boxes),
 * [2] triangle tests.  The counting launch runs slower than pm_trace_photons;
 * time the latter. */
int pm_trace_work(pm_ctx* ctx, const pm_trace_opts* opts, int64_t* out_paths, uint64_t out_work[3]);

/* Photon output of paths [p0, p1) without a capacity cut (parity testing and
 * path-range sharding).  Writes device arrays of capacity (p1-p0)*max_bounces
 * photons per map: pos/dir (3 floats), and per path counts[2] (global,
 * caustic).  power_capacity sets the photon power (intensity / power_capacity). */
int pm_trace_paths(pm_ctx* ctx, const pm_trace_opts* opts, int64_t p0, int64_t p1, int64_t power_capacity,
                   float* g_pos, float* g_dir, float* c_pos, float* c_dir, uint32_t* counts,
                   int64_t* out_ng, int64_t* out_nc);

/* Replace a map's photon list with caller data (host or device arrays, 3
 * floats per photon) -- the input side of PhotonGrid::build and of the
 * photon-map reader load() (Initializer.cu:102-141). */
int pm_set_photons(pm_ctx* ctx, int map, int64_t n, const float* pos, const float* power, const float* dir);

/* Grid build.  Replaces PhotonGrid(num_photons, aabb).build(photons, 1000,
 * 5000) (PhotonGrid.cuh:44-66, PhotonGrid.cu:41-218).  aabb: NULL = scene AABB. */
int pm_build_grid(pm_ctx* ctx, int map, const pm_grid_opts* opts, const float* aabb);

/* Device pointers to a map's photon list and grid (valid until the next call
 * that replaces them).  A traced map's direction and power lists and its
 * grid's sorted power are not written by the photon pass and the grid build
 * (the grid reads 32-byte position + direction records, the gather the
 * uniform power); the first pm_get_photons or pm_save_photons after them
 * writes them on the context stream and synchronises it. */
int pm_get_photons(pm_ctx* ctx, int map, pm_photon_view* out);

/* Photon-map file in the reference's layout: u64 count, then per photon
 * pos[3] power[3] inc_dir[3] float32 (the reader is Initializer.cu:102-141).
 * Save writes the map's traced-order list; load fills the list (build next). */
int pm_save_photons(pm_ctx* ctx, int map, const char* path);
int pm_load_photons(pm_ctx* ctx, int map, const char* path);

/* kNN gather + radiance estimate over a built map.  Replaces
 * PhotonGrid::find_nearests + Raytracer::get_color_from_photon_grid
 * (PhotonGrid.cu:257-284, Raytracer.cuh:110-138) for n query points.
 * Device arrays: qpos/qnrm 3 floats per query; out_rad 3 floats per query;
 * out_ids (optional) k per query, source indices ascending by (distance, index),
 * 0xffffffff padding; out_cnt (optional) neighbours found. */
int pm_gather(pm_ctx* ctx, int map, int64_t n, const float* qpos, const float* qnrm, int k, float radius,
              float* out_rad, uint32_t* out_ids, int32_t* out_cnt);

/* Camera like Camera(position, direction, up, fov, W, H) (Camera.cuh:43-65). */
int pm_camera_setup(const float position[3], const float direction[3], const float up[3], float vertical_fov_deg,
                    int32_t width, int32_t height, pm_camera* out);

/* One frame.  Replaces Drawer::draw_in_gpu / Raytracer::render_gpu
 * (Drawer.cu:22-41, Raytracer.cuh:245-279): out_rgb8 is a device buffer of
 * width*height*3 bytes (row 0 = bottom row, as the reference's canvas);
 * out_radiance (optional) 3 floats per pixel, before tone mapping.
 * The global map must be built; the caustic map is used when built. */
int pm_render(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* opts, uint8_t* out_rgb8, float* out_radiance);

/* The rows [y0, y1) of pm_render's frame (a pixel-row band; no counterpart in
 * the reference, whose frame is one launch): the eye pass runs only the pixel
 * blocks that meet those rows, so the band costs about its share of the
 * frame.  Pixels of the band are pm_render's bit for bit; every other pixel
 * of out_rgb8 / out_radiance holds 0 or, in the pixel blocks that straddle
 * the band's edges, pm_render's value.  For frames split over GPUs. */
int pm_render_rows(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* opts, int32_t y0, int32_t y1,
                   uint8_t* out_rgb8, float* out_radiance);

/* A whole frame in one call: pm_trace_photons(trace), pm_build_grid of the
 * global map (and of the caustic map when trace fills one and k_caustic > 0)
 * with grid, then pm_render's frame.  The eye pass needs neither the photons
 * nor the grid, so it is queued on a second stream of the context right after
 * the photon pass's kernels (its blocks take the tracer's SMs as its last
 * paths end), followed there by the ordering of its requests for the gather,
 * beside the grid build.
 * Results are pm_trace_photons + pm_build_grid + pm_render's
 * (Initializer.cu:142-177 followed by Drawer::draw_in_gpu, Drawer.cu:22-41). */
int pm_frame(pm_ctx* ctx, const pm_trace_opts* trace, const pm_grid_opts* grid, const pm_camera* cam,
             const pm_render_opts* opts, uint8_t* out_rgb8, float* out_radiance, int64_t* out_paths);

/* Headless frame output, in place of the reference's GL pixel-buffer display
 * (Drawer.cu:22-41, Window.cuh:88-126).  Both take a frame in pm_render's
 * layout (row 0 = the bottom row, Camera.cuh:67-81) in device or host memory
 * (device buffers are copied to the host first; the calling thread's current
 * device must own them) and need no pm_ctx.
 * pm_write_ppm: rgb8 = width*height*3 bytes, written as a binary PPM (P6,
 * maxval 255), top row first.
 * pm_write_pfm: radiance = width*height*3 floats, written as a colour PFM
 * ("PF", scale -1.0: little-endian), whose rows run bottom to top like the
 * canvas.  Errors: PM_ERR_INVALID (null, non-positive size), PM_ERR_CUDA (the
 * device copy), PM_ERR_IO (the file). */
int pm_write_ppm(const char* path, const uint8_t* rgb8, int32_t width, int32_t height);
int pm_write_pfm(const char* path, const float* radiance, int32_t width, int32_t height);

/* Device prefix sum used by the grid build (exposed for known-answer tests):
 * exclusive (inclusive = 0) or inclusive scan of n u32 device values. */
int pm_scan_u32(pm_ctx* ctx, const uint32_t* in, uint32_t* out, int64_t n, int inclusive);

/* Test hook for the bounded device waits (no counterpart in the reference,
 * whose grid scan waits on a spin barrier without a limit,
 * CudaGridSynchronizer.cuh:13-27): the inclusive look-back scan of
 * pm_scan_u32 with each wait limited to spin_limit polls (1 .. 2^22) and tile
 * silent_tile (tiles of 4096 values; -1: none) publishing nothing, so the
 * tiles after it wait on a flag that nothing sets.  Their waits give up, the
 * kernel ends normally and the call returns PM_ERR_TIMEOUT with the context
 * still usable (out then holds no valid sums).  With silent_tile = -1 it is
 * pm_scan_u32 (inclusive). */
int pm_debug_scan_stall(pm_ctx* ctx, const uint32_t* in, uint32_t* out, int64_t n, int64_t spin_limit,
                        int32_t silent_tile);

/* Allocation-free scan (no counterpart in the reference).  For callers that
 * may not allocate device memory: hosts that reserve the whole device for their
 * own pool, or frame loops that must not call cudaMalloc / cudaFree (which can
 * synchronise the device) while work is in flight.  Same scan as pm_scan_u32
 * on the caller's device buffers (in, out: n u32 each), issued on `stream`
 * (a cudaStream_t; NULL = the default stream) of the current device, which
 * is synchronised before returning.  Needs no pm_ctx: the look-back workspace
 * is a fixed 32,784-byte array in the library's device memory, held on every
 * GPU that loads the library until the process exits.  n above
 * PM_NOALLOC_SCAN_MAX returns PM_ERR_INVALID.  The first call on a device
 * looks up the array's address (once per device); make it before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race, so
 * serialise them.  Errors are returned as codes only (there is no context
 * for pm_last_error). */
#define PM_NOALLOC_SCAN_MAX 16777216
int pm_scan_u32_noalloc(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, void* stream);

/* Per-stage device times of the last pm_trace_photons / pm_build_grid /
 * pm_render calls in milliseconds (CUDA events on the context stream):
 * [0] trace, [1] grid build (global map), [2] eye pass, [3] gather (request
 * ordering + global gather + caustic gather; in pm_frame the ordering runs
 * beside the grid build and is not counted here), [4] resolve, [5] the k_trace
 * kernels alone, [6] the global gather kernel alone.  In pm_frame the eye pass
 * is queued beside the photon pass, so [2] spans the photon pass as well and
 * [0] includes the eye blocks' share of the GPU; [1] runs from the grid
 * build's start to the gather's start (the join of both streams). */
int pm_stage_times(pm_ctx* ctx, float out_ms[8]);

/* ---------------------------------------------------------------------------
 * Learned radiance cache (no counterpart in the reference).  A small MLP maps
 * (hit point, shading normal) to the global-map radiance estimate that
 * Raytracer::get_color_from_photon_grid (CudaPhotonMapping/Raytracer.cuh:110-138)
 * computes by a kNN gather.  Inputs: the point normalised to a box and the
 * octahedral normal, encoded with sin / cos at 6 octaves (60 features); 4
 * hidden layers of width 64 with ReLU; RGB output.  BF16 weights and
 * activations on the tensor cores with FP32 accumulation; FP32 Adam.
 * Parameters are PM_CACHE_PARAMS floats: 5 layers x [64 out][64 in], layer 0
 * reads inputs 0..59, layer 4 writes outputs 0..2 (the rest stays zero).
 * All sample arrays are device pointers, 3 floats per sample. */
#define PM_CACHE_PARAMS (5 * 64 * 64)

typedef struct pm_cache_opts {
    uint64_t seed;          /* weight initialisation */
    float lr, beta1, beta2, eps;   /* Adam */
    float out_scale;        /* radiance = out_scale * network output (targets are divided by it) */
    float aabb[6];          /* encoding box (min xyz, max xyz); all zero: the scene's box */
    int32_t octave0;        /* lowest encoding octave (frequencies pi 2^(octave0 + f), f = 0..5), 0..8 */
} pm_cache_opts;

/* (Re)initialise the cache: weights from the seed, Adam moments zero. */
int pm_cache_init(pm_ctx* ctx, const pm_cache_opts* opts);

/* One Adam step on the mean squared error over n samples (target: radiance,
 * weight: per-sample weight or null).  *out_loss (optional) = the step's mean
 * squared error in network units (before the update). */
int pm_cache_train_step(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                        int64_t n, float* out_loss);

/* `steps` Adam steps over consecutive batches of `batch` samples of the n-sample
 * pool, starting at *inout_offset (null: 0) and wrapping to 0 where a batch
 * would run past n; *inout_offset receives the next offset.  No host
 * synchronisation between steps.  With out_loss set, the call waits for the
 * steps, checks their device status and stores the last step's loss (as
 * pm_cache_train_step reports it).  With out_loss null it returns once the
 * steps are queued, on the context's own training stream after everything
 * queued so far: work issued next that does not touch the cache (a photon
 * pass, the eye pass of pm_render_learned) runs beside them, every call that
 * reads or writes the cache or synchronises the context waits for them, and
 * a device-side failure of theirs is reported by the next synchronising call.
 * The sample arrays must stay valid until then. */
int pm_cache_train_steps(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                         int64_t n, int64_t batch, int steps, int64_t* inout_offset, float* out_loss);

/* Gradient of that loss with respect to the parameters, without an update
 * (host output of PM_CACHE_PARAMS floats), and the loss. */
int pm_cache_gradient(pm_ctx* ctx, const float* pos, const float* nrm, const float* target, const float* weight,
                      int64_t n, float* out_grad_host, float* out_loss);

/* Radiance predicted for n samples (out_rgb: device, 3 floats per sample). */
int pm_cache_infer(pm_ctx* ctx, const float* pos, const float* nrm, int64_t n, float* out_rgb);

/* Training points: the primary hits of n camera rays through stratified
 * jittered image positions (sample i lies in pixel floor(i * W * H / n) in
 * row-major order, at a seeded uniform offset), 3 floats of position and shading normal
 * and a weight (1 where the render gathers the global map there, else 0) per
 * sample; device outputs.  Label them with pm_gather. */
int pm_cache_sample_points(pm_ctx* ctx, const pm_camera* cam, int64_t n, uint64_t seed, float* out_pos,
                           float* out_nrm, float* out_weight);

typedef struct pm_learned_opts {
    int32_t tile;           /* screen tile edge in pixels */
    int32_t probes;         /* exact-gather probes per tile (first request of fixed pixels) */
    float max_rel_err;      /* a tile whose cache bias over its probes, sum_c |sum_k (cache - exact)| /
                               sum_c sum_k exact, exceeds this uses the exact gather;
                               negative: every tile does (the plain render's estimates) */
    float noise_z;          /* 0..100: the bias must also exceed the threshold by noise_z standard
                               errors of the probe differences' sum (sum_c sqrt(n) s_c, s_c the
                               sample standard deviation over the n probes), so that the exact
                               probes' own kNN noise does not flag a tile; 0: threshold only */
} pm_learned_opts;

typedef struct pm_learned_stats {
    int64_t tiles, fallback_tiles, requests, fallback_requests;
} pm_learned_stats;

/* pm_render with the global-map estimate taken from the cache, checked per
 * tile against exact gathers at the probes; tiles above max_rel_err (and all
 * caustic estimates) use the kNN gather.  out_stats optional. */
int pm_render_learned(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* opts, const pm_learned_opts* lopts,
                      uint8_t* out_rgb8, float* out_radiance, pm_learned_stats* out_stats);

/* The learned frame as one replayable CUDA graph (no counterpart in the
 * reference, whose frame is Drawer::draw_in_gpu, Drawer.cu:22-41): `steps`
 * Adam steps on consecutive `batch`-sample slices of the training pool
 * (device arrays, 3 floats per sample, the slicing of pm_cache_train_steps
 * from pool_offset), then pm_render_learned's frame into out_rgb8 /
 * out_radiance (device, fixed at creation; radiance optional).  The global
 * map only (k_caustic must be 0 when a caustic map is built).  Creation runs
 * one frame eagerly to load its kernels and puts the cache back as it was,
 * then captures on the context's stream (which must not be the legacy default
 * stream).  The graph reads the context's scene, photon map and cache: create
 * it again after pm_set_scene, pm_build_grid or pm_cache_init (a run refuses
 * with PM_ERR_INVALID otherwise).  Each run is one graph launch and one
 * status check; out_stats optional.
 * overlap_training = 0: the frame's training, then its render with the
 * trained cache (pm_cache_train_steps + pm_render_learned).
 * overlap_training = 1: the render reads the cache as the previous frames
 * trained it (a copy taken at the frame's start) and the frame's training runs
 * beside the whole render, for the frames that follow (pm_render_learned +
 * pm_cache_train_steps, in that order). */
typedef struct pm_learned_graph pm_learned_graph;
int pm_learned_graph_create(pm_ctx* ctx, const pm_camera* cam, const pm_render_opts* opts, const pm_learned_opts* lopts,
                            const float* pool_pos, const float* pool_nrm, const float* pool_target, int64_t pool_n,
                            int64_t batch, int32_t steps, int64_t pool_offset, int32_t overlap_training,
                            uint8_t* out_rgb8, float* out_radiance, pm_learned_graph** out);
int pm_learned_graph_run(pm_learned_graph* graph, pm_learned_stats* out_stats);
/* The pool offset the next frame's training starts at. */
int pm_learned_graph_offset(pm_learned_graph* graph, int64_t* out_offset);
void pm_learned_graph_destroy(pm_learned_graph* graph);

/* Host copies of the FP32 master parameters (get / set, PM_CACHE_PARAMS floats). */
int pm_cache_get_params(pm_ctx* ctx, float* out_params_host);
int pm_cache_set_params(pm_ctx* ctx, const float* params_host);

/* Read-only device view of the last render's gather requests (valid until
 * the next render).  Request q: a[q] = (hit point, triangle index bits),
 * b[q] = (shading normal, flag bits: 1 global estimate, 2 caustic estimate,
 * 4 exact fallback of the learned render), c[q] = (path weight, pixel index
 * bits); the requests of pixel p are px_base[p] .. px_base[p] + px_count[p] - 1
 * in hit order. */
typedef struct pm_request_view {
    int64_t count, pixels;
    const float* a;
    const float* b;
    const float* c;
    const uint32_t* px_base;
    const uint32_t* px_count;
    const float* est_global;   /* the global estimates the resolve used, 3 floats per request */
} pm_request_view;
int pm_get_requests(pm_ctx* ctx, pm_request_view* out);

/* ---------------------------------------------------------------------------
 * Batched form (no counterpart in the reference).  Many scene instances,
 * each with its own scene, camera, photon budget, k and radius, rendered per
 * frame by kernels that take all instances' work from one queue per stage:
 * one photon-tracing launch over every instance's paths, one grid build (one
 * sort over all instances' keys), one eye pass over all pixels, one
 * persistent gather over all requests, one resolve.  The frame is captured
 * once into a CUDA graph and replayed.  Each instance's image equals a
 * single-instance pm_trace_photons + pm_build_grid + pm_render of it with the
 * same grid sizing (bit for bit when the batch uses the reference's sizing;
 * autotuned cell sizes change only the float summation order of estimates).
 * A batch builds global maps only (no caustic map). */
typedef struct pm_batch pm_batch;

typedef struct pm_batch_instance {
    const pm_scene_desc* scene;   /* host arrays, copied at creation */
    pm_camera camera;
    uint64_t seed;                /* photon streams (frame f uses seed + f) */
    int64_t photons;              /* global-map capacity */
    int32_t max_bounces;          /* 1..32 */
    int32_t k;                    /* 1..256 */
    float radius;
    int32_t max_depth;            /* eye path depth 0..5 */
} pm_batch_instance;

typedef struct pm_batch_opts {
    int32_t device;
    int32_t autotune;             /* 1: cell size, gather block shape and trace refill chosen by timing
                                     candidate frames at creation; 0: the reference's grid sizing */
    int32_t use_graph;            /* 1: capture the frame into a CUDA graph and replay it */
} pm_batch_opts;

typedef struct pm_batch_info {
    int32_t instances;
    int64_t paths, photon_slots, keys, pixels, request_capacity;
    int32_t desired_per_cell;     /* chosen grid sizing (photons per cell) */
    int32_t gather_warps;         /* chosen gather block shape (warps per block) */
    int32_t trace_refill;         /* chosen trace refill threshold */
    int32_t graph;                /* 1 when frames replay a captured graph */
    int32_t launches_per_frame;   /* kernels one frame launches */
    float ms_last_frame;          /* device time of the last frame (CUDA events) */
    int64_t photons_last_frame;   /* photons stored by the last frame (after the capacity cuts) */
    int64_t requests_last_frame;
    int32_t underfilled;          /* instances whose last frame produced fewer photons than their capacity */
    float stage_ms[5];            /* trace, grid, eye, gather, resolve of one eager frame timed at creation */
    float gather_guess;           /* chosen first-ring guess of the gather walk (photons in units of k; 0: none) */
    float subcell_khint;          /* chosen sub-cell split: 0 = pm_grid_opts' default, else the automatic
                                     split for subcell_khint x each instance's k */
} pm_batch_info;

/* Creation traces each instance once (calibration), builds the grids, runs
 * the autotuner when asked, and captures the frame graph.  On failure *out
 * may still hold the batch: read pm_batch_last_error, then pm_batch_destroy. */
int pm_batch_create(pm_batch** out, const pm_batch_instance* instances, int32_t n, const pm_batch_opts* opts);
void pm_batch_destroy(pm_batch* b);
const char* pm_batch_last_error(const pm_batch* b);
/* One frame of every instance (photon streams seeded with seed + frame). */
int pm_batch_frame(pm_batch* b, uint64_t frame);
/* Device pointer to instance i's last image (uchar3, width x height, rows as pm_render). */
int pm_batch_image(pm_batch* b, int32_t i, const uint8_t** out_rgb8, int32_t* width, int32_t* height);
int pm_batch_get_info(pm_batch* b, pm_batch_info* out);
/* The photon list instance i stored in the last pm_batch_frame (its global
 * map before the grid's cell sort, canonical order: path, then bounce), as
 * device pointers into the batch (3 floats per photon each), valid until the
 * next pm_batch_frame or pm_batch_destroy; *count photons.  The same list as
 * pm_trace_photons of the instance with seed + frame.  PM_ERR_INVALID before
 * the first frame. */
int pm_batch_photons(pm_batch* b, int32_t i, const float** pos, const float** power, const float** dir,
                     int64_t* count);

/* Gather requests (eye-path hits that query the global map) of the last
 * pm_render call: the number of kNN queries its gather stage answered. */
int pm_render_requests(pm_ctx* ctx, int64_t* out);

/* Number of kernels this context has launched so far. */
int pm_launch_count(pm_ctx* ctx, int64_t* out);

/* Device status word (bits: 1 timeout, 2 overflow, 4 stack, 8 bad input); read + clear. */
int pm_status(pm_ctx* ctx, uint32_t* out_bits);

#ifdef __cplusplus
}
#endif

#endif /* PM_API_H */
