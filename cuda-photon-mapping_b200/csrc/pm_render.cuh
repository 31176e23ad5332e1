// pm_render.cuh -- eye pass (gather requests) and per-pixel resolve.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_scene.cuh"

namespace pm {

constexpr int RENDER_MAX_DEPTH = 5;                          // eye-path depth limit of this library
constexpr int RENDER_MAX_HITS = (1 << RENDER_MAX_DEPTH) - 1; // binary hit tree

struct CameraDev {
    float pos[3], fwd[3], right[3], up[3];
    float vw, vh, focal;
    int W, H;
};

// Gather request of one eye-path hit (3 float4):
//   a = (hit point, triangle bits)  b = (shading normal, flags bits)  c = (path weight, pixel bits)
// flags bit 0: the global-map estimate is needed (not inside an object, albedo non-zero)
struct Requests {
    float4* a;
    float4* b;
    float4* c;
    int64_t cap;
    unsigned long long* counter;   // requests written
    uint32_t* px_base;             // first request of each pixel
    uint32_t* px_count;            // requests of each pixel (hit order)
};

// block_order (optional, eye_blocks(cam) entries): the pixel block each thread
// block of the launch takes (a permutation), e.g. the slow ones first.
// nblocks >= 0: only the first nblocks entries of block_order run (a subset of
// the pixel blocks); pixels of the other blocks get no requests written.
cudaError_t eye_pass(const DevScene& S, const CameraDev& cam, int max_depth, Requests R, unsigned* status,
                     cudaStream_t st, const int* block_order = nullptr, int64_t nblocks = -1);
// 27-bit Morton code of each request's hit point in the box aabb (9 bits per
// axis: three radix passes of 9 bits)
constexpr int REQUEST_KEY_BITS = 27;
cudaError_t request_keys(const float4* a, int64_t n, const float aabb[6], uint32_t* keys, cudaStream_t st);
// pixel blocks of the eye pass (EYE_THREADS consecutive pixels each)
int64_t eye_blocks(int64_t npx);
int eye_threads();

// The k-th of P probe pixels of a tile x tile block: a g x g lattice
// (g = ceil(sqrt(P))) of cell centres, row by row.
__host__ __device__ inline void probe_xy(int k, int P, int T, int& dx, int& dy) {
    int g = 1;
    while (g * g < P) g++;
    dx = ((k % g) * 2 + 1) * T / (2 * g);
    dy = ((k / g) * 2 + 1) * T / (2 * g);
}
// The first gather request of P probe pixels per tile x tile block of the
// image (probe s = tile s / P, lattice point s % P), traced directly from the
// camera: where the pixel's primary ray hits a surface that needs the global
// estimate, ppos = (hit point, triangle bits), pnrm = (shading normal, 1);
// else (0, 0, 0, 0), (0, 0, 1, 0).  The same values (by the same device code)
// as the eye pass's first request of those pixels, so the probes' exact
// gathers can run before or beside the eye pass.
cudaError_t probe_hits(const DevScene& S, const CameraDev& cam, int tile, int P, float4* ppos, float4* pnrm,
                       cudaStream_t st);

// ---- several instances in one launch: global pixel g of instance i lies in
// [px_off[i], px_off[i+1]); requests and outputs are indexed by global pixel ----
struct RenderInstDev {
    DevScene S;
    CameraDev cam;
    int max_depth;
    int cls;                  // the gather class of the instance's requests (0 or 1)
};
// The requests of class-0 instances go to [0, split) from R.counter[0], those
// of class-1 instances to [split, R.cap) from R.counter[1] (R.counter: 2
// device counters, zeroed here), so each gather launch visits its own range.
cudaError_t eye_pass_multi(const RenderInstDev* tab, const int64_t* px_off, int ninst, int64_t npx, Requests R,
                           int64_t split, unsigned* status, cudaStream_t st);
cudaError_t resolve_multi(const RenderInstDev* tab, const int64_t* px_off, int ninst, int64_t npx, Requests R,
                          const float* est_g, float tone_t, uint8_t* rgb8, float* radiance, cudaStream_t st);

// Primary hits of n camera rays through uniformly jittered image positions
// (sample i draws its position from the Philox stream (seed, i, tag)): hit
// point, shading normal as the eye pass stores it, weight 1 where the eye pass
// would request the global-map estimate (hit, albedo non-zero), else 0.
cudaError_t sample_primary_hits(const DevScene& S, const CameraDev& cam, int64_t n, uint64_t seed, float* pos,
                                float* nrm, float* weight, cudaStream_t st);

// Combines the estimates of each pixel's requests in hit order, tone-maps and
// quantises (CudaPhotonMapping/Raytracer.cuh:187-211, 238-240, 277).
// est_c may be null (no caustic map).  rgb8: 3 bytes per pixel; radiance: 3
// floats per pixel (optional).  tone_t = 1 / exposure as the reference computes it.
cudaError_t resolve(const DevScene& S, const CameraDev& cam, Requests R, const float* est_g, const float* est_c,
                    float tone_t, uint8_t* rgb8, float* radiance, cudaStream_t st);

}  // namespace pm
