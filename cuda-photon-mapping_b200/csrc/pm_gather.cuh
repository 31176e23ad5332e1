// pm_gather.cuh -- kNN photon gather + radiance estimate.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pm {

struct GatherGrid {
    const float4* gpos;        // sorted photons: xyz + source id bits
    const float* gdir;         // direction / power arrays the estimate reads (3 floats per slot)
    const float* gpow;
    const uint32_t* key_starts;  // cells * S^3 + 1: photons of sub-cell key k are [key_starts[k], key_starts[k+1])
    float mn[3];               // grid origin (scene AABB min)
    int gx, gy, gz;
    float cell;
    int S;                     // sub-cells per cell axis
    float guess;               // the walk's first-ring bound is guessed to hold about guess x k photons
                               // (GATHER_GUESS by default; 0: no guess).  Speed only: answers do not change
    bool pow_uniform;          // every photon has power pw (a traced map): the estimate reads no power array
    float pw[3];
};
// 1080p frame of 10M photons, k 64: 2.0 -> 3.07 ms, 1.6 -> 3.03, 1.5 -> 3.02,
// 1.4 -> 3.01, 1.2 -> 3.21 (more walks restart); k 200 at r 0.02 on 30M
// photons: 7.03 ms at 2.0 and 1.6, 7.04 at 1.5, 7.07 at 1.4 (and on the
// 100M-photon 4K frame 1.5 measured 27.9 ms against 27.4 at 2.0)
constexpr float GATHER_GUESS = 1.6f;

struct GatherQueries {
    int64_t n;
    // either packed 3-float arrays ...
    const float* pos3;
    const float* nrm3;
    // ... or float4 records (xyz; flag bits in w of nrm4): a record is gathered
    // when (flags & flag_mask) != 0, otherwise its estimate is zero
    const float4* pos4;
    const float4* nrm4;
    uint32_t flag_mask;
    // optional: query i is record idx[i] (read from and written to that index)
    const uint32_t* idx;
};

struct GatherOut {
    float* rad;               // 3 floats per query (required)
    uint32_t* ids;            // k per query, ascending (distance, id); UINT_MAX padding (optional)
    int* cnt;                 // neighbours found (optional)
    float* rk;                // largest selected distance (optional)
};

// k <= 256.  require_full: the estimate is written only when k neighbours were
// found (the caustic rule of CudaPhotonMapping/Raytracer.cuh:200), zero otherwise.
// Queries listed in Q.idx (records in Q.pos4 / Q.nrm4, Q.n = list capacity),
// as many as the device count *n_dev says; persistent launch over the
// resident warps, *queue (device scratch) the work counter.
cudaError_t gather_listed(const GatherGrid& G, const GatherQueries& Q, const unsigned long long* n_dev,
                          unsigned long long* queue, float r, int k, const GatherOut& O, int sm_count,
                          cudaStream_t st);

cudaError_t gather(const GatherGrid& G, const GatherQueries& Q, float r, int k, int require_full,
                   const GatherOut& O, unsigned* status, cudaStream_t st);

// ---- requests of several instances in one work queue ----
struct GatherInstDev {
    GatherGrid G;
    float r;
    int k;
    int cls;                  // gather_class(k): which store size answers it
};
int gather_class(int k);
// Q: the request records (pos4 / nrm4 with flag_mask), Q.n = their capacity;
// rec_c: their third records (global pixel bits in w); the requests of class
// 0 lie in [0, split), n_req[0] of them, those of class 1 in [split, Q.n),
// n_req[1] of them (eye_pass_multi's layout); queues: 2 device counters
// (scratch); px_off: ninst + 1 pixel offsets; warps: block shape, 4 or 8
// warps per block.  Two persistent launches (store classes of k <= 96 and
// k <= 256), each over its own range; O.rad only (ids, cnt, rk null).
cudaError_t gather_multi(const GatherInstDev* tab, const int64_t* px_off, int ninst, const GatherQueries& Q,
                         const float4* rec_c, const unsigned long long* n_req, int64_t split,
                         unsigned long long* queues, const GatherOut& O, int warps, int sm_count, cudaStream_t st);

}  // namespace pm
