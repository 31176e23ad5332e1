// pm_trace.cuh -- photon tracing entry points (see pm_trace.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_scene.cuh"

namespace pm {

struct TraceBatch {
    DevScene S;
    uint64_t seed;
    uint32_t tag;
    int max_bounces;          // <= 32
    int64_t p0, npaths;       // paths [p0, p0 + npaths)
    float power[3];           // photon power (light intensity / global capacity)
    // scratch sized for npaths (stage: max_bounces * npaths float4 each)
    unsigned long long* path_counter;
    float4* stage_pos;
    float4* stage_dir;
    uint32_t* cnt_g;
    uint32_t* cnt_c;
    uint32_t* scan_g;
    uint32_t* scan_c;
    uint32_t* totals;         // [0] global photons of the batch, [1] caustic
    void* scan_ws;
    unsigned* status;
    int sm_count;
    int refill;               // k_trace refill threshold in lanes (1..32); 0: the default
};

struct PhotonList {
    float* pos;               // 3 floats per photon
    float* dir;
    float* pow;
    int64_t cap;
    int64_t filled;           // photons already in the list before this batch
};

// trace one batch and append its photons (canonical order) to the two lists;
// totals[0..1] receive the batch's photon counts before the capacity cut
cudaError_t trace_batch(TraceBatch& B, PhotonList& G, PhotonList& C, cudaStream_t st);

}  // namespace pm
