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
    float4* stage;            // 32-byte photon records: 2 float4 per slot, max_bounces * npaths slots
    uint32_t* cnt_g;
    uint32_t* cnt_c;
    uint32_t* scan_g;
    uint32_t* scan_c;
    uint32_t* totals;         // [0] global photons of the batch, [1] caustic
    void* scan_ws;
    unsigned* status;
    int sm_count;
    int refill;               // k_trace refill threshold in lanes (1..32); 0: the default
    cudaEvent_t k_begin = nullptr, k_end = nullptr;   // when set: recorded around the k_trace launch
    unsigned long long* work = nullptr;   // when set: the work-counting launch adds rays, node visits, triangle tests
};


struct PhotonList {
    float* pos;               // 3 floats per photon
    float* dir;
    float* pow;
    int64_t cap;
    int64_t filled;           // photons already in the list before this batch
    float4* rec = nullptr;    // when set: also (position, 0), (direction, 0) per photon, 32-byte aligned
    bool lists = true;        // false (with rec set): dir and pow are not written; photon_lists_from_rec
                              // fills them later from rec and the batch's power
};

// dir[i] = rec[2i + 1].xyz and pow[i] = pw for i < n (the lists a batch traced
// with PhotonList::lists = false left unwritten); pow only when dir is null
cudaError_t photon_lists_from_rec(const float4* rec, int64_t n, const float pw[3], float* dir, float* pow,
                                  cudaStream_t st);

// ---- several scene instances in one launch (global map only) ----
struct TraceInst {
    DevScene S;
    uint64_t seed;
    uint32_t tag;
    int max_bounces;
    int64_t p0;               // first path index of the instance's stream
    float power[3];
};
struct TraceInstOut {         // where the instance's photons go
    int64_t ph0, cap;
    float power[3];
};
struct TraceMulti {
    int ninst;
    int64_t total;            // paths over all instances
    const int64_t* path_off;  // device, ninst + 1: instance i traces global paths [off[i], off[i+1])
    void* table;              // device, trace_multi_table_bytes(ninst): per-instance parameters
    const TraceInstOut* outs; // device, ninst
    unsigned long long* path_counter;
    float4* stage;            // 2 float4 per slot, max_bounces * total slots
    uint32_t* cnt_g;          // total each
    uint32_t* cnt_c;
    uint32_t* scan_g;
    uint32_t* totals;         // [0] global photons of all instances
    void* scan_ws;
    float* pos;               // global photon list: 3 floats per photon, instance regions at ph0
    float* dir;
    float* pow;
    int64_t* inst_total;      // device, ninst: photons produced before the cut
    unsigned* status;
    int sm_count;
    int refill;
};
size_t trace_multi_table_bytes(int ninst);
// upload the per-instance parameter table (synchronises the stream)
cudaError_t trace_multi_tables(const TraceMulti& M, const TraceInst* insts, cudaStream_t st);
// one launch over all instances' paths, scan, canonical-order compaction (no host round trip)
cudaError_t trace_multi(const TraceMulti& M, cudaStream_t st);

// trace one batch and append its photons (canonical order) to the two lists;
// totals[0..1] receive the batch's photon counts before the capacity cut
cudaError_t trace_batch(TraceBatch& B, PhotonList& G, PhotonList& C, cudaStream_t st);

}  // namespace pm
