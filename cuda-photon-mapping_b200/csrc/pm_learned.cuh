// pm_learned.cuh -- the learned render's per-tile cache check (see pm_learned.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_render.cuh"

namespace pm {

constexpr uint32_t LEARNED_FALLBACK = 4u;   // request flag: answered by the exact gather

// The request each of the P probes per tile of edge `tile` stands for (its
// pixel's first request when that needs the global estimate, else
// UINT32_MAX), after the eye pass; ppos / pnrm are the probe records of
// probe_hits (pm_render.cuh), checked against the requests bit for bit
// (a mismatch raises ST_BAD_INPUT in status).
cudaError_t learned_probe_req(const CameraDev& cam, const Requests& R, int tile, int P, const float4* ppos,
                              const float4* pnrm, uint32_t* preq, unsigned* status, cudaStream_t st);

// Tile flags from the probes' exact and cached estimates (bias above
// max_rel_err plus noise_z standard errors), then flag bit
// LEARNED_FALLBACK on every global request of a flagged tile, whose index also
// goes to fallback_list (nreq entries of room, any order).
// counts[0] += flagged tiles, counts[1] += fallback requests (= list length).
// nreq_dev (optional): the request count on the device, nreq then a capacity.
cudaError_t learned_select(const CameraDev& cam, const Requests& R, int64_t nreq, const unsigned long long* nreq_dev,
                           int tile, int P, const uint32_t* preq, const float* probe_exact, const float* cached,
                           float max_rel_err, float noise_z, uint8_t* tile_flag, unsigned long long* counts,
                           uint32_t* fallback_list, int sm_count, cudaStream_t st);

// est = exact estimate for fallback requests, the cache's otherwise
cudaError_t learned_merge(const Requests& R, int64_t nreq, const unsigned long long* nreq_dev, const float* cached,
                          const float* exact, float* est, int sm_count, cudaStream_t st);

}  // namespace pm
