// pm_mlp.cuh -- learned radiance cache: a small MLP on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory).
//
// Network: the hit point (3, normalised to the scene box) and the octahedral
// shading normal (2) are encoded with sin / cos at 6 octaves each (60 inputs,
// padded to 64), then 4 hidden layers of width 64 with ReLU and an RGB output
// (padded to 16):  64 -> 64 -> 64 -> 64 -> 64 -> 16.  Octaves f = octave0 ..
// octave0 + 5 (octave0 = 0 by default).  Weights are FP32 master
// copies updated by Adam; the kernels read BF16 copies.  Activations and
// gradients between layers are BF16; every product accumulates in FP32.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace pm {

constexpr int MLP_LAYERS = 5;
constexpr int MLP_DIM = 64;                       // padded input width = hidden width
constexpr int MLP_OUT = 16;                       // padded output width (RGB used)
constexpr int MLP_FEATURES = 60;                  // encoded inputs
constexpr int MLP_LAYER_STRIDE = MLP_DIM * MLP_DIM;
constexpr int MLP_PARAMS = MLP_LAYERS * MLP_LAYER_STRIDE;   // [layer][out][in], layer 4 uses out < 16

__host__ __device__ constexpr int mlp_out_dim(int l) { return l == MLP_LAYERS - 1 ? MLP_OUT : MLP_DIM; }

struct MlpNet {
    const __nv_bfloat16* w;     // MLP_PARAMS bf16 weights
    float lo[3], inv[3];        // encoding box: u = (p - lo) * inv
    float freq0;                // lowest encoding frequency multiplier: 2^octave0
    float out_scale;            // radiance = out_scale * network output
};

// Inputs: n samples, either 3-float position / normal arrays or float4
// request records (xyz; in rec_nrm the w bits hold flags, a record is used
// when (flags & flag_mask) != 0).
struct MlpInputs {
    int64_t n;
    const float* pos3;
    const float* nrm3;
    const float4* rec_pos;
    const float4* rec_nrm;
    uint32_t flag_mask;
    // optional, for launches whose sizes live on the device (graph replay):
    const unsigned long long* n_dev;   // inference: min(*n_dev, n) samples (n a capacity)
    const int64_t* base_dev;           // training on pos3 / nrm3: sample i is array entry *base_dev + i
    int64_t base_wrap;                 // > 0: a base with base + n > base_wrap reads from entry 0 instead
};

// One training pass over n samples: accumulates d(loss)/d(weights) into grad
// (MLP_PARAMS floats, zeroed by the caller) and sum(weight * |y - t|^2) into
// *loss_sum, where loss = grad_scale / 2 * sum over samples and channels of
// weight * (y - target / out_scale)^2.  target: 3 floats per sample;
// weight: 1 float per sample or null (all 1).
cudaError_t mlp_train(const MlpNet& net, const MlpInputs& in, const float* target, const float* weight,
                      float grad_scale, float* grad, float* loss_sum, unsigned* status, int sm_count,
                      cudaStream_t st);

// Network outputs (3 floats per sample, times out_scale); unused records get 0.
cudaError_t mlp_infer(const MlpNet& net, const MlpInputs& in, float* out, unsigned* status, int sm_count,
                      cudaStream_t st);

// Adam step on the FP32 master weights; refreshes the BF16 copies and zeroes grad.
cudaError_t mlp_adam(float* w32, __nv_bfloat16* w16, float* grad, float* m, float* v, int step, float lr,
                     float beta1, float beta2, float eps, cudaStream_t st);

// The same with the step number on the device: *step_dev += 1 (unless
// increment is false: the caller advanced it), then the step uses it for the
// bias corrections (a replayed graph advances it itself).
cudaError_t mlp_adam_dev(float* w32, __nv_bfloat16* w16, float* grad, float* m, float* v, int* step_dev, float lr,
                         float beta1, float beta2, float eps, cudaStream_t st, bool increment = true);

// BF16 copies of FP32 weights.
cudaError_t mlp_to_bf16(const float* w32, __nv_bfloat16* w16, cudaStream_t st);

}  // namespace pm
