// Pre-include for compiling the reference's photon tracer (CPM/PhotonTracing.cu
// and the device functions it calls) as HOST code, for the tracer pin of the
// oracle.  TEST INFRASTRUCTURE ONLY; it changes no reference file.
//
// nvcc compiles a .cu file twice: once for the device (__CUDA_ARCH__ defined)
// and once for the host.  ref_trace.cu includes the reference only in the host
// pass, and in that pass this file turns the reference's device-only code into
// plain host code:
//  * __device__, __constant__ and __shared__ expand to nothing, so `trace`,
//    `destiny`, `Model::gpu_get_random_point_with_normal`,
//    `Ray::reflect_spherical`, ... become host functions and the reference's
//    __device__ / __constant__ globals become host globals;
//  * threadIdx / blockIdx / blockDim read per-host-thread values, so one
//    OpenMP thread plays one reference thread (its slot in the reference's
//    per-thread arrays);
//  * curand_uniform(state) draws the next uniform of the photon path the
//    calling host thread is tracing (the injected per-path Philox stream
//    shared with the oracle and the CUDA kernels);
//  * the CUDA runtime calls the reference's host set-up makes
//    (cudaMalloc / cudaMemcpy / cudaMemcpyToSymbol / cudaFree) act on host
//    memory (and cudaGetLastError reports success), and the device atomics the included headers name act on plain
//    host integers (they run on one host thread per slot).
// Kernels (__global__) keep their qualifier: their bodies are never run here.
//
// In the device pass the reference stays device code (its vec3 rounds toward
// zero, CPM/vec3.cuh:18-20: the reference's GPU numerics), with two changes
// for the harness kernel of ref_trace.cu that runs it on the GPU, one path per
// thread: curand_uniform(state) draws the calling thread's injected path
// stream, and __constant__ globals become __device__ globals, so that the
// harness's set-up kernel can give them their values (the reference sets them
// with cudaMemcpyToSymbol from its host code).
#include "shim.h"
#include <device_launch_parameters.h>
#include <cstdint>
#include <cstdlib>
#include <unordered_set>

// CPM/PhotonTracing.cu:386 passes the kernel `emit` as a void* (an implicit
// function-to-object pointer conversion MSVC accepts); route it through a cast.
int calculate_max_blocks_number(int threads_per_block, void* kernel_func);
template <class F> int calculate_max_blocks_number(int t, F* f) { return calculate_max_blocks_number(t, (void*)f); }

#ifndef __CUDA_ARCH__
extern thread_local uint3 pm_ref_thread_idx;
extern thread_local uint3 pm_ref_block_idx;
extern thread_local dim3 pm_ref_block_dim;
float pm_ref_uniform();

template <class T> inline cudaError_t pm_ref_malloc(T** p, size_t n) {
    *p = (T*)std::calloc(n ? n : 1, 1);
    return cudaSuccess;
}
inline cudaError_t pm_ref_free(void* p) { std::free(p); return cudaSuccess; }
inline cudaError_t pm_ref_memcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) {
    std::memcpy(dst, src, n);
    return cudaSuccess;
}
template <class T> inline cudaError_t pm_ref_memcpy_to_symbol(T& symbol, const void* src, size_t n, size_t off = 0,
                                                              cudaMemcpyKind = cudaMemcpyHostToDevice) {
    std::memcpy((char*)&symbol + off, src, n);
    return cudaSuccess;
}
inline unsigned pm_ref_atomic_add(unsigned* a, unsigned v) { unsigned o = *a; *a = o + v; return o; }
inline int pm_ref_atomic_add(int* a, int v) { int o = *a; *a = o + v; return o; }
inline int pm_ref_atomic_cas(int* a, int cmp, int v) { int o = *a; if (o == cmp) *a = v; return o; }
inline int pm_ref_atomic_exch(int* a, int v) { int o = *a; *a = v; return o; }

#undef __device__
#define __device__
#undef __constant__
#define __constant__
#undef __shared__
#define __shared__
#define threadIdx pm_ref_thread_idx
#define blockIdx pm_ref_block_idx
#define blockDim pm_ref_block_dim
#define curand_uniform(state) pm_ref_uniform()
#define cudaMalloc pm_ref_malloc
#define cudaFree pm_ref_free
#define cudaMemcpy pm_ref_memcpy
#define cudaMemcpyToSymbol pm_ref_memcpy_to_symbol
#define cudaGetLastError() cudaSuccess
#define atomicAdd pm_ref_atomic_add
#define atomicCAS pm_ref_atomic_cas
#define atomicExch pm_ref_atomic_exch
#else
__device__ float pm_ref_dev_uniform();
#define curand_uniform(state) pm_ref_dev_uniform()
#undef __constant__
#define __constant__ __device__
#endif
