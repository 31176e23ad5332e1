// pm_device.cuh -- device-side building blocks shared by the photon-mapping kernels.
//
// Arithmetic contract of every kernel in this library: IEEE binary32 with
// round-to-nearest, correctly rounded division and square root, and no FMA
// contraction (the library is compiled with --fmad=false).  Vector
// expressions are evaluated in the operation order of the reference's vec3
// (CudaPhotonMapping/vec3.cuh), so positions, directions and every decision
// taken on them (rejection loops, Russian roulette, kNN membership) agree bit
// for bit with a host build of the same expressions.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pm {

// ------------------------------------------------------------ status word --
// Kernels never trap: they record the first problem in a device status word
// that the host reads after the launch sequence.
enum StatusBits : unsigned {
    ST_TIMEOUT = 1u,         // a bounded spin (decoupled look-back) gave up
    ST_OVERFLOW = 2u,        // a fixed-capacity buffer would have overflowed
    ST_STACK = 4u,           // a per-thread stack exceeded its capacity
    ST_BAD_INPUT = 8u,       // an index read from memory was out of range
};
__device__ __forceinline__ void raise_status(unsigned* status, unsigned bit) {
    if (status) atomicOr(status, bit);
}

// ------------------------------------------------------------------ vec3 --
struct V3 { float x, y, z; };
__host__ __device__ __forceinline__ V3 v3(float a, float b, float c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 vscale(V3 a, float t) { return v3(t * a.x, t * a.y, t * a.z); }
__device__ __forceinline__ V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float vlength(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ bool vnull(V3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
// reciprocal-multiply normalisation (the member vec3::normalize)
__device__ __forceinline__ V3 vnorm_recip(V3 a) {
    if (vnull(a)) return a;
    float u = 1.0f / vlength(a);
    return v3(a.x * u, a.y * u, a.z * u);
}
// divide-by-length normalisation (the static vec3::normalize)
__device__ __forceinline__ V3 vnorm_div(V3 a) {
    if (vnull(a)) return a;
    float l = vlength(a);
    return v3(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ float vmax3(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
// three-source float min / max (PTX min.f32 / max.f32 with three inputs,
// sm_100 and later): one instruction for two fminf / fmaxf, the same value
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ V3 vmin1(V3 a, float m) { return v3(fminf(a.x, m), fminf(a.y, m), fminf(a.z, m)); }
__device__ __forceinline__ bool vnear(V3 a, V3 b) {   // |a - b| < 1e-3 per component
    return fabsf(a.x - b.x) < 0.001f && fabsf(a.y - b.y) < 0.001f && fabsf(a.z - b.z) < 0.001f;
}
__device__ __forceinline__ V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ void st3(float* p, V3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }

// --------------------------------------------------------------- Philox --
// Philox-4x32-10 (Salmon et al., SC'11).  Draw i of stream (seed, tag, path) is
// word (i & 3) of Philox(counter = (i >> 2, path_lo, path_hi, tag), key = seed).
__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}
// uniform in (0, 1]
__device__ __forceinline__ float unit_from_u32(uint32_t x) {
    return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

struct Stream {
    uint32_t k0, k1, plo, phi, tag;
    uint32_t n;
    uint4 buf;
    __device__ __forceinline__ void init(uint64_t seed, uint64_t path, uint32_t t) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        plo = (uint32_t)path; phi = (uint32_t)(path >> 32); tag = t; n = 0;
    }
    __device__ __forceinline__ float next() {
        if ((n & 3u) == 0u) buf = philox10(make_uint4(n >> 2, plo, phi, tag), k0, k1);
        uint32_t w = (n & 3u) == 0u ? buf.x : (n & 3u) == 1u ? buf.y : (n & 3u) == 2u ? buf.z : buf.w;
        ++n;
        return unit_from_u32(w);
    }
};

// ------------------------------------------------------------- warp util --
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace pm
