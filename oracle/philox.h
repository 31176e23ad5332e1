// philox.h -- the injected per-path random stream (TEST INFRASTRUCTURE ONLY).
//
// Shared by the oracle (pm_oracle.cpp) and the reference tracer harness
// (ref_host/ref_trace.cu), so both consume exactly the stream the CUDA kernels
// draw: it replaces curand (CPM/CudaRandom.cu:6-11) with a counter-based stream
// per photon path.  Pinned by the Random123 known-answer vectors in the tests.
#pragma once
#include <cstdint>

// callable from device code where nvcc compiles this file (the reference
// tracer harness runs the reference's device functions on the GPU too)
#ifdef __CUDACC__
#define ORACLE_HD __host__ __device__
#else
#define ORACLE_HD
#endif

namespace oracle_rng {

// ------------------------------------------------------------- Philox -------
// Philox-4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11: multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key increments
// 0x9E3779B9 / 0xBB67AE85, ten rounds.
ORACLE_HD inline void philox10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
// uniform in (0,1]: ((x >> 8) + 1) * 2^-24, exact in binary32.
ORACLE_HD inline float u32_to_unit(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

// The injected stream of one photon path: draw i of path p under (seed, tag) is
// word (i & 3) of Philox(counter = (i >> 2, p_lo, p_hi, tag), key = (seed_lo, seed_hi)).
struct Stream {
    uint32_t k0, k1, plo, phi, tag;
    uint32_t n = 0, block = 0xffffffffu;
    uint32_t out[4];
    ORACLE_HD Stream(uint64_t seed, uint64_t path, uint32_t t)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), plo((uint32_t)path), phi((uint32_t)(path >> 32)), tag(t) {}
    ORACLE_HD float next() {
        uint32_t b = n >> 2;
        if (b != block) {
            out[0] = b; out[1] = plo; out[2] = phi; out[3] = tag;
            philox10(out, k0, k1);
            block = b;
        }
        float u = u32_to_unit(out[n & 3]);
        ++n;
        return u;
    }
};

}  // namespace oracle_rng
