// Counter-based random numbers: Philox-4x32 with 10 rounds (Salmon, Moraes,
// Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011).
// A job's stream is addressed by (key = job seed, counter = event index), so
// the numbers a replica draws depend only on the job, the replica and the
// proposal index -- never on the CTA, slot or batch that runs it.
#pragma once
#include <cstdint>

namespace sqs {

struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;  // round multipliers
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // key schedule (Weyl) increments
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t h0 = mulhi32(M0, c.x), l0 = M0 * c.x;
        const uint32_t h1 = mulhi32(M1, c.z), l1 = M1 * c.z;
        c = U4{h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform in (0, 1) from 24 random bits
__host__ __device__ __forceinline__ float u01(uint32_t v) { return ((float)(v >> 8) + 0.5f) * (1.0f / 16777216.0f); }

}  // namespace sqs
