/*
 * merlict_b200_philox.h -- counter-based uniforms shared by host and device.
 *
 * Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
 * random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
 * multiplications with the Weyl key schedule.  Photon `stream` draws its
 * k-th uniform from the block with counter (k, stream_lo, stream_hi, tag)
 * and key (seed_lo, seed_hi); the first two output words form 64 bits, of
 * which the top 53 become a double in [0, 1).
 *
 * The same inline function is compiled into the CUDA kernels, the CPU
 * oracle and the reference harness, so a photon traced on the GPU and the
 * same photon fed to merlict's Propagator through a replaying
 * random::Generator see identical uniforms.
 */
#ifndef MERLICT_B200_PHILOX_H_
#define MERLICT_B200_PHILOX_H_

#include <stdint.h>

#if defined(__CUDACC__)
#define MLGPU_HD __host__ __device__ __forceinline__
#else
#define MLGPU_HD static inline
#endif

#define MLGPU_PHILOX_M0 0xD2511F53u
#define MLGPU_PHILOX_M1 0xCD9E8D57u
#define MLGPU_PHILOX_W0 0x9E3779B9u
#define MLGPU_PHILOX_W1 0xBB67AE85u
#define MLGPU_PHILOX_TAG 0x6d6c6374u

MLGPU_HD uint64_t mlgpu_philox_bits(
    uint64_t seed, uint64_t stream, uint32_t k
) {
    uint32_t c0 = k;
    uint32_t c1 = (uint32_t)stream;
    uint32_t c2 = (uint32_t)(stream >> 32);
    uint32_t c3 = MLGPU_PHILOX_TAG;
    uint32_t k0 = (uint32_t)seed;
    uint32_t k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)MLGPU_PHILOX_M0 * (uint64_t)c0;
        const uint64_t p1 = (uint64_t)MLGPU_PHILOX_M1 * (uint64_t)c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += MLGPU_PHILOX_W0;
        k1 += MLGPU_PHILOX_W1;
    }
    return ((uint64_t)c0 << 32) | (uint64_t)c1;
}

/* Uniform in [0, 1) with 53 random bits. */
MLGPU_HD double mlgpu_philox_uniform(uint64_t seed, uint64_t stream, uint32_t k) {
    return (double)(mlgpu_philox_bits(seed, stream, k) >> 11) *
        (1.0 / 9007199254740992.0);
}

#endif  /* MERLICT_B200_PHILOX_H_ */
