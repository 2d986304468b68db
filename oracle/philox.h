/*
 * philox.h -- Philox4x32-10 counter-based generator for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY: this header belongs to the oracle (the CPU
 * restatement used to check the CUDA path).  The product keeps its own device
 * implementation in szsnn_b200/csrc/common.cuh; both follow the published
 * algorithm of Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11 (Philox-4x32, 10 rounds).  The two are compared
 * bit-for-bit by the parity tests.
 *
 * Stream conventions shared by oracle and device (the reference has no RNG on
 * its hot path; its only source model, Const_rate, is periodic):
 *   Poisson source draw : ctr = {index in population, step_lo, step_hi, 0x504F4953}, key = seed
 *   network generator   : ctr = {row in block, k, block_stream, 0x53594E47}, key = seed
 *   uniform float       : (r >> 8) * 2^-24, exact in fp32, range [0, 1)
 *   bounded integer     : (uint32)(((uint64)r * range) >> 32)
 */
#ifndef SZSNN_ORACLE_PHILOX_H
#define SZSNN_ORACLE_PHILOX_H
#include <stdint.h>

#define ORC_PHILOX_M0 0xD2511F53u
#define ORC_PHILOX_M1 0xCD9E8D57u
#define ORC_PHILOX_W0 0x9E3779B9u
#define ORC_PHILOX_W1 0xBB67AE85u

#define ORC_STREAM_POISSON 0x504F4953u
#define ORC_STREAM_GEN     0x53594E47u

typedef struct { uint32_t v[4]; } orc_u32x4;

static inline orc_u32x4 orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                   uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)ORC_PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)ORC_PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += ORC_PHILOX_W0; k1 += ORC_PHILOX_W1;
    }
    orc_u32x4 o = {{c0, c1, c2, c3}};
    return o;
}

static inline float orc_u24(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }

static inline uint32_t orc_bounded(uint32_t r, uint32_t range)
{
    return (uint32_t)(((uint64_t)r * (uint64_t)range) >> 32);
}

#endif
