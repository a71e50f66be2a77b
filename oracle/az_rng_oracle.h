/*
 * Oracle copy of the counter-based RNG (test infrastructure).
 *
 * Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11), restated from the paper: ten rounds of two 32x32
 * multiplies with the published round constants and Weyl key increments.
 *
 * The draw for (seed, pixel, sample, node, dim) is lane (dim & 3) of
 * Philox(counter = {pixel, sample, node.digits, node.level << 24 | dim >> 2},
 *        key = {seed lo, seed hi}), mapped to [0,1) as (x >> 8) * 2^-24.
 * This replaces azimuth's Random01 (src/azimuth_math.cpp:1-8, libc rand()).
 */
#ifndef AZ_RNG_ORACLE_H
#define AZ_RNG_ORACLE_H
#include <stdint.h>

static inline void az_oracle_philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1,
                                           uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float az_oracle_u01(uint64_t seed, uint32_t pixel, uint32_t sample,
                                  uint32_t digits, uint32_t level, uint32_t dim) {
    uint32_t ctr[4] = {pixel, sample, digits, (level << 24) | (dim >> 2)};
    uint32_t out[4];
    az_oracle_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), out);
    return (float)(out[dim & 3u] >> 8) * (1.0f / 16777216.0f);
}
#endif
