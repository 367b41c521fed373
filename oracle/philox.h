/* TEST INFRASTRUCTURE ONLY (CPU checker).
 *
 * Philox4x32-10 counter-based generator, restated from its published
 * description (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the round
 * constants 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 /
 * 0xBB67AE85. The device library carries its own implementation; the tests
 * compare the two stream for stream.
 *
 * The reference samples with torch::multinomial (dnn_solver_poisson.cpp:92,
 * 107), whose generator is not part of its interface; walks here are keyed
 * instead so that every walk's draws are independent of batching.
 */
#ifndef ORC_PHILOX_H
#define ORC_PHILOX_H
#include <stdint.h>

static inline void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                     uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
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

/* Two doubles in [0,1) with 53 random bits each from one Philox block. */
static inline void orc_philox_uniform2(uint64_t seed, uint64_t stream, uint32_t c2, uint32_t c3,
                                       double* u0, double* u1) {
    uint32_t ctr[4] = {(uint32_t)stream, (uint32_t)(stream >> 32), c2, c3};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    const double s = 1.0 / 9007199254740992.0; /* 2^-53 */
    *u0 = (double)(((uint64_t)(o[0] >> 5) << 26) | (uint64_t)(o[1] >> 6)) * s;
    *u1 = (double)(((uint64_t)(o[2] >> 5) << 26) | (uint64_t)(o[3] >> 6)) * s;
}
#endif
