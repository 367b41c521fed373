// Shared device helpers of the FRW transition engine (sm_100a).
#pragma once

#include <cuda_fp16.h>
#include <math_constants.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/drwc.h"

#define DRWC_DEV __device__ __forceinline__

namespace drwc {

constexpr int kMaxRhs = 8;  // centre-source cells (even N: 8, odd N: 1 or 3)

// Philox4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32 multiplies
// with Weyl-sequence key bumps.
DRWC_DEV uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Two doubles in [0,1) (53 random bits each) for counter (stream, c2, c3).
DRWC_DEV double2 philox_uniform2(uint64_t seed, uint64_t stream, uint32_t c2, uint32_t c3) {
    uint4 o = philox4x32_10(make_uint4((uint32_t)stream, (uint32_t)(stream >> 32), c2, c3),
                            make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double s = 1.0 / 9007199254740992.0;
    double u0 = (double)((((uint64_t)(o.x >> 5)) << 26) | (uint64_t)(o.y >> 6)) * s;
    double u1 = (double)((((uint64_t)(o.z >> 5)) << 26) | (uint64_t)(o.w >> 6)) * s;
    return make_double2(u0, u1);
}

// Exactly rounded FP64 ops that the compiler may not contract into FMAs, so
// geometry matches a plain (non-contracted) CPU evaluation bit for bit.
DRWC_DEV double dadd(double a, double b) { return __dadd_rn(a, b); }
DRWC_DEV double dsub(double a, double b) { return __dsub_rn(a, b); }
DRWC_DEV double dmul(double a, double b) { return __dmul_rn(a, b); }
DRWC_DEV double ddiv(double a, double b) { return __ddiv_rn(a, b); }

}  // namespace drwc
