// qx_philox.h -- Philox4x32-10 counter-based generator, host and device.
// Written from Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy
// as 1, 2, 3" (SC'11): multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
// increments 0x9E3779B9 / 0xBB67AE85, 10 rounds.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define QX_HD __host__ __device__ __forceinline__
#else
#define QX_HD inline
#endif

namespace qx {

struct U4 {
    uint32_t v[4];
};

QX_HD U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    U4 o;
    o.v[0] = c0;
    o.v[1] = c1;
    o.v[2] = c2;
    o.v[3] = c3;
    return o;
}

// uniform in (0, 1): (w + 1/2) / 2^32
QX_HD double u01(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

}  // namespace qx
