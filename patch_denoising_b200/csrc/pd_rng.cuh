// Counter-based standard normals shared by the Monte-Carlo kernels.
//
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) keyed by the 64-bit seed, counter (column group, row lo,
// row hi, draw); the four output words give four normals by the Box-Muller
// transform (hardware-approximate log / sin / cos: their error is far below the
// Monte-Carlo spread of the level), so element (r, c) of draw d is a pure
// function of (seed, d, r, c).
#pragma once
#include <stdint.h>

namespace pd {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

// 4 standard normals for (row, column group cg) of draw `draw`.
__device__ __forceinline__ void normals4(uint64_t seed, uint32_t draw, uint64_t row, uint32_t cg, float z[4]) {
  uint32_t c[4] = {cg, (uint32_t)row, (uint32_t)(row >> 32), draw};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    // u1 in (0, 1], u2 in [0, 1)
    const float u1 = ((float)c[2 * h] + 1.0f) * 2.3283064365386963e-10f;
    const float u2 = (float)c[2 * h + 1] * 2.3283064365386963e-10f;
    const float rad = sqrtf(-2.0f * __logf(u1));
    float sn, cs;
    __sincosf(6.283185307179586f * u2, &sn, &cs);
    z[2 * h] = rad * cs;
    z[2 * h + 1] = rad * sn;
  }
}

}  // namespace pd
