// ms_philox.h -- Philox4x32-10 counter-based generator (J. Salmon, M. Moraes,
// R. Dror, D. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11),
// used for reproducible thermal (frozen-phonon) displacements and detector noise.
#pragma once
#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define MS_PHILOX_HD __host__ __device__ inline
#else
#define MS_PHILOX_HD inline
#endif

namespace ms {

MS_PHILOX_HD void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;  // round multipliers
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // Weyl key increments
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    if (round > 0) {
      k0 += W0;
      k1 += W1;
    }
    const uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Standard normal from two 32-bit words by the Box-Muller form of the
// reference's noise (U.cu:2389-2397): u = r * 2^-32 in [0, 1),
// z = sqrt(-2 log(FLT_MIN + u1)) sin(6.2831852 u2) in FP64, clipped to [-3, 3].
MS_PHILOX_HD double clipped_normal(uint32_t r1, uint32_t r2) {
  const double u1 = (double)r1 * 2.3283064365386963e-10, u2 = (double)r2 * 2.3283064365386963e-10;
  double z = sqrt(-2.0 * log(1.17549435e-38 + u1)) * sin((double)(2.0f * 3.1415926f) * u2);
  if (z <= -3.0) z = -3.0;
  if (z >= 3.0) z = 3.0;
  return z;
}

}  // namespace ms
