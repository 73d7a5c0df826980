// ms_common.cuh -- shared definitions of the B200 multislice engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MS_HD __host__ __device__ __forceinline__
#define MS_D __device__ __forceinline__

namespace ms {

// Number of xy bins per axis and z-bin height of the atom index; fixed by the
// reference (U.cu:1407-1409, "DONT CHANGE UNLESS CHANGE ELSEWHERE").
constexpr int kBins = 50;
constexpr int kBins2 = kBins * kBins;

MS_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
MS_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
MS_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
MS_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
MS_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// FP32 operations that the compiler may not contract into FMAs: the discrete
// decisions (bins, cut-offs, apertures) must round exactly as the host-side
// definition of the problem does.
MS_D float fmul_x(float a, float b) { return __fmul_rn(a, b); }
MS_D float fadd_x(float a, float b) { return __fadd_rn(a, b); }
MS_D float fsub_x(float a, float b) { return __fsub_rn(a, b); }
MS_D float fdiv_x(float a, float b) { return __fdiv_rn(a, b); }
MS_D float fsqrt_x(float a) { return __fsqrt_rn(a); }

}  // namespace ms
