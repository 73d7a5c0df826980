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

MS_HD float2 cconjf(float2 a) { return make_float2(a.x, -a.y); }

// sin and cos of x (|x| < 1e4): Cody-Waite reduction by pi/2 with a
// three-part constant (products exact through FMA), then Taylor polynomials on
// [-pi/4, pi/4] (sin to r^9, cos to r^10: truncation below 2e-9) and the
// quadrant swap.  FMA-pipe only, no slow path: a few dozen instructions.
MS_D void sincos_red(float x, float* s, float* c) {
  const float k = rintf(x * 0.636619772f);
  float r = fmaf(-k, 1.5707963705062866f, x);
  r = fmaf(-k, -4.371138828673793e-08f, r);
  r = fmaf(-k, -1.7763568394002505e-15f, r);
  const float r2 = r * r;
  float ps = fmaf(r2, 2.7557319223985893e-06f, -1.984126984126984e-04f);
  ps = fmaf(r2, ps, 8.333333333333333e-03f);
  ps = fmaf(r2, ps, -0.16666666666666666f);
  const float sn = fmaf(r * r2, ps, r);
  float pc = fmaf(r2, -2.755731922398589e-07f, 2.48015873015873e-05f);
  pc = fmaf(r2, pc, -1.388888888888889e-03f);
  pc = fmaf(r2, pc, 4.1666666666666664e-02f);
  pc = fmaf(r2, pc, -0.5f);
  const float cs = fmaf(r2, pc, 1.0f);
  const int q = ((int)k) & 3;
  const float ss = (q & 1) ? cs : sn, cc = (q & 1) ? sn : cs;
  *s = (q & 2) ? -ss : ss;
  *c = ((q + 1) & 2) ? -cc : cc;
}

}  // namespace ms
