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

// Packed FP32x2 arithmetic of sm_100 (PTX add/mul/fma.rn.f32x2: two
// independent, correctly rounded FP32 operations in one instruction) on pairs
// held in 64-bit registers (low half = first value).
typedef unsigned long long f2p;
MS_D f2p pk2(float lo, float hi) {
  f2p r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
MS_D void up2(f2p v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
MS_D f2p add2(f2p a, f2p b) {
  f2p d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
MS_D f2p mul2(f2p a, f2p b) {
  f2p d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
MS_D f2p fma2(f2p a, f2p b, f2p c) {
  f2p d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// sin and cos of two values at once: sincos_red with its polynomial and
// reduction steps on the packed FP32x2 pipe.  Each lane rounds exactly as the
// scalar fmaf/multiply of sincos_red does, so the results are bit-identical.
MS_D void sincos_red2(float x0, float x1, float* s0, float* c0, float* s1, float* c1) {
  const f2p x = pk2(x0, x1);
  float q0, q1;
  up2(mul2(x, pk2(0.636619772f, 0.636619772f)), q0, q1);
  const float k0 = rintf(q0), k1 = rintf(q1);
  const f2p nk = pk2(-k0, -k1);
  f2p r = fma2(nk, pk2(1.5707963705062866f, 1.5707963705062866f), x);
  r = fma2(nk, pk2(-4.371138828673793e-08f, -4.371138828673793e-08f), r);
  r = fma2(nk, pk2(-1.7763568394002505e-15f, -1.7763568394002505e-15f), r);
  const f2p r2 = mul2(r, r);
  f2p ps = fma2(r2, pk2(2.7557319223985893e-06f, 2.7557319223985893e-06f),
                pk2(-1.984126984126984e-04f, -1.984126984126984e-04f));
  ps = fma2(r2, ps, pk2(8.333333333333333e-03f, 8.333333333333333e-03f));
  ps = fma2(r2, ps, pk2(-0.16666666666666666f, -0.16666666666666666f));
  const f2p sn = fma2(mul2(r, r2), ps, r);
  f2p pc = fma2(r2, pk2(-2.755731922398589e-07f, -2.755731922398589e-07f),
                pk2(2.48015873015873e-05f, 2.48015873015873e-05f));
  pc = fma2(r2, pc, pk2(-1.388888888888889e-03f, -1.388888888888889e-03f));
  pc = fma2(r2, pc, pk2(4.1666666666666664e-02f, 4.1666666666666664e-02f));
  pc = fma2(r2, pc, pk2(-0.5f, -0.5f));
  const f2p cs = fma2(r2, pc, pk2(1.0f, 1.0f));
  float sa, sb, ca, cb;
  up2(sn, sa, sb);
  up2(cs, ca, cb);
  const int qa = ((int)k0) & 3, qb = ((int)k1) & 3;
  const float ssa = (qa & 1) ? ca : sa, cca = (qa & 1) ? sa : ca;
  const float ssb = (qb & 1) ? cb : sb, ccb = (qb & 1) ? sb : cb;
  *s0 = (qa & 2) ? -ssa : ssa;
  *c0 = ((qa + 1) & 2) ? -cca : cca;
  *s1 = (qb & 2) ? -ssb : ssb;
  *c1 = ((qb + 1) & 2) ? -ccb : ccb;
}

// sincos_red2 for arguments whose quarter-turn count is 0 (|x * 2/pi| <= 0.5
// as sincos_red2 rounds the product, so rint gives 0): the reduction steps are
// then exact identities and the quadrant swap does nothing, so the polynomials
// alone give bit-identical results.
MS_D bool sincos_small_ok(float x) { return fabsf(x * 0.636619772f) <= 0.5f; }
MS_D void sincos_small2(float x0, float x1, float* s0, float* c0, float* s1, float* c1) {
  const f2p r = pk2(x0, x1);
  const f2p r2 = mul2(r, r);
  f2p ps = fma2(r2, pk2(2.7557319223985893e-06f, 2.7557319223985893e-06f),
                pk2(-1.984126984126984e-04f, -1.984126984126984e-04f));
  ps = fma2(r2, ps, pk2(8.333333333333333e-03f, 8.333333333333333e-03f));
  ps = fma2(r2, ps, pk2(-0.16666666666666666f, -0.16666666666666666f));
  const f2p sn = fma2(mul2(r, r2), ps, r);
  f2p pc = fma2(r2, pk2(-2.755731922398589e-07f, -2.755731922398589e-07f),
                pk2(2.48015873015873e-05f, 2.48015873015873e-05f));
  pc = fma2(r2, pc, pk2(-1.388888888888889e-03f, -1.388888888888889e-03f));
  pc = fma2(r2, pc, pk2(4.1666666666666664e-02f, 4.1666666666666664e-02f));
  pc = fma2(r2, pc, pk2(-0.5f, -0.5f));
  const f2p cs = fma2(r2, pc, pk2(1.0f, 1.0f));
  up2(sn, *s0, *s1);
  up2(cs, *c0, *c1);
}

}  // namespace ms
