// ms_ctf.cuh -- objective-lens transfer weight shared by the fused column
// pass and the plain imaging path.
#pragma once
#include "ms_common.cuh"

namespace ms {

// E_s E_d exp(-i chi) * scale at spatial frequency (kx, ky), following
// imagingKernel2 (U.cu:1044-1080): zero outside k^2 < objap2 (FP32 decision),
// chi = pi lambda k^2 (Cs lambda^2 k^2 / 2 + df + A2 sin 2(phi - phi2)
//       + 2/3 A3 lambda k sin 3(phi - phi3)),
// E_s = exp(-beta^2/(4 lambda^2) (2 pi lambda k df + 2 pi lambda^3 Cs k^3)^2),
// E_d = exp(-delta^2 pi^2 lambda^2 k^4 / 4),
// with the reference's pi literals.  Phase and envelopes are evaluated in
// FP64 and the phase is reduced modulo 2 pi before the FP32 sincos.
__device__ __forceinline__ float2 ctf_weight(double lam, double Cs, double df, double A2, double phi2,
                                             double A3, double phi3, double beta, double delta,
                                             float objap2, float kxf, float kyf, float scale) {
  const float k2f = fadd_x(fmul_x(kxf, kxf), fmul_x(kyf, kyf));
  if (!(k2f < objap2)) return make_float2(0.f, 0.f);
  const double kx = kxf, ky = kyf, k2 = kx * kx + ky * ky, k = sqrt(k2);
  const double factor = beta * beta / (4.0 * lam * lam);
  const double a1 = 3.141593 * k * lam * 2.0 * df + 2.0 * 3.141593 * lam * lam * lam * Cs * k2 * k;
  const double es = exp(-factor * a1 * a1);
  const double ed = exp(-0.25 * delta * delta * 3.141593 * 3.141593 * k2 * k2 * lam * lam);
  const double phi = atan2(ky, kx);
  const double chi = 3.1415926 * lam * k2 *
                     (0.5 * Cs * lam * lam * k2 + df + A2 * sin(2.0 * (phi - phi2)) +
                      2.0 * A3 * lam * sqrt(k2) * sin(3.0 * (phi - phi3)) / 3.0);
  const double twopi = 6.283185307179586;
  const float chr = (float)(chi - twopi * rint(chi / twopi));
  float s, c;
  sincosf(chr, &s, &c);
  const float amp = (float)(es * ed) * scale;
  return make_float2(amp * c, -amp * s);
}

}  // namespace ms
