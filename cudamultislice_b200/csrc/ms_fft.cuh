// ms_fft.cuh -- register/shared-memory Stockham FFT of one line (row or column).
//
// A line of N = E * P complex points is owned by P consecutive threads of one
// warp (P <= 32); thread t holds element t + P*j in register j ("strided natural
// layout"), which makes global loads and stores of a line fully coalesced.
// The transform is two Stockham radix passes, N = E * P:
//   pass 1: radix-E butterfly entirely in registers (butterfly i = t);
//   exchange through the line's shared-memory slot (padded one point every E
//   so that the stride-E writes hit 32 distinct banks);
//   pass 2: E radix-P butterflies (E/P per thread) with twiddles W_N^{r*i}
//   read from a per-size table laid out [r][i] (coalesced, L1-resident); its
//   outputs land back in the strided natural layout, so the next pointwise
//   operation (transmission, propagator) needs no reordering.
// The in-register butterflies are radix-2 decimation-in-frequency networks
// with compile-time twiddle constants; trivial twiddles cost no multiply.
// Forward = exp(-2 pi i jk/N) (cuFFT CUFFT_FORWARD), both directions unnormalised.
#pragma once
#include "ms_common.cuh"

namespace ms {
namespace fft {

// cos(2 pi j / 32) for j = 0..8 (first quadrant); the rest follows by symmetry.
MS_HD constexpr float cos32_q(int j) {
  return j == 0 ? 1.0f
       : j == 1 ? 0.98078528040323043f
       : j == 2 ? 0.92387953251128674f
       : j == 3 ? 0.83146961230254524f
       : j == 4 ? 0.70710678118654757f
       : j == 5 ? 0.55557023301960229f
       : j == 6 ? 0.38268343236508984f
       : j == 7 ? 0.19509032201612833f
                : 0.0f;
}
MS_HD constexpr float cos32(int j) {
  return j <= 8 ? cos32_q(j) : j <= 16 ? -cos32_q(16 - j) : j <= 24 ? -cos32_q(j - 16) : cos32_q(32 - j);
}
MS_HD constexpr float sin32(int j) { return cos32((j + 24) & 31); }  // sin(a) = cos(a - pi/2)

MS_HD constexpr int brev(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}
MS_HD constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

// x * W_M^J, W = exp(-2 pi i / M) forward, exp(+2 pi i / M) inverse; M divides 32.
template <int J, int M, bool INV>
MS_D float2 twc(float2 x) {
  constexpr int j = ((J % M) + M) % M * (32 / M);
  if constexpr (j == 0) {
    return x;
  } else if constexpr (j == 16) {
    return make_float2(-x.x, -x.y);
  } else if constexpr (j == 8) {  // -i forward, +i inverse
    return INV ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
  } else if constexpr (j == 24) {  // +i forward, -i inverse
    return INV ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
  } else {
    constexpr float c = cos32(j);
    constexpr float s = INV ? sin32(j) : -sin32(j);
    return make_float2(x.x * c - x.y * s, x.x * s + x.y * c);
  }
}

// Radix-2 DIF network on R registers: natural-order input, bit-reversed output.
template <int R, int SPAN, bool INV>
struct Dif {
  template <int START, int J>
  static MS_D void bfly(float2 (&x)[R]) {
    const float2 a = x[START + J], b = x[START + J + SPAN];
    x[START + J] = cadd(a, b);
    x[START + J + SPAN] = twc<J, 2 * SPAN, INV>(csub(a, b));
    if constexpr (J + 1 < SPAN)
      bfly<START, J + 1>(x);
    else if constexpr (START + 2 * SPAN < R)
      bfly<START + 2 * SPAN, 0>(x);
  }
  static MS_D void run(float2 (&x)[R]) {
    bfly<0, 0>(x);
    if constexpr (SPAN > 1) Dif<R, SPAN / 2, INV>::run(x);
  }
};

template <int R, bool INV>
MS_D void dft(float2 (&x)[R]) {
  if constexpr (R > 1) Dif<R, R / 2, INV>::run(x);
}

// Split of a line length into registers per thread (E) and threads per line (P).
template <int N>
struct Plan;
template <> struct Plan<64>   { static constexpr int E = 8,  P = 8;  };
template <> struct Plan<128>  { static constexpr int E = 16, P = 8;  };
template <> struct Plan<256>  { static constexpr int E = 16, P = 16; };
template <> struct Plan<512>  { static constexpr int E = 32, P = 16; };
template <> struct Plan<1024> { static constexpr int E = 32, P = 32; };

// Shared-memory footprint of one line: N points plus one pad point every E,
// rounded so that consecutive lines start 8 points (mod 16) apart, which keeps
// two lines read by one 16-lane phase on disjoint banks.
template <int N>
MS_HD constexpr int line_stride() {
  constexpr int E = Plan<N>::E;
  constexpr int raw = N + N / E;
  return ((raw + 15) / 16) * 16 + 8;
}
template <int N>
MS_D int padi(int n) { return n + n / Plan<N>::E; }

// One N-point transform of the line held by threads t = 0..P-1 of a group.
// `sm` is this line's shared slot (line_stride<N>() points), `tw` the
// [r][i] twiddle table of size N (forward values; conjugated for INV).
// Every thread of the warp must call this (it issues __syncwarp()).
template <int N, bool INV>
MS_D void line_fft(float2 (&v)[Plan<N>::E], float2* __restrict__ sm, int t,
                   const float2* __restrict__ tw) {
  constexpr int E = Plan<N>::E, P = Plan<N>::P, LE = ilog2(E), LP = ilog2(P);
  static_assert(E * P == N && E % P == 0, "bad plan");
  // pass 1: radix-E on registers (Ns = 1, no twiddles)
  dft<E, INV>(v);
#pragma unroll
  for (int q = 0; q < E; ++q) sm[padi<N>(t * E + q)] = v[brev(q, LE)];
  __syncwarp();
  // pass 2: E radix-P butterflies, E/P per thread, then back to registers
#pragma unroll
  for (int b = 0; b < E / P; ++b) {
    const int i = t + P * b;
    float2 x[P];
#pragma unroll
    for (int r = 0; r < P; ++r) x[r] = sm[padi<N>(i + r * E)];
#pragma unroll
    for (int r = 1; r < P; ++r) {
      float2 w = __ldg(tw + r * E + i);
      if (INV) w.y = -w.y;
      x[r] = cmul(x[r], w);
    }
    dft<P, INV>(x);
#pragma unroll
    for (int q = 0; q < P; ++q) v[b + q * (E / P)] = x[brev(q, LP)];
  }
  __syncwarp();
}

}  // namespace fft
}  // namespace ms
