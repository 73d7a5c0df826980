// ms_slice_loop.cuh -- the whole conventional slice loop of one instance in
// one persistent cooperative kernel.
//
// The two-pass slice step of ms_slice_impl.cuh (row pass: IFFT_row ->
// x exp(i sigma V) -> FFT_row; column pass: FFT_col -> x P(k)/N -> IFFT_col)
// runs here for all S slices inside a single launch.  Every CTA is resident
// for the whole loop (cooperative launch, one CTA per SM): between the phases
// the CTAs meet at a grid barrier instead of a kernel boundary, so a slice
// costs no launch, ramp-up or drain, the frequency tables stay in shared
// memory, and the next slice's potential rows are prefetched into L2 while
// the column phase runs.
//
// Work split (lines of N points, one warp per line, E = N/32 points per
// thread): row r goes to CTA r % G, warp r / G; column unit u (CW adjacent
// columns, CW warps interleaved so that every warp access covers whole 32-byte
// sectors) to CTA u % G, group u / G.  A wave of 1024^2 puts at most 7 rows
// and 8 columns on one SM per phase.
//
// Grid barrier: a monotonic arrival counter (zeroed before each launch); the
// k-th barrier waits for k * G arrivals.  Each wait is bounded by a time limit
// (default one second, %globaltimer): a CTA that runs out sets the error word
// and returns, and the others see the error word and return too, so a lost
// arrival ends the kernel with an error status instead of a hang.
#pragma once
#include "ms_slice_impl.cuh"

namespace ms {

MS_D unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barrier number `epoch` (1, 2, ...).  Returns false (in every thread of
// the CTA) when the grid must stop: this CTA's wait ran out or another CTA
// reported an error.  TIGHT = false: the arrival is an atomic add and the
// wait polls with a short sleep; TIGHT = true: the arrival is a release
// reduction (no round trip) and the wait polls back to back, checking the
// clock and the error word every 32 polls.
template <bool TIGHT>
MS_D bool loop_barrier(const LoopSync& s, unsigned int epoch) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    __threadfence();
    if constexpr (TIGHT)
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(s.count) : "memory");
    else
      atomicAdd(s.count, 1u);
    const unsigned int target = epoch * gridDim.x + s.expect_extra;
    const unsigned long long t0 = global_ns();
    for (unsigned int it = 0;; ++it) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(s.count) : "memory");
      if (v >= target) break;
      if (!TIGHT || (it & 31) == 31) {
        if (*reinterpret_cast<volatile int*>(s.error) != 0) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > s.limit_ns) {
          atomicExch(s.error, kLoopTimeout);
          ok = 0;
          break;
        }
      }
      if constexpr (!TIGHT) __nanosleep(32);
    }
    __threadfence();
  }
  return __syncthreads_and(ok) != 0;
}

template <class PL, int CW>
struct LoopShape {
  static constexpr int N = PL::N, E = PL::E, P = PL::P;
  static_assert(P == 32, "the persistent loop runs one warp per line");
  static constexpr int NT = 256;                 // threads per CTA
  static constexpr int WARPS = NT / 32;          // rows per CTA per round
  static constexpr int GS = CW * P;              // threads of one column unit
  static constexpr int GROUPS = NT / GS;         // column units per CTA per round
  static constexpr int ROW_SLOT = PL::SLOT;
  static constexpr int COL_SLOT = ((N + N / PL::R1 + 15) / 16) * 16 + 16 / CW;
  static constexpr int EXCH = (WARPS * ROW_SLOT > GROUPS * CW * COL_SLOT) ? WARPS * ROW_SLOT : GROUPS * CW * COL_SLOT;
  // exchange slots, then ky (N floats, padded to float2) and py (N float2)
  static constexpr size_t SMEM = ((size_t)EXCH + (N + 1) / 2 + N) * sizeof(float2);
};

// Row phase of one line: [IFFT_row] -> x exp(i sigma V) -> FFT_row, in place
// on the wave (or from psi0 on the first slice).
template <class PL, bool INV>
MS_D void loop_row(const PassAArgs& a, const float2* in, float2* out, const float* __restrict__ V, int line, int t,
                   float2* sm) {
  constexpr int NX = PL::N, E = PL::E, P = PL::P;
  const long long row0 = (long long)line * NX;
  float2 v[E];
  float vv[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = in[row0 + t + P * j];
#pragma unroll
  for (int j = 0; j < E; ++j) vv[j] = V[row0 + t + P * j];
  if constexpr (INV) {
    fft::conj_all(v);
    fft::line_fft<PL>(v, sm, t, a.tw);
    fft::conj_all(v);
  }
#pragma unroll
  for (int j = 0; j < E; j += 2) {
    float s0, c0, s1, c1;
    sincos_red2(fmul_x(a.sigma, vv[j]), fmul_x(a.sigma, vv[j + 1]), &s0, &c0, &s1, &c1);
    v[j] = cmul(v[j], make_float2(c0, s0));
    v[j + 1] = cmul(v[j + 1], make_float2(c1, s1));
  }
  fft::line_fft<PL>(v, sm, t, a.tw);
#pragma unroll
  for (int j = 0; j < E; ++j) out[row0 + t + P * j] = v[j];
}

// Column phase of one unit of CW columns starting at c0: FFT_col -> x P/N
// (band-limited) -> IFFT_col, in place.
template <class PL, int CW>
MS_D void loop_col(const PassBArgs& b, float2* wave, int c0, int cl, int t, float2* sm,
                   const float* __restrict__ sky, const float2* __restrict__ spy) {
  using SH = LoopShape<PL, CW>;
  constexpr int E = PL::E, P = PL::P, GS = SH::GS;
  const int nx = b.nx;
  const int col = c0 + cl;
  const float2* src = wave + (long long)t * nx + col;
  const int step = P * nx;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = src[j * step];
#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    fft::line_fft<fft::PaddedPlan<PL>, GS>(v, sm, t, b.tw);
    if (it == 0) {
      col_mid<PL, B_PROPAGATE>(v, b, sky, spy, col, t, 0);
      fft::conj_all(v);
    } else {
      fft::conj_all(v);
    }
  }
  int ostep;
  asm volatile("mov.b32 %0, %1;" : "=r"(ostep) : "r"(step));
  float2* dst = wave + (long long)t * nx + col;
#pragma unroll
  for (int j = 0; j < E; ++j) dst[j * ostep] = v[j];
}

// Bulk L2 prefetch of the potential rows this CTA's warps read in the next
// row phase (issued during the column phase; one 4-byte-per-point row each).
template <class PL>
MS_D void prefetch_rows(const float* V, int G) {
  constexpr int NX = PL::N;
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int line = w * G + blockIdx.x;
  if (lane == 0 && line < NX) {
    const float* p = V + (long long)line * NX;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"((unsigned)(NX * sizeof(float)))
                 : "memory");
  }
}

template <class PL, int CW, bool TIGHT>
__global__ void __launch_bounds__(256, 1) k_slice_loop(LoopArgs L) {
  using SH = LoopShape<PL, CW>;
  constexpr int N = PL::N, GS = SH::GS, GROUPS = SH::GROUPS;
  extern __shared__ float2 smem[];
  float* sky = reinterpret_cast<float*>(smem + SH::EXCH);
  float2* spy = smem + SH::EXCH + (N + 1) / 2;
  for (int i = threadIdx.x; i < N; i += SH::NT) {
    sky[i] = L.b.ky[i];
    spy[i] = L.b.py[i];
  }
  __syncthreads();
  const int G = gridDim.x;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // this thread's column-unit coordinates
  const int g = threadIdx.x / GS, gr = threadIdx.x % GS;
  const int cl = gr % CW, t = gr / CW;
  unsigned int epoch = 0;
  for (int s = 0; s < L.S; ++s) {
    const float* V = L.Vstack + (long long)s * L.vstride;
    // ---- row phase ----
    for (int line = warp * G + blockIdx.x; line < N; line += SH::WARPS * G) {
      float2* sm = smem + warp * SH::ROW_SLOT;
      if (s == 0)
        loop_row<PL, false>(L.a, L.psi0, L.wave, V, line, lane, sm);
      else
        loop_row<PL, true>(L.a, L.wave, L.wave, V, line, lane, sm);
    }
    if (!loop_barrier<TIGHT>(L.sync, ++epoch)) return;
    // ---- column phase ----
    if (s + 1 < L.S) prefetch_rows<PL>(V + L.vstride, G);
    for (int u = g * G + blockIdx.x; u < L.b.nx / CW; u += GROUPS * G)
      loop_col<PL, CW>(L.b, L.wave, u * CW, cl, t, smem + (g * CW + cl) * SH::COL_SLOT, sky, spy);
    if (s + 1 < L.S && !loop_barrier<TIGHT>(L.sync, ++epoch)) return;
  }
}

// Plans of the persistent loop per line length: the packed plan variant with
// one warp per line (its twiddle table is that variant's).
template <int N>
struct LoopPlan;
template <> struct LoopPlan<256> { static constexpr int V = 4; };
template <> struct LoopPlan<512> { static constexpr int V = 4; };
template <> struct LoopPlan<1024> { static constexpr int V = 3; };
// Variants of the loop kernel (chosen per grid by the engine's autotuner):
// the column unit width CW and the barrier form.
constexpr int kLoopVariants = 5;
template <int V> struct LoopVariant;
template <> struct LoopVariant<0> { static constexpr int CW = 4; static constexpr bool TIGHT = false; };
template <> struct LoopVariant<1> { static constexpr int CW = 8; static constexpr bool TIGHT = false; };
template <> struct LoopVariant<2> { static constexpr int CW = 4; static constexpr bool TIGHT = true; };
template <> struct LoopVariant<3> { static constexpr int CW = 8; static constexpr bool TIGHT = true; };
template <> struct LoopVariant<4> { static constexpr int CW = 2; static constexpr bool TIGHT = true; };

}  // namespace ms
