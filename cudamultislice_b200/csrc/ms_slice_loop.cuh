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

// v *= exp(i sigma V) over a thread's E points: the polynomial-only sincos
// when every phase of the warp is within a quarter turn of 0 (bit-identical,
// the usual case for slices of a few angstroms), else the reduced one.
template <int E>
MS_D void transmit_line(float2 (&v)[E], float (&vv)[E], float sigma) {
  bool small = true;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    vv[j] = fmul_x(sigma, vv[j]);
    small = small && sincos_small_ok(vv[j]);
  }
  if (__all_sync(0xffffffffu, small)) {
#pragma unroll
    for (int j = 0; j < E; j += 2) {
      float s0, c0, s1, c1;
      sincos_small2(vv[j], vv[j + 1], &s0, &c0, &s1, &c1);
      v[j] = cmul(v[j], make_float2(c0, s0));
      v[j + 1] = cmul(v[j + 1], make_float2(c1, s1));
    }
  } else {
#pragma unroll
    for (int j = 0; j < E; j += 2) {
      float s0, c0, s1, c1;
      sincos_red2(vv[j], vv[j + 1], &s0, &c0, &s1, &c1);
      v[j] = cmul(v[j], make_float2(c0, s0));
      v[j + 1] = cmul(v[j + 1], make_float2(c1, s1));
    }
  }
}

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
// clock and the error word every 32 polls.  FENCED: full fences around the
// arrival and after the wait (as cooperative groups' grid sync); without
// them the release reduction and the acquire load carry the ordering (both
// are cumulative over what the CTA's bar.sync has ordered before them).
template <bool TIGHT, bool FENCED = true>
MS_D bool loop_barrier(const LoopSync& s, unsigned int epoch) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    if constexpr (FENCED || !TIGHT) __threadfence();
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
    if constexpr (FENCED || !TIGHT) __threadfence();
  }
  return __syncthreads_and(ok) != 0;
}

template <class PL, int CW, int NT_>
struct LoopShape {
  static constexpr int N = PL::N, E = PL::E, P = PL::P;
  static_assert(P == 32 || P == 64, "the persistent loop runs lines of one or two warps");
  static constexpr int NT = NT_;                 // threads per CTA
  static constexpr int LINES = NT / P;           // rows per CTA per round
  static constexpr int GS = CW * P;              // threads of one column unit
  static constexpr int GROUPS = NT / GS;         // column units per CTA per round
  static_assert(GROUPS >= 1 && NT % GS == 0, "column units must tile the CTA");
  static constexpr int ROW_SLOT = PL::SLOT;
  static constexpr int COL_SLOT = ((N + N / PL::R1 + 15) / 16) * 16 + 16 / CW;
  static constexpr int EXCH = (LINES * ROW_SLOT > GROUPS * CW * COL_SLOT) ? LINES * ROW_SLOT : GROUPS * CW * COL_SLOT;
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
  transmit_line<E>(v, vv, a.sigma);
  fft::line_fft<PL>(v, sm, t, a.tw);
#pragma unroll
  for (int j = 0; j < E; ++j) out[row0 + t + P * j] = v[j];
}

// Column phase of one unit of CW columns starting at c0: FFT_col -> x P/N
// (band-limited) -> IFFT_col, in place.
template <class PL, int CW>
MS_D void loop_col(const PassBArgs& b, float2* wave, int c0, int cl, int t, float2* sm,
                   const float* __restrict__ sky, const float2* __restrict__ spy) {
  constexpr int E = PL::E, P = PL::P, GS = CW * P;
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

// Bulk L2 prefetch of the potential rows this CTA's lines read in the next
// row phase (issued during the column phase; one 4-byte-per-point row each).
template <class PL>
MS_D void prefetch_rows(const float* V, int G) {
  constexpr int NX = PL::N, P = PL::P;
  const int li = threadIdx.x / P, lt = threadIdx.x % P;
  const int line = li * G + blockIdx.x;
  if (lt == 0 && line < NX) {
    const float* p = V + (long long)line * NX;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"((unsigned)(NX * sizeof(float)))
                 : "memory");
  }
}

template <class PL, int CW, bool TIGHT, int NT, bool FENCED = true>
__global__ void __launch_bounds__(NT, 1) k_slice_loop(LoopArgs L) {
  using SH = LoopShape<PL, CW, NT>;
  constexpr int N = PL::N, P = PL::P, GS = SH::GS, GROUPS = SH::GROUPS;
  extern __shared__ float2 smem[];
  float* sky = reinterpret_cast<float*>(smem + SH::EXCH);
  float2* spy = smem + SH::EXCH + (N + 1) / 2;
  for (int i = threadIdx.x; i < N; i += SH::NT) {
    sky[i] = L.b.ky[i];
    spy[i] = L.b.py[i];
  }
  __syncthreads();
  const int G = gridDim.x;
  const int li = threadIdx.x / P, lt = threadIdx.x % P;  // row line of the CTA, index within it
  // this thread's column-unit coordinates
  const int g = threadIdx.x / GS, gr = threadIdx.x % GS;
  const int cl = gr % CW, t = gr / CW;
  unsigned int epoch = 0;
  for (int s = 0; s < L.S; ++s) {
    const float* V = L.Vstack + (long long)s * L.vstride;
    // ---- row phase ----
    for (int line = li * G + blockIdx.x; line < N; line += SH::LINES * G) {
      float2* sm = smem + li * SH::ROW_SLOT;
      if (s == 0)
        loop_row<PL, false>(L.a, L.psi0, L.wave, V, line, lt, sm);
      else
        loop_row<PL, true>(L.a, L.wave, L.wave, V, line, lt, sm);
    }
    if (!loop_barrier<TIGHT, FENCED>(L.sync, ++epoch)) return;
    // ---- column phase ----
    if (s + 1 < L.S) prefetch_rows<PL>(V + L.vstride, G);
    for (int u = g * G + blockIdx.x; u < L.b.nx / CW; u += GROUPS * G)
      loop_col<PL, CW>(L.b, L.wave, u * CW, cl, t, smem + (g * CW + cl) * SH::COL_SLOT, sky, spy);
    if (s + 1 < L.S && !loop_barrier<TIGHT>(L.sync, ++epoch)) return;
  }
}

// ---------------------------------------------------------------------------
// Batched loop: the instances of up to two groups (grid sizes N0 >= N1) share
// every phase.  A row phase covers every line of every instance, a column
// phase every column unit of every instance, with grid barriers between them,
// so the barrier cost is shared by B instance-steps and each warp handles
// several lines per phase.  Lines and units are numbered group 0 first, then
// instance by instance, and dealt round-robin over the CTAs' line slots.
// ---------------------------------------------------------------------------

// Row phase of one line of a batched instance: [IFFT_row] -> x t -> FFT_row
// in place, t = exp(i sigma V) from V on the fly or a stored transmission.
template <class PL, bool TC>
MS_D void batch_row(const LoopGroup& G, int s, int inst, int line, int t, float2* sm, bool first) {
  constexpr int NX = PL::N, E = PL::E, P = PL::P;
  const long long nn = (long long)NX * NX;
  float2* w = G.wave + inst * nn + (long long)line * NX;
  const long long q0 = inst * G.inst_stride + (long long)s * G.slice_stride + (long long)line * NX;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = w[t + P * j];
  if constexpr (!TC) {
    float vv[E];
#pragma unroll
    for (int j = 0; j < E; ++j) vv[j] = G.Vstack[q0 + t + P * j];
    if (!first) {
      fft::conj_all(v);
      fft::line_fft<PL>(v, sm, t, G.a.tw);
      fft::conj_all(v);
    }
    transmit_line<E>(v, vv, G.a.sigma);
  } else {
    float2 tc[E];
#pragma unroll
    for (int j = 0; j < E; ++j) tc[j] = G.tstack[q0 + t + P * j];
    if (!first) {
      fft::conj_all(v);
      fft::line_fft<PL>(v, sm, t, G.a.tw);
      fft::conj_all(v);
    }
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = cmul(v[j], tc[j]);
  }
  fft::line_fft<PL>(v, sm, t, G.a.tw);
#pragma unroll
  for (int j = 0; j < E; ++j) w[t + P * j] = v[j];
}

// Column phase of one unit of a batched instance: FFT_col, then either the
// propagator and IFFT_col (in place), or, on the last slice of a group with a
// detector, the annular sum of |FFT_col|^2 inside the band limit (the last
// propagation only masks: |FFT2(psi_exit)|^2 = |P|^2 |FFT_col|^2), FP64 per
// warp, added to sig[inst] with the scale 1/N.
template <class PL, int CW>
MS_D void batch_col(const LoopGroup& G, int inst, int c0, int cl, int t, float2* sm, const float* __restrict__ sky,
                    const float2* __restrict__ spy, bool detect) {
  constexpr int NY = PL::N, E = PL::E, P = PL::P, GS = CW * P;
  const int nx = NY;
  const long long nn = (long long)NY * NY;
  float2* base = G.wave + inst * nn;
  const int col = c0 + cl;
  const float2* src = base + (long long)t * nx + col;
  const int step = P * nx;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = src[j * step];
  if (detect) {
    fft::line_fft<fft::PaddedPlan<PL>, GS>(v, sm, t, G.b.tw);
    const float kx = G.b.kx[col];
    const float kx2 = fmul_x(kx, kx);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const float ky = sky[t + P * j];
      const float k2 = fadd_x(kx2, fmul_x(ky, ky));
      const bool keep = k2 < G.b.k2_lt && k2 >= G.b.kin2 && k2 < G.b.kout2;  // sqrt(k^2) < kmax
      if (keep) acc += v[j].x * v[j].x + v[j].y * v[j].y;
    }
    double d = (double)acc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d != 0.0) atomicAdd(G.sig + inst, d * (double)G.b.scale);
    return;
  }
#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    fft::line_fft<fft::PaddedPlan<PL>, GS>(v, sm, t, G.b.tw);
    if (it == 0) {
      col_mid<PL, B_PROPAGATE>(v, G.b, sky, spy, col, t, 0);
    }
    fft::conj_all(v);
  }
  int ostep;
  asm volatile("mov.b32 %0, %1;" : "=r"(ostep) : "r"(step));
  float2* dst = base + (long long)t * nx + col;
#pragma unroll
  for (int j = 0; j < E; ++j) dst[j * ostep] = v[j];
}

template <class PL0, class PL1, int CW>
struct BatchShape {
  using A = LoopShape<PL0, CW, 256>;
  using B = LoopShape<PL1, CW, 256>;
  static constexpr int NT = 256;
  static constexpr int LINES_ROWS = NT / 32;  // row lines in flight per CTA
  static constexpr int EXCH = A::EXCH > B::EXCH ? A::EXCH : B::EXCH;
  static constexpr int N0 = PL0::N, N1 = PL1::N;
  // exchange slots, then ky0 | ky1 (floats, padded to float2) and py0 | py1
  static constexpr int KY = (N0 + N1 + 1) / 2;
  static constexpr size_t SMEM = ((size_t)EXCH + KY + N0 + N1) * sizeof(float2);
};

// TC: the groups multiply by stored transmissions (tstack) rather than
// forming exp(i sigma V) from Vstack.
template <class PL0, class PL1, int CW, bool TC>
__global__ void __launch_bounds__(256, 1) k_batch_loop(BatchLoopArgs L) {
  using SH = BatchShape<PL0, PL1, CW>;
  using SA = typename SH::A;
  using SB = typename SH::B;
  static_assert(PL0::P == 32 && PL1::P == 32, "batched loop runs one warp per line");
  constexpr int N0 = PL0::N, N1 = PL1::N, GS = CW * 32, GROUPS = SH::NT / GS;
  extern __shared__ float2 smem[];
  float* sky0 = reinterpret_cast<float*>(smem + SH::EXCH);
  float* sky1 = sky0 + N0;
  float2* spy0 = smem + SH::EXCH + SH::KY;
  float2* spy1 = spy0 + N0;
  const LoopGroup& G0 = L.g[0];
  const LoopGroup& G1 = L.g[1];
  const bool has1 = G1.n > 0 && G1.B > 0;
  for (int i = threadIdx.x; i < N0; i += SH::NT) {
    sky0[i] = G0.b.ky[i];
    spy0[i] = G0.b.py[i];
  }
  if (has1)
    for (int i = threadIdx.x; i < N1; i += SH::NT) {
      sky1[i] = G1.b.ky[i];
      spy1[i] = G1.b.py[i];
    }
  __syncthreads();
  const int G = gridDim.x;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = threadIdx.x / GS, gr = threadIdx.x % GS;
  const int cl = gr % CW, t = gr / CW;
  // one slot size for both grids: the CTA's column groups may hold units of
  // different grids at the same time (N0 >= N1, so group 0's slots are the larger)
  constexpr int CSLOT = SA::COL_SLOT > SB::COL_SLOT ? SA::COL_SLOT : SB::COL_SLOT;
  constexpr int RSLOT = SA::ROW_SLOT > SB::ROW_SLOT ? SA::ROW_SLOT : SB::ROW_SLOT;
  static_assert(SH::LINES_ROWS * RSLOT <= SH::EXCH && GROUPS * CW * CSLOT <= SH::EXCH, "exchange slots overflow");
  const long long rows0 = (long long)G0.B * N0, rows1 = has1 ? (long long)G1.B * N1 : 0;
  const long long units0 = (long long)G0.B * (N0 / CW), units1 = has1 ? (long long)G1.B * (N1 / CW) : 0;
  unsigned int epoch = 0;
  for (int s = 0; s < L.S; ++s) {
    const bool first = s == 0, last = s + 1 == L.S;
    // ---- row phase: every line of every instance ----
    for (long long r = (long long)warp * G + blockIdx.x; r < rows0 + rows1; r += (long long)SA::LINES * G) {
      float2* sm = smem + warp * RSLOT;
      if (r < rows0)
        batch_row<PL0, TC>(G0, s, (int)(r / N0), (int)(r % N0), lane, sm, first);
      else
        batch_row<PL1, TC>(G1, s, (int)((r - rows0) / N1), (int)((r - rows0) % N1), lane, sm, first);
    }
    if (!loop_barrier<true>(L.sync, ++epoch)) return;
    // ---- column phase: every column unit of every instance ----
    for (long long u = (long long)g * G + blockIdx.x; u < units0 + units1; u += (long long)GROUPS * G) {
      float2* sm = smem + (g * CW + cl) * CSLOT;
      if (u < units0) {
        batch_col<PL0, CW>(G0, (int)(u / (N0 / CW)), (int)(u % (N0 / CW)) * CW, cl, t, sm, sky0, spy0,
                           last && G0.sig != nullptr);
      } else {
        const long long v = u - units0;
        batch_col<PL1, CW>(G1, (int)(v / (N1 / CW)), (int)(v % (N1 / CW)) * CW, cl, t, sm, sky1, spy1,
                           last && G1.sig != nullptr);
      }
    }
    if (!last && !loop_barrier<true>(L.sync, ++epoch)) return;
  }
}

// Variants of the loop kernel (chosen per grid by the engine's autotuner):
// narrow (lines of one warp, 256-thread CTAs) or wide (lines of two warps,
// 512-thread CTAs: twice the warps per SM, one more exchange pass), the
// column unit width CW and the barrier form.
constexpr int kLoopVariants = 10;
template <int V> struct LoopVariant;
template <> struct LoopVariant<0> { static constexpr int CW = 4, NT = 256; static constexpr bool TIGHT = false, FENCED = true; };
template <> struct LoopVariant<1> { static constexpr int CW = 8, NT = 256; static constexpr bool TIGHT = false, FENCED = true; };
template <> struct LoopVariant<2> { static constexpr int CW = 4, NT = 256; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<3> { static constexpr int CW = 8, NT = 256; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<4> { static constexpr int CW = 2, NT = 256; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<5> { static constexpr int CW = 4, NT = 512; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<6> { static constexpr int CW = 2, NT = 512; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<7> { static constexpr int CW = 8, NT = 512; static constexpr bool TIGHT = true, FENCED = true; };
template <> struct LoopVariant<8> { static constexpr int CW = 8, NT = 256; static constexpr bool TIGHT = true, FENCED = false; };
template <> struct LoopVariant<9> { static constexpr int CW = 4, NT = 256; static constexpr bool TIGHT = true, FENCED = false; };

// FFT plan variant (PlanSel) of the loop per line length: the packed plan with
// one warp per line (narrow loop variants) or two warps per line (wide).
template <int N, bool WIDE>
struct LoopPlan;
template <> struct LoopPlan<256, false> { static constexpr int V = 4; };
template <> struct LoopPlan<512, false> { static constexpr int V = 4; };
template <> struct LoopPlan<1024, false> { static constexpr int V = 3; };
template <> struct LoopPlan<256, true> { static constexpr int V = 5; };
template <> struct LoopPlan<512, true> { static constexpr int V = 5; };
template <> struct LoopPlan<1024, true> { static constexpr int V = 4; };

}  // namespace ms
