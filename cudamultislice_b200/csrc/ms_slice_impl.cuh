// ms_slice_impl.cuh -- templates of the fused slice passes, instantiated per
// line length in ms_slice_n*.cu (see ms_slice.cuh for the scheme).
#pragma once
#include <cuda.h>
#include <stdint.h>
#include <cmath>
#include <mutex>

#include "ms_ctf.cuh"
#include "ms_fft.cuh"
#include "ms_slice.cuh"

namespace ms {

// FFT plan variants per line length (chosen at run time by the autotuner):
// variant 0 keeps the most points per thread (fewest exchanges), higher
// variants spread a line over more threads (more warps in flight); variants
// 3..5 are 0..2 with the butterflies on the packed FP32x2 pipe.
template <int N, int V>
struct PlanSel;
template <> struct PlanSel<64, 0>   { using T = fft::Plan<64, 8, 8, 8>; };
template <> struct PlanSel<64, 1>   { using T = fft::Plan<64, 4, 4, 4, 4>; };
template <> struct PlanSel<64, 2>   { using T = fft::Plan<64, 4, 4, 4, 4>; };
template <> struct PlanSel<128, 0>  { using T = fft::Plan<128, 16, 16, 8>; };
template <> struct PlanSel<128, 1>  { using T = fft::Plan<128, 8, 8, 4, 4>; };
template <> struct PlanSel<128, 2>  { using T = fft::Plan<128, 4, 4, 4, 4, 2>; };
template <> struct PlanSel<256, 0>  { using T = fft::Plan<256, 16, 16, 16>; };
template <> struct PlanSel<256, 1>  { using T = fft::Plan<256, 8, 8, 8, 4>; };
template <> struct PlanSel<256, 2>  { using T = fft::Plan<256, 4, 4, 4, 4, 4>; };
template <> struct PlanSel<512, 0>  { using T = fft::Plan<512, 32, 32, 16>; };
template <> struct PlanSel<512, 1>  { using T = fft::Plan<512, 16, 16, 8, 4>; };
template <> struct PlanSel<512, 2>  { using T = fft::Plan<512, 8, 8, 8, 8>; };
template <> struct PlanSel<1024, 0> { using T = fft::Plan<1024, 32, 32, 32>; };
template <> struct PlanSel<1024, 1> { using T = fft::Plan<1024, 16, 16, 16, 4>; };
template <> struct PlanSel<1024, 2> { using T = fft::Plan<1024, 8, 8, 8, 8, 2>; };
template <> struct PlanSel<2048, 0> { using T = fft::Plan<2048, 32, 32, 8, 8>; };
template <> struct PlanSel<2048, 1> { using T = fft::Plan<2048, 16, 16, 16, 8>; };
template <> struct PlanSel<2048, 2> { using T = fft::Plan<2048, 8, 8, 8, 8, 4>; };
template <> struct PlanSel<4096, 0> { using T = fft::Plan<4096, 32, 32, 32, 4>; };
template <> struct PlanSel<4096, 1> { using T = fft::Plan<4096, 16, 16, 16, 16>; };
template <> struct PlanSel<4096, 2> { using T = fft::Plan<4096, 16, 8, 8, 8, 8>; };
template <> struct PlanSel<64, 3> { using T = fft::Plan<64, 8, 8, 8, 1, 1, true>; };
template <> struct PlanSel<64, 4> { using T = fft::Plan<64, 4, 4, 4, 4, 1, true>; };
template <> struct PlanSel<64, 5> { using T = fft::Plan<64, 4, 4, 4, 4, 1, true>; };
template <> struct PlanSel<128, 3> { using T = fft::Plan<128, 16, 16, 8, 1, 1, true>; };
template <> struct PlanSel<128, 4> { using T = fft::Plan<128, 8, 8, 4, 4, 1, true>; };
template <> struct PlanSel<128, 5> { using T = fft::Plan<128, 4, 4, 4, 4, 2, true>; };
template <> struct PlanSel<256, 3> { using T = fft::Plan<256, 16, 16, 16, 1, 1, true>; };
template <> struct PlanSel<256, 4> { using T = fft::Plan<256, 8, 8, 8, 4, 1, true>; };
template <> struct PlanSel<256, 5> { using T = fft::Plan<256, 4, 4, 4, 4, 4, true>; };
template <> struct PlanSel<512, 3> { using T = fft::Plan<512, 32, 32, 16, 1, 1, true>; };
template <> struct PlanSel<512, 4> { using T = fft::Plan<512, 16, 16, 8, 4, 1, true>; };
template <> struct PlanSel<512, 5> { using T = fft::Plan<512, 8, 8, 8, 8, 1, true>; };
template <> struct PlanSel<1024, 3> { using T = fft::Plan<1024, 32, 32, 32, 1, 1, true>; };
template <> struct PlanSel<1024, 4> { using T = fft::Plan<1024, 16, 16, 16, 4, 1, true>; };
template <> struct PlanSel<1024, 5> { using T = fft::Plan<1024, 8, 8, 8, 8, 2, true>; };
template <> struct PlanSel<2048, 3> { using T = fft::Plan<2048, 32, 32, 8, 8, 1, true>; };
template <> struct PlanSel<2048, 4> { using T = fft::Plan<2048, 16, 16, 16, 8, 1, true>; };
template <> struct PlanSel<2048, 5> { using T = fft::Plan<2048, 8, 8, 8, 8, 4, true>; };
template <> struct PlanSel<4096, 3> { using T = fft::Plan<4096, 32, 32, 32, 4, 1, true>; };
template <> struct PlanSel<4096, 4> { using T = fft::Plan<4096, 16, 16, 16, 16, 1, true>; };
template <> struct PlanSel<4096, 5> { using T = fft::Plan<4096, 16, 8, 8, 8, 8, true>; };

constexpr int kPlanVariants = 6;

// Threads per CTA: rows, 256 (whole lines), 64 or 128 for the unpacked
// 32-point plans of lines of 32 or 64 threads (two lines per CTA: more CTAs,
// which a single instance, one wave, needs; the packed twin keeps whole
// 256-thread CTAs);
// columns, 4 columns per CTA for lines of 64 or more threads (256 threads for
// shorter lines), so that a warp's accesses cover whole 32-byte sectors,
// halved for the narrow plans.
template <class PL>
__host__ __device__ constexpr int rows_per_cta() {
  return PL::P >= 256 ? 1 : (!PL::PK && PL::E >= 32 && PL::P <= 64) ? 2 : 256 / PL::P;
}
// The packed 32-point column plans take half the columns per CTA: twice the
// CTAs, which a single instance (one wave) needs, and registers enough for
// two CTAs without spilling; their unpacked twins keep the wide tiles that
// win in batches (the autotuner chooses per batch).
template <class PL>
__host__ __device__ constexpr bool narrow_cols() { return PL::PK && PL::E >= 32; }
template <class PL>
__host__ __device__ constexpr int cols_per_cta() {
  return (PL::P < 64 ? 256 / PL::P : 4) / (narrow_cols<PL>() ? 2 : 1);
}
// Column CTAs resident per SM that the register budget is sized for: two,
// unless that would leave fewer than 64 registers per thread for 16 or more
// points per thread.  (Left free, the compiler hoists the pointwise step's
// table loads and the next pass's twiddles far enough to hold one CTA per SM.)
template <class PL>
__host__ __device__ constexpr int col_min_ctas() {
  return cols_per_cta<PL>() * PL::P <= (PL::E <= 8 ? 512 : 256) ? 2 : 1;
}
// The column pass interleaves CW adjacent columns per warp row: thread
// (column c, index t) is thread t * CW + c of its group, so every 8-byte load
// and store of a warp covers CW columns of 32/CW rows (CW x 8 contiguous bytes
// per row) straight from and to registers, with no staging tile.  The CW * P
// threads of a group share their columns' exchange barriers.
template <class PL>
__host__ __device__ constexpr int col_interleave() { return cols_per_cta<PL>() < 8 ? cols_per_cta<PL>() : 8; }
template <class PL>
__host__ __device__ constexpr int col_group() { return col_interleave<PL>() * PL::P; }
// Column slots (padded map, fft::PaddedPlan) 16/CW points (mod 16) apart: a
// 16-lane phase covers 16/CW consecutive points of CW columns, which then fall
// in distinct bank pairs.
template <class PL>
__host__ __device__ constexpr int col_slot() {
  return ((PL::N + PL::N / PL::R1 + 15) / 16) * 16 + 16 / col_interleave<PL>();
}

// Programmatic dependent launch: the passes are launched with programmatic
// stream serialisation, so a pass may start while the previous kernel of the
// stream drains.  Every pass signals its dependents at entry and waits for its
// predecessor's completion (and memory) before its first global access.
MS_D void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
MS_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Per-point operands of the row pass's pointwise work, loaded with the line
// so that their latency overlaps the inverse transform: V (transmission,
// stencil, adjoint), T (residual), and the second wave (stencil, adjoint)
// where registers allow.
template <class PL, int FLAGS>
struct RowOperands {
  static constexpr int E = PL::E, P = PL::P, NX = PL::N;
  static constexpr bool HAS_V = (FLAGS & (A_MULT_T | A_FD | A_ADJ)) != 0;
  static constexpr bool HAS_T = (FLAGS & A_RESID) != 0;
  static constexpr bool HAS_W = (FLAGS & (A_FD | A_ADJ)) != 0 && E <= 16;
  static constexpr bool HAS_TC = (FLAGS & A_MULT_TC) != 0;
  float V[HAS_V ? E : 1];
  float2 TC[HAS_TC ? E : 1];
  float T[HAS_T ? E : 1];
  float2 W[HAS_W ? E : 1];
  MS_D void load(const PassAArgs& a, long long inst, int line, long long row0, int t) {
    const long long r0 = inst * a.batch_stride_V + (long long)line * NX;
    if constexpr (HAS_V) {
#pragma unroll
      for (int j = 0; j < E; ++j) V[j] = a.V[r0 + t + P * j];
    }
    if constexpr (HAS_T) {
#pragma unroll
      for (int j = 0; j < E; ++j) T[j] = a.T[r0 + t + P * j];
    }
    if constexpr (HAS_TC) {
#pragma unroll
      for (int j = 0; j < E; ++j) TC[j] = a.tr[r0 + t + P * j];
    }
    if constexpr (HAS_W) {
#pragma unroll
      for (int j = 0; j < E; ++j) W[j] = a.in2[row0 + t + P * j];
    }
  }
  MS_D float2 w(const PassAArgs& a, long long row0, int j, int t) const {
    if constexpr (HAS_W) return W[j];
    else return a.in2[row0 + t + P * j];
  }
};

// Pointwise work of the row pass between its inverse and forward transforms.
template <class PL, int FLAGS>
MS_D void row_mid(float2 (&v)[PL::E], const PassAArgs& a, const RowOperands<PL, FLAGS>& op, long long inst,
                  int line, long long row0, int t) {
  constexpr int NX = PL::N, E = PL::E, P = PL::P;
  if constexpr ((FLAGS & A_FD) != 0) {
    float2* pc = a.out2 + row0;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int x = t + P * j;
      pc[x] = v[j];
      const float f = 2.0f - a.fd_kv * op.V[j];
      v[j] = csub(cmul(a.fd_rc, cscale(v[j], f)), cmul(a.fd_ratio, op.w(a, row0, j, t)));
    }
  }
  if constexpr ((FLAGS & A_SAVE) != 0) {
    float2* o = a.out2 + row0;
#pragma unroll
    for (int j = 0; j < E; ++j) o[t + P * j] = v[j];
  }
  if constexpr ((FLAGS & A_MULT_T) != 0) {
    // two points per packed sincos (bit-identical to sincos_red per point);
    // the polynomial-only form when every phase of the warp is within a
    // quarter turn of 0 (bit-identical too)
    bool small = true;
#pragma unroll
    for (int j = 0; j < E; ++j) small = small && sincos_small_ok(fmul_x(a.sigma, op.V[j]));
    if (__all_sync(0xffffffffu, small)) {
#pragma unroll
      for (int j = 0; j < E; j += 2) {
        float s0, c0, s1, c1;
        sincos_small2(fmul_x(a.sigma, op.V[j]), fmul_x(a.sigma, op.V[j + 1]), &s0, &c0, &s1, &c1);
        v[j] = cmul(v[j], make_float2(c0, s0));
        v[j + 1] = cmul(v[j + 1], make_float2(c1, s1));
      }
    } else {
#pragma unroll
      for (int j = 0; j < E; j += 2) {
        float s0, c0, s1, c1;
        sincos_red2(fmul_x(a.sigma, op.V[j]), fmul_x(a.sigma, op.V[j + 1]), &s0, &c0, &s1, &c1);
        v[j] = cmul(v[j], make_float2(c0, s0));
        v[j + 1] = cmul(v[j + 1], make_float2(c1, s1));
      }
    }
  }
  if constexpr ((FLAGS & A_MULT_TC) != 0) {
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = cmul(v[j], op.TC[j]);
  }
  if constexpr ((FLAGS & A_RESID) != 0) {
    const long long r0 = inst * a.batch_stride_V + (long long)line * NX;
    float* img = a.out_f ? a.out_f + r0 : nullptr;
    double part = 0.0;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int x = t + P * j;
      const float I = v[j].x * v[j].x + v[j].y * v[j].y;
      if (img) img[x] = I;
      const float r = I - op.T[j];
      part += (double)r * (double)r;
      v[j] = cscale(v[j], 2.0f * r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(a.loss, part);
  }
  if constexpr ((FLAGS & A_ADJ) != 0) {
    const long long r0 = inst * a.batch_stride_V + (long long)line * NX;
    float* dV = a.out_f + r0;
    const float m2s = -2.0f * a.sigma;
#pragma unroll
    for (int j = 0; j < E; j += 2) {
      float s0, c0, s1, c1;
      sincos_red2(fmul_x(a.sigma, op.V[j]), fmul_x(a.sigma, op.V[j + 1]), &s0, &c0, &s1, &c1);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int jj = j + h, x = t + P * jj;
        const float2 tt = h ? make_float2(c1, s1) : make_float2(c0, s0);
        const float2 q = cmul(tt, op.w(a, row0, jj, t));
        dV[x] = m2s * (v[jj].x * q.y - v[jj].y * q.x);
        v[jj] = cmul(cconj(tt), v[jj]);
      }
    }
  }
}

template <class PL, int FLAGS>
MS_D void pass_a_body(PassAArgs a) {
  constexpr int NX = PL::N, E = PL::E, P = PL::P, LS = PL::SLOT;
  constexpr bool INVF = (FLAGS & A_INV) != 0, FWDF = (FLAGS & A_FWD) != 0;
  extern __shared__ float2 smem[];
  const int g = threadIdx.x / P, t = threadIdx.x % P;
  const int line = blockIdx.x * rows_per_cta<PL>() + g;
  float2* sm = smem + g * LS;
  const long long inst = blockIdx.y;
  const long long row0 = inst * a.batch_stride_wave + (long long)line * NX;

  pdl_launch_dependents();
  pdl_wait();
  float2 v[E];
  const float2* in = a.in + row0;
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = in[t + P * j];
  RowOperands<PL, FLAGS> op;
  op.load(a, inst, line, row0, t);

  if constexpr (!INVF) row_mid<PL, FLAGS>(v, a, op, inst, line, row0, t);
  if constexpr (INVF || FWDF) {
    // one copy of the transform code: iteration 0 is the inverse
    // conj(FFT(conj(.))) followed by the pointwise work, iteration 1 the forward
#pragma unroll 1
    for (int it = INVF ? 0 : 1; it < (FWDF ? 2 : 1); ++it) {
      if (it == 0) fft::conj_all(v);
      fft::line_fft<PL>(v, sm, t, a.tw);
      if (it == 0) {
        fft::conj_all(v);
        if constexpr (INVF) row_mid<PL, FLAGS>(v, a, op, inst, line, row0, t);
      }
    }
  }

  if constexpr ((FLAGS & A_INTENSITY) != 0) {
    float* o = a.out_f + row0;
#pragma unroll
    for (int j = 0; j < E; ++j) o[t + P * j] = (v[j].x * v[j].x + v[j].y * v[j].y) * a.scale;
  } else if constexpr ((FLAGS & A_REAL) != 0) {
    float* o = a.out_f + row0;
#pragma unroll
    for (int j = 0; j < E; ++j) o[t + P * j] = v[j].x * a.scale;
  } else if constexpr ((FLAGS & A_RESID) != 0 && !FWDF) {
    // residual only: the loss (and the image) are the results
  } else {
    float2* o = a.out + row0;
    if (a.scale != 1.0f) {
#pragma unroll
      for (int j = 0; j < E; ++j) v[j] = cscale(v[j], a.scale);
    }
#pragma unroll
    for (int j = 0; j < E; ++j) o[t + P * j] = v[j];
  }
}

// Pointwise work of the column pass on the column spectrum (between the
// forward and the inverse transform, or before the epilogue).
// Column modes whose pointwise work reads the row frequencies ky, and the
// propagator's row factors py: staged in shared memory per CTA.
template <int MODE>
__host__ __device__ constexpr bool col_uses_ky() {
  return MODE == B_PROPAGATE || MODE == B_PROPAGATE_ADJ || MODE == B_CTF || MODE == B_CTF_ADJ ||
         MODE == B_BANDLIMIT || MODE == B_FD || MODE == B_DETECT;
}
template <int MODE>
__host__ __device__ constexpr bool col_uses_py() { return MODE == B_PROPAGATE || MODE == B_PROPAGATE_ADJ; }
// Columns of at most 1024 points stage ky and py in shared memory; longer
// columns read them through L1, which keeps their CTAs' shared memory to the
// exchange slots.
template <class PL, int MODE>
__host__ __device__ constexpr bool col_stages_ky() { return col_uses_ky<MODE>() && PL::N <= 1024; }
template <class PL, int MODE>
__host__ __device__ constexpr bool col_stages_py() { return col_uses_py<MODE>() && PL::N <= 1024; }

template <class PL, int MODE>
MS_D void col_mid(float2 (&v)[PL::E], const PassBArgs& a, const float* __restrict__ sky,
                  const float2* __restrict__ spy, int col, int t, long long base) {
  constexpr int NY = PL::N, E = PL::E, P = PL::P;
  const float scale = a.scale;
  if constexpr (MODE == B_PROPAGATE) {
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    const float2 pxv = a.px[col];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = sky[n];
      // CreatePropsKernel (U.cu:419): keep sqrtf(kx^2+ky^2) < kmax
      const bool keep = fadd_x(kx2, fmul_x(ky, ky)) < a.k2_lt;
      // the two unit factors one after the other (no rounded product table)
      v[j] = keep ? cmul(cmul(v[j], pxv), spy[n]) : make_float2(0.f, 0.f);
    }
  } else if constexpr (MODE == B_PROPAGATE_ADJ) {
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    const float2 pxv = a.px[col];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = sky[n];
      const bool keep = fadd_x(kx2, fmul_x(ky, ky)) < a.k2_lt;
      v[j] = keep ? cscale(cmul(cmul(v[j], cconj(pxv)), cconj(spy[n])), scale) : make_float2(0.f, 0.f);
    }
  } else if constexpr (MODE == B_CTF || MODE == B_CTF_ADJ) {
    const float kx = a.kx[col];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float2 w = ctf_weight(a.ctf.wavel, a.ctf.Cs, a.ctf.df, a.ctf.A2, a.ctf.phi2, a.ctf.A3, a.ctf.phi3,
                                  a.ctf.beta, a.ctf.delta, a.ctf.objap2, kx, sky[n], scale);
      v[j] = cmul(v[j], MODE == B_CTF ? w : cconj(w));
    }
  } else if constexpr (MODE == B_BANDLIMIT) {
    // BandLimitKernel (U.cu:1025-1042): keep k <= kmax
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const float ky = sky[t + P * j];
      const bool keep = fadd_x(kx2, fmul_x(ky, ky)) < a.k2_le;  // sqrt(k^2) <= kmax
      v[j] = keep ? cscale(v[j], scale) : make_float2(0.f, 0.f);
    }
  } else if constexpr (MODE == B_FD) {
    // Psi_{n+1} = BL (FFT2(q) + c k^2 Psi_n)
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    float2* sp = a.spec + base;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = sky[n];
      const float ky2 = fmul_x(ky, ky);
      const bool keep = fadd_x(kx2, ky2) < a.k2_le;  // sqrt(k^2) <= kmax
      const long long o = (long long)col * NY + n;  // spectrum kept column-major
      const float2 s0 = sp[o];
      const float k2 = kx * kx + ky * ky;
      const float2 nv = keep ? cadd(v[j], cscale(cmul(a.fd_c, s0), k2)) : make_float2(0.f, 0.f);
      sp[o] = nv;
      v[j] = cscale(nv, scale);
    }
  }
}

template <class PL, int MODE>
__global__ void __launch_bounds__(cols_per_cta<PL>() * PL::P, col_min_ctas<PL>()) k_pass_b(PassBArgs a) {
  constexpr int NY = PL::N, E = PL::E, P = PL::P, CB = cols_per_cta<PL>(), LS = col_slot<PL>();
  constexpr int NT = CB * P, CW = col_interleave<PL>(), GS = col_group<PL>();
  constexpr bool TWO = MODE == B_PROPAGATE || MODE == B_CTF || MODE == B_BANDLIMIT || MODE == B_FD ||
                      MODE == B_PROPAGATE_ADJ || MODE == B_CTF_ADJ;
  extern __shared__ float2 smem[];
  const int nx = a.nx;
  const int c0 = blockIdx.x * CB;
  const long long base = (long long)blockIdx.y * a.batch_stride_wave;
  const float scale = a.scale;
  const int g = threadIdx.x / GS, gr = threadIdx.x % GS;
  const int cl = g * CW + gr % CW, t = gr / CW;
  const int col = c0 + cl;
  float2* sm = smem + cl * LS;

  // constant frequency tables for the pointwise work (written before any pass
  // runs, so they may be read before the predecessor completes)
  constexpr bool SKY = col_stages_ky<PL, MODE>(), SPY = col_stages_py<PL, MODE>();
  float* sky_s = reinterpret_cast<float*>(smem + CB * LS);
  float2* spy_s = smem + CB * LS + (SKY ? (NY + 1) / 2 : 0);
  pdl_launch_dependents();
  if constexpr (SKY) {
    for (int i = threadIdx.x; i < NY; i += NT) sky_s[i] = a.ky[i];
  }
  if constexpr (SPY) {
    for (int i = threadIdx.x; i < NY; i += NT) spy_s[i] = a.py[i];
  }
  const float* sky = SKY ? sky_s : a.ky;
  const float2* spy = SPY ? spy_s : a.py;
  // this thread's E points of its column, rows t + P j, all loads in flight
  pdl_wait();
  const float2* src = a.in + base + (long long)t * nx + col;
  const int step = P * nx;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = src[j * step];
  if constexpr (SKY || SPY) __syncthreads();  // tables of every group

  // iteration 0: forward (or, for B_INV_ONLY, the conjugated inverse) and the
  // pointwise work; iteration 1: the inverse as conj(FFT(conj(.)))
#pragma unroll 1
  for (int it = 0; it < (TWO ? 2 : 1); ++it) {
    if (MODE == B_INV_ONLY) fft::conj_all(v);
    fft::line_fft<fft::PaddedPlan<PL>, GS>(v, sm, t, a.tw);
    if (it == 0) {
      if constexpr (MODE == B_INV_ONLY) {
        fft::conj_all(v);
      } else if constexpr (TWO) {
        col_mid<PL, MODE>(v, a, sky, spy, col, t, base);
        fft::conj_all(v);
      }
    } else {
      fft::conj_all(v);
    }
  }

  if constexpr (MODE == B_CBED) {
    // AddTDSWaves (U.cu:2734-2766): |FFT(psi)| placed by CentreKernel's shift
    const int xs = (col < nx / 2) ? col + nx / 2 : col - nx / 2;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const int ys = (n < NY / 2) ? n + NY / 2 : n - NY / 2;
      const float m = sqrtf(v[j].x * v[j].x + v[j].y * v[j].y) * scale;
      atomicAdd(a.acc + (long long)ys * nx + xs, m);
    }
  } else if constexpr (MODE == B_DETECT) {
    // |FFT2(psi_exit)|^2 = |P|^2 |FFT_col(Y)|^2: the last propagation only
    // masks, so the detector reads the column spectrum before the inverse.
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = sky[n];
      const float k2 = fadd_x(kx2, fmul_x(ky, ky));
      const bool keep = k2 < a.k2_lt && k2 >= a.kin2 && k2 < a.kout2;  // sqrt(k^2) < kmax
      if (keep) acc += v[j].x * v[j].x + v[j].y * v[j].y;
    }
    double d = (double)acc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d != 0.0) atomicAdd(a.sig + blockIdx.y, d * (double)scale);
  } else {
    // natural order: v[j] is row t + P j of this thread's column.  The row
    // step is passed through an opaque move so that the load addresses are
    // recomputed here rather than held in registers across the transforms.
    int ostep;
    asm volatile("mov.b32 %0, %1;" : "=r"(ostep) : "r"(step));
    float2* dst = a.out + base + (long long)t * nx + col;
    if (MODE == B_CTF_ADJ && a.accumulate) {
#pragma unroll
      for (int j = 0; j < E; ++j) dst[j * ostep] = cadd(dst[j * ostep], v[j]);
    } else {
#pragma unroll
      for (int j = 0; j < E; ++j) dst[j * ostep] = v[j];
    }
  }
}

// The row pass kernels: k_pass_a leaves registers to the compiler (32-point
// plans then take more than 128, one CTA per SM), k_pass_a_cap sizes them for
// row_cap_ctas CTAs (a little spilling can cost less than the lost overlap).
// (The column pass, k_pass_b above, sizes every plan by col_min_ctas.)
// Row CTAs per SM a capped row plan is sized for (0: left to the compiler).
// Fewer registers cost latency hiding at one instance while more CTAs win in
// batches, so plan shapes keep a free and a capped twin and the autotuner
// chooses: the unpacked 32-point plan is sized for two CTAs (a bound only for
// its 256-thread CTAs, lines of 128 threads), the packed 16-point plan for
// three; their twins stay free.
template <class PL>
constexpr int row_cap_ctas() { return (PL::E >= 32 && !PL::PK) ? 2 : (PL::E == 16 && PL::PK) ? 3 : 0; }
template <class PL>
constexpr bool capped_plan() { return row_cap_ctas<PL>() > 0; }

template <class PL, int FLAGS>
__global__ void __launch_bounds__(rows_per_cta<PL>() * PL::P) k_pass_a(PassAArgs a) {
  pass_a_body<PL, FLAGS>(a);
}
template <class PL, int FLAGS>
__global__ void __launch_bounds__(rows_per_cta<PL>() * PL::P, row_cap_ctas<PL>()) k_pass_a_cap(PassAArgs a) {
  pass_a_body<PL, FLAGS>(a);
}


// Raises a kernel's dynamic shared-memory limit once per device.  `mask`
// holds one bit per device, set only after the attribute call succeeded (a
// failed call is retried on the next launch); the mutex keeps a second host
// thread from launching before the first one has raised the limit.
template <class K>
cudaError_t set_smem_once(unsigned long long& mask, K kernel, size_t smem) {
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (mask >> dev & 1ull) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) mask |= 1ull << dev;
  return e;
}

// Launch with programmatic stream serialisation (see pdl_wait).
template <class K, class Args>
cudaError_t launch_pdl(K kernel, dim3 grid, int threads, size_t smem, cudaStream_t s, const Args& args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args);
}

template <class PL, int FLAGS>
cudaError_t run_a(const PassAArgs& a, int batch, cudaStream_t s) {
  constexpr int lines = rows_per_cta<PL>();
  const size_t smem = (size_t)lines * PL::SLOT * sizeof(float2);
  if (a.ny % lines) return cudaErrorInvalidValue;
  auto kernel = [] {
    if constexpr (capped_plan<PL>()) return k_pass_a_cap<PL, FLAGS>;
    else return k_pass_a<PL, FLAGS>;
  }();
  static unsigned long long done = 0;
  if (cudaError_t e = set_smem_once(done, kernel, smem)) return e;
  return launch_pdl(kernel, dim3(a.ny / lines, batch), lines * PL::P, smem, s, a);
}

// ---------------------------------------------------------------------------
// Column pass for long columns (2048 and 4096 points) with tensor-copy
// staging.  A CTA's CB columns are CB adjacent complex values of every row: a
// warp's direct loads of them touch 32/CB rows each, and at these sizes the
// L1's request rate, not HBM, bounded the pass.  Here one thread issues
// 2-D tensor copies of [256 rows x CB columns] boxes into shared memory, the
// threads take their points from there (a warp reads 256 contiguous bytes),
// and the results leave the same way: written to shared memory in row order,
// then stored by tensor copies.  The staging buffer doubles as the FFT's
// exchange slots once every thread holds its points.
// ---------------------------------------------------------------------------
constexpr int kTmaRows = 256;  // rows per box (the tensor-copy box limit)

MS_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Waits for the phase of the mbarrier at shared address bar with the given
// parity to complete, for at most one second of %globaltimer; false if the
// wait ran out.
MS_D bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  unsigned long long t0, tn;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(tn));
    if (tn - t0 > 1000000000ull) return false;
  }
}

// Tensor copies of CB adjacent columns (all NY rows, boxes of 256 rows) from
// the wave into dst, completing on the mbarrier at bar (one thread).
template <int NY, int CB>
MS_D void tma_load_columns(const CUtensorMap* tin, float2* dst, int c0, unsigned bar) {
  constexpr unsigned kBytes = (unsigned)(NY * CB * sizeof(float2));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kBytes) : "memory");
#pragma unroll 1
  for (int k = 0; k < NY / kTmaRows; ++k) {
    const unsigned d = smem_u32(dst + (size_t)k * kTmaRows * CB);
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            d),
        "l"(tin), "r"(2 * c0), "r"(k * kTmaRows), "r"(bar)
        : "memory");
  }
}

// Tensor copies of CB adjacent columns from src back to the wave, committed as
// one bulk group (one thread).
template <int NY, int CB>
MS_D void tma_store_columns(const CUtensorMap* tout, const float2* src, int c0) {
#pragma unroll 1
  for (int k = 0; k < NY / kTmaRows; ++k) {
    const unsigned sa = smem_u32(src + (size_t)k * kTmaRows * CB);
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tout),
                 "r"(2 * c0), "r"(k * kTmaRows), "r"(sa)
                 : "memory");
  }
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Exchange slot length for CB interleaved columns (as col_slot: slots 16/CB
// points apart mod 16).
template <class PL, int CB>
__host__ __device__ constexpr int tma_col_slot() {
  return ((PL::N + PL::N / PL::R1 + 15) / 16) * 16 + 16 / CB;
}
template <class PL, int CB>
__global__ void __launch_bounds__(CB * PL::P, CB == 2 ? 2 : 1)
    k_pass_b_tma(PassBArgs a, const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout) {
  constexpr int NY = PL::N, E = PL::E, P = PL::P, LS = tma_col_slot<PL, CB>();
  constexpr int GS = CB * P;
  static_assert(NY % kTmaRows == 0 && (2 * CB * 4) % 16 == 0, "boxes of 256 rows, 16-byte rows");
  extern __shared__ __align__(1024) float2 smem_tma[];
  __shared__ __align__(8) unsigned long long mbar;
  float2* stage = smem_tma;  // [NY][CB], then the exchange slots
  const int c0 = blockIdx.x * CB;
  const int cl = threadIdx.x % CB, t = threadIdx.x / CB;
  const int col = c0 + cl;
  float2* sm = smem_tma + cl * LS;
  const unsigned bar = smem_u32(&mbar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_launch_dependents();
  pdl_wait();
  if (threadIdx.x == 0) tma_load_columns<NY, CB>(&tin, stage, c0, bar);
  // bounded wait for the tiles (one second of %globaltimer); a wait that runs
  // out sets the error word and leaves this CTA's columns as they were
  const bool ok = mbar_wait_bounded(bar, 0);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) {
      atomicExch(a.err, 1);
      mbar_wait_bounded(bar, 0);  // copies still in flight: a bounded time to land
    }
    __syncthreads();
    return;
  }
  // this thread's E points of its column, rows t + P j
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = stage[(size_t)(t + P * j) * CB + cl];
  __syncthreads();  // (the staging buffer becomes the exchange slots)

#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    fft::line_fft<fft::PaddedPlan<PL>, GS>(v, sm, t, a.tw);
    if (it == 0) col_mid<PL, B_PROPAGATE>(v, a, a.ky, a.py, col, t, 0);
    fft::conj_all(v);
  }
  __syncthreads();  // (every exchange done: the buffer is the staging area again)
#pragma unroll
  for (int j = 0; j < E; ++j) stage[(size_t)(t + P * j) * CB + cl] = v[j];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0) {
    tma_store_columns<NY, CB>(&tout, stage, c0);
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // (the writes, not only the reads)
  }
}

// 2-D tensor map of a wave [ny][nx] complex (as 2 nx floats per row) for
// boxes of [256 rows x cb columns]; false if the driver entry point is missing
// or the encoding fails.
bool wave_tensor_map(CUtensorMap* m, const float2* base, int nx, int ny, int cb);

template <class PL, int MODE>
cudaError_t run_b(const PassBArgs& a, int batch, cudaStream_t s) {
  constexpr int CB = cols_per_cta<PL>();
  constexpr int TCB = 2;  // columns per CTA of the staged pass (two CTAs per SM)
  if constexpr (MODE == B_PROPAGATE && PL::N >= 2048 && TCB * PL::P <= 1024) {
    if (a.err && batch == 1 && a.nx % TCB == 0 && a.ny == PL::N &&
        ((uintptr_t)a.in % 16) == 0 && ((uintptr_t)a.out % 16) == 0 && ((size_t)a.nx * sizeof(float2)) % 16 == 0) {
      CUtensorMap tin, tout;
      if (wave_tensor_map(&tin, a.in, a.nx, a.ny, TCB) && wave_tensor_map(&tout, a.out, a.nx, a.ny, TCB)) {
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        const size_t stage = (size_t)PL::N * TCB * sizeof(float2);
        const size_t slots = (size_t)TCB * tma_col_slot<PL, TCB>() * sizeof(float2);
        const size_t smem = stage > slots ? stage : slots;
        auto kernel = k_pass_b_tma<PL, TCB>;
        static unsigned long long done = 0;
        if (cudaError_t e = set_smem_once(done, kernel, smem)) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(a.nx / TCB, 1);
        cfg.blockDim = dim3(TCB * PL::P);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kernel, a, tin, tout);
      }
    }
  }
  const size_t smem = (size_t)CB * col_slot<PL>() * sizeof(float2) +
                      (col_stages_ky<PL, MODE>() ? (size_t)(PL::N + 1) / 2 * sizeof(float2) : 0) +
                      (col_stages_py<PL, MODE>() ? (size_t)PL::N * sizeof(float2) : 0);
  if (a.nx % CB) return cudaErrorInvalidValue;
  auto kernel = k_pass_b<PL, MODE>;
  static unsigned long long done = 0;
  if (cudaError_t e = set_smem_once(done, kernel, smem)) return e;
  return launch_pdl(kernel, dim3(a.nx / CB, batch), CB * PL::P, smem, s, a);
}

template <class PL>
cudaError_t dispatch_a_plan(const PassAArgs& a, int flags, int batch, cudaStream_t s) {
  switch (flags) {
    case A_FWD: return run_a<PL, A_FWD>(a, batch, s);
    case A_INV: return run_a<PL, A_INV>(a, batch, s);
    case A_MULT_T | A_FWD: return run_a<PL, A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_MULT_T | A_FWD: return run_a<PL, A_INV | A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_INTENSITY: return run_a<PL, A_INV | A_INTENSITY>(a, batch, s);
    case A_INV | A_REAL: return run_a<PL, A_INV | A_REAL>(a, batch, s);
    case A_INV | A_FD | A_FWD: return run_a<PL, A_INV | A_FD | A_FWD>(a, batch, s);
    case A_SAVE | A_MULT_T | A_FWD: return run_a<PL, A_SAVE | A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_SAVE | A_MULT_T | A_FWD: return run_a<PL, A_INV | A_SAVE | A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_RESID: return run_a<PL, A_INV | A_RESID>(a, batch, s);
    case A_INV | A_RESID | A_FWD: return run_a<PL, A_INV | A_RESID | A_FWD>(a, batch, s);
    case A_INV | A_ADJ | A_FWD: return run_a<PL, A_INV | A_ADJ | A_FWD>(a, batch, s);
    case A_MULT_TC | A_FWD: return run_a<PL, A_MULT_TC | A_FWD>(a, batch, s);
    case A_INV | A_MULT_TC | A_FWD: return run_a<PL, A_INV | A_MULT_TC | A_FWD>(a, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class PL>
cudaError_t dispatch_b_plan(const PassBArgs& a, int mode, int batch, cudaStream_t s) {
  switch (mode) {
    case B_FWD_ONLY: return run_b<PL, B_FWD_ONLY>(a, batch, s);
    case B_INV_ONLY: return run_b<PL, B_INV_ONLY>(a, batch, s);
    case B_PROPAGATE: return run_b<PL, B_PROPAGATE>(a, batch, s);
    case B_CTF: return run_b<PL, B_CTF>(a, batch, s);
    case B_CBED: return run_b<PL, B_CBED>(a, batch, s);
    case B_DETECT: return run_b<PL, B_DETECT>(a, batch, s);
    case B_BANDLIMIT: return run_b<PL, B_BANDLIMIT>(a, batch, s);
    case B_FD: return run_b<PL, B_FD>(a, batch, s);
    case B_PROPAGATE_ADJ: return run_b<PL, B_PROPAGATE_ADJ>(a, batch, s);
    case B_CTF_ADJ: return run_b<PL, B_CTF_ADJ>(a, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class PL>
void fill_twiddles(float2* out) {
  const long double twopi = 6.283185307179586476925286766559L;
  const int R[4] = {PL::R1, PL::R2, PL::R3, PL::R4};
  int ns = R[0], off = 0;
  for (int p = 1; p < PL::NPASS; ++p) {
    const int m = ns * R[p];
    for (int r = 0; r < R[p]; ++r)
      for (int k = 0; k < ns; ++k) {
        const long double ang = twopi * (long double)(((long long)r * k) % m) / (long double)m;
        out[off + r * ns + k] = unit_fp32((double)std::cos(ang), (double)(-std::sin(ang)));
      }
    off += m;
    ns = m;
  }
}

// Entry points of one line length (defined in ms_slice_n<N>.cu).
template <int N>
cudaError_t dispatch_a_n(const PassAArgs& a, int variant, int flags, int batch, cudaStream_t s);
template <int N>
cudaError_t dispatch_b_n(const PassBArgs& a, int variant, int mode, int batch, cudaStream_t s);
template <int N>
int twiddles_n(int variant, float2* out);

#define MS_SLICE_INSTANTIATE(N)                                                                      \
  template <>                                                                                        \
  cudaError_t dispatch_a_n<N>(const PassAArgs& a, int variant, int flags, int batch, cudaStream_t s) { \
    switch (variant) {                                                                               \
      case 0: return dispatch_a_plan<PlanSel<N, 0>::T>(a, flags, batch, s);                          \
      case 1: return dispatch_a_plan<PlanSel<N, 1>::T>(a, flags, batch, s);                          \
      case 2: return dispatch_a_plan<PlanSel<N, 2>::T>(a, flags, batch, s);                          \
      case 3: return dispatch_a_plan<PlanSel<N, 3>::T>(a, flags, batch, s);                          \
      case 4: return dispatch_a_plan<PlanSel<N, 4>::T>(a, flags, batch, s);                          \
      case 5: return dispatch_a_plan<PlanSel<N, 5>::T>(a, flags, batch, s);                          \
      default: return cudaErrorInvalidValue;                                                         \
    }                                                                                                \
  }                                                                                                  \
  template <>                                                                                        \
  cudaError_t dispatch_b_n<N>(const PassBArgs& a, int variant, int mode, int batch, cudaStream_t s) {  \
    switch (variant) {                                                                               \
      case 0: return dispatch_b_plan<PlanSel<N, 0>::T>(a, mode, batch, s);                           \
      case 1: return dispatch_b_plan<PlanSel<N, 1>::T>(a, mode, batch, s);                           \
      case 2: return dispatch_b_plan<PlanSel<N, 2>::T>(a, mode, batch, s);                           \
      case 3: return dispatch_b_plan<PlanSel<N, 3>::T>(a, mode, batch, s);                           \
      case 4: return dispatch_b_plan<PlanSel<N, 4>::T>(a, mode, batch, s);                           \
      case 5: return dispatch_b_plan<PlanSel<N, 5>::T>(a, mode, batch, s);                           \
      default: return cudaErrorInvalidValue;                                                         \
    }                                                                                                \
  }                                                                                                  \
  template <>                                                                                        \
  int twiddles_n<N>(int variant, float2* out) {                                                      \
    switch (variant) {                                                                               \
      case 0: fill_twiddles<PlanSel<N, 0>::T>(out); return PlanSel<N, 0>::T::TWSIZE;                 \
      case 1: fill_twiddles<PlanSel<N, 1>::T>(out); return PlanSel<N, 1>::T::TWSIZE;                 \
      case 2: fill_twiddles<PlanSel<N, 2>::T>(out); return PlanSel<N, 2>::T::TWSIZE;                 \
      case 3: fill_twiddles<PlanSel<N, 3>::T>(out); return PlanSel<N, 3>::T::TWSIZE;                 \
      case 4: fill_twiddles<PlanSel<N, 4>::T>(out); return PlanSel<N, 4>::T::TWSIZE;                 \
      case 5: fill_twiddles<PlanSel<N, 5>::T>(out); return PlanSel<N, 5>::T::TWSIZE;                 \
      default: return 0;                                                                             \
    }                                                                                                \
  }

}  // namespace ms
