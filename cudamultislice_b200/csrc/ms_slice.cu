// ms_slice.cu -- fused slice-step passes (see ms_slice.cuh for the scheme).
#include <cmath>

#include "ms_ctf.cuh"
#include "ms_fft.cuh"
#include "ms_slice.cuh"

namespace ms {

namespace {

constexpr int kWarpsA = 4;
constexpr int kWarpsB = 4;

// Line slot strides (in points).  Rows: consecutive slots 8 points (mod 16)
// apart so two 8-thread lines sharing a 16-lane phase use disjoint banks.
// Columns: slots 2 points (mod 16) apart so the transposing tile load (8
// columns x 2 rows per 16-lane phase) is conflict-free.
template <int N>
__host__ __device__ constexpr int stride_rows() {
  return ((N + N / fft::Plan<N>::E + 15) / 16) * 16 + 8;
}
template <int N>
__host__ __device__ constexpr int stride_cols() {
  return ((N + N / fft::Plan<N>::E + 15) / 16) * 16 + 2;
}

template <int NX, int FLAGS>
__global__ void __launch_bounds__(kWarpsA * 32) k_pass_a(PassAArgs a) {
  using PL = fft::Plan<NX>;
  constexpr int E = PL::E, P = PL::P, LPW = 32 / P, LS = stride_rows<NX>();
  extern __shared__ float2 smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / P, t = lane % P;
  const int line = (blockIdx.x * kWarpsA + warp) * LPW + g;
  float2* sm = smem + (warp * LPW + g) * LS;
  const long long inst = blockIdx.y;
  const long long row0 = inst * a.batch_stride_wave + (long long)line * NX;

  float2 v[E];
  const float2* in = a.in + row0;
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = in[t + P * j];

  if constexpr ((FLAGS & A_INV) != 0) fft::line_fft<NX, true>(v, sm, t, a.tw);
  if constexpr ((FLAGS & A_MULT_T) != 0) {
    const float* V = a.V + inst * a.batch_stride_V + (long long)line * NX;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      float s, c;
      sincosf(fmul_x(a.sigma, V[t + P * j]), &s, &c);
      v[j] = cmul(v[j], make_float2(c, s));
    }
  }
  if constexpr ((FLAGS & A_FWD) != 0) fft::line_fft<NX, false>(v, sm, t, a.tw);

  if constexpr ((FLAGS & A_INTENSITY) != 0) {
    float* o = a.out_f + row0;
#pragma unroll
    for (int j = 0; j < E; ++j) o[t + P * j] = (v[j].x * v[j].x + v[j].y * v[j].y) * a.scale;
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

template <int NY, int MODE>
__global__ void __launch_bounds__(kWarpsB * 32) k_pass_b(PassBArgs a, float scale) {
  using PL = fft::Plan<NY>;
  constexpr int E = PL::E, P = PL::P, LPW = 32 / P, CB = kWarpsB * LPW, LS = stride_cols<NY>();
  constexpr int NT = kWarpsB * 32;
  extern __shared__ float2 smem[];
  const int nx = a.nx;
  const int c0 = blockIdx.x * CB;
  const long long base = (long long)blockIdx.y * a.batch_stride_wave;
  const float2* in = a.in + base;

  // transposing tile load: NY rows x CB columns -> one padded slot per column
  for (int idx = threadIdx.x; idx < NY * CB; idx += NT) {
    const int r = idx / CB, c = idx % CB;
    smem[c * LS + fft::padi<NY>(r)] = in[(long long)r * nx + c0 + c];
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / P, t = lane % P;
  const int cl = warp * LPW + g;
  const int col = c0 + cl;
  float2* sm = smem + cl * LS;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = sm[fft::padi<NY>(t + P * j)];
  __syncwarp();

  if constexpr (MODE == B_INV_ONLY) {
    fft::line_fft<NY, true>(v, sm, t, a.tw);
  } else {
    fft::line_fft<NY, false>(v, sm, t, a.tw);
  }

  if constexpr (MODE == B_PROPAGATE) {
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    const float2 pxv = a.px[col];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = a.ky[n];
      // CreatePropsKernel (U.cu:419): keep sqrtf(kx^2+ky^2) < kmax
      const bool keep = fsqrt_x(fadd_x(kx2, fmul_x(ky, ky))) < a.kmax;
      const float2 w = keep ? cmul(pxv, a.py[n]) : make_float2(0.f, 0.f);
      v[j] = cmul(v[j], w);
    }
    fft::line_fft<NY, true>(v, sm, t, a.tw);
  } else if constexpr (MODE == B_CTF) {
    const float kx = a.kx[col];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      v[j] = cmul(v[j], ctf_weight(a.ctf.wavel, a.ctf.Cs, a.ctf.df, a.ctf.A2, a.ctf.phi2, a.ctf.A3, a.ctf.phi3, a.ctf.beta, a.ctf.delta, a.ctf.objap2, kx, a.ky[n], scale));
    }
    fft::line_fft<NY, true>(v, sm, t, a.tw);
  } else if constexpr (MODE == B_CBED) {
    // AddTDSWaves (U.cu:2734-2766): |FFT(psi)| placed by CentreKernel's shift
    const int ny = NY;
    const int xs = (col < nx / 2) ? col + nx / 2 : col - nx / 2;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const int ys = (n < ny / 2) ? n + ny / 2 : n - ny / 2;
      const float m = sqrtf(v[j].x * v[j].x + v[j].y * v[j].y) * scale;
      atomicAdd(a.acc + (long long)ys * nx + xs, m);
    }
    return;  // nothing to store back
  } else if constexpr (MODE == B_DETECT) {
    // |FFT2(psi_exit)|^2 = |P|^2 |FFT_col(Y)|^2: the last propagation only
    // masks, so the detector reads the column spectrum before the inverse.
    const float kx = a.kx[col];
    const float kx2 = fmul_x(kx, kx);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int n = t + P * j;
      const float ky = a.ky[n];
      const float k2 = fadd_x(kx2, fmul_x(ky, ky));
      const bool keep = fsqrt_x(k2) < a.kmax && k2 >= a.kin2 && k2 < a.kout2;
      if (keep) acc += v[j].x * v[j].x + v[j].y * v[j].y;
    }
    double d = (double)acc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if (lane == 0 && d != 0.0) atomicAdd(a.sig + blockIdx.y, d * (double)scale);
    return;
  }

  __syncthreads();  // every slot's FFT scratch use is finished
#pragma unroll
  for (int j = 0; j < E; ++j) sm[fft::padi<NY>(t + P * j)] = v[j];
  __syncthreads();
  float2* out = a.out + base;
  for (int idx = threadIdx.x; idx < NY * CB; idx += NT) {
    const int r = idx / CB, c = idx % CB;
    out[(long long)r * nx + c0 + c] = smem[c * LS + fft::padi<NY>(r)];
  }
}

template <int NX, int FLAGS>
cudaError_t run_a(const PassAArgs& a, int batch, cudaStream_t s) {
  constexpr int LPW = 32 / fft::Plan<NX>::P;
  constexpr int lines = kWarpsA * LPW;
  const size_t smem = (size_t)lines * stride_rows<NX>() * sizeof(float2);
  if (a.ny % lines) return cudaErrorInvalidValue;
  static unsigned long long attr_done = 0;  // one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr_done >> dev & 1ull)) {
    cudaError_t e = cudaFuncSetAttribute(k_pass_a<NX, FLAGS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done |= 1ull << dev;
  }
  dim3 grid(a.ny / lines, batch);
  k_pass_a<NX, FLAGS><<<grid, kWarpsA * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <int NY, int MODE>
cudaError_t run_b(const PassBArgs& a, float scale, int batch, cudaStream_t s) {
  constexpr int LPW = 32 / fft::Plan<NY>::P;
  constexpr int CB = kWarpsB * LPW;
  const size_t smem = (size_t)CB * stride_cols<NY>() * sizeof(float2);
  if (a.nx % CB) return cudaErrorInvalidValue;
  static unsigned long long attr_done = 0;  // one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr_done >> dev & 1ull)) {
    cudaError_t e = cudaFuncSetAttribute(k_pass_b<NY, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done |= 1ull << dev;
  }
  dim3 grid(a.nx / CB, batch);
  k_pass_b<NY, MODE><<<grid, kWarpsB * 32, smem, s>>>(a, scale);
  return cudaGetLastError();
}

template <int NX>
cudaError_t dispatch_a_flags(const PassAArgs& a, int flags, int batch, cudaStream_t s) {
  switch (flags) {
    case A_FWD: return run_a<NX, A_FWD>(a, batch, s);
    case A_INV: return run_a<NX, A_INV>(a, batch, s);
    case A_MULT_T | A_FWD: return run_a<NX, A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_MULT_T | A_FWD: return run_a<NX, A_INV | A_MULT_T | A_FWD>(a, batch, s);
    case A_INV | A_INTENSITY: return run_a<NX, A_INV | A_INTENSITY>(a, batch, s);
    case A_MULT_T: return run_a<NX, A_MULT_T>(a, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int NY>
cudaError_t dispatch_b_mode(const PassBArgs& a, int mode, float scale, int batch, cudaStream_t s) {
  switch (mode) {
    case B_FWD_ONLY: return run_b<NY, B_FWD_ONLY>(a, scale, batch, s);
    case B_INV_ONLY: return run_b<NY, B_INV_ONLY>(a, scale, batch, s);
    case B_PROPAGATE: return run_b<NY, B_PROPAGATE>(a, scale, batch, s);
    case B_CTF: return run_b<NY, B_CTF>(a, scale, batch, s);
    case B_CBED: return run_b<NY, B_CBED>(a, scale, batch, s);
    case B_DETECT: return run_b<NY, B_DETECT>(a, scale, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

int plan_e(int n) {
  switch (n) {
    case 64: return fft::Plan<64>::E;
    case 128: return fft::Plan<128>::E;
    case 256: return fft::Plan<256>::E;
    case 512: return fft::Plan<512>::E;
    case 1024: return fft::Plan<1024>::E;
    default: return 0;
  }
}

}  // namespace

bool fused_supported(int nx, int ny) { return plan_e(nx) > 0 && plan_e(ny) > 0; }

void make_twiddles(int n, float2* out) {
  const int E = plan_e(n), P = n / E;
  const long double twopi = 6.283185307179586476925286766559L;
  for (int r = 0; r < P; ++r)
    for (int i = 0; i < E; ++i) {
      const long long m = (long long)r * i % n;
      const long double ang = twopi * (long double)m / (long double)n;
      out[r * E + i] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
    }
}

cudaError_t launch_pass_a(const PassAArgs& a, int flags, int batch, cudaStream_t s) {
  switch (a.nx) {
    case 64: return dispatch_a_flags<64>(a, flags, batch, s);
    case 128: return dispatch_a_flags<128>(a, flags, batch, s);
    case 256: return dispatch_a_flags<256>(a, flags, batch, s);
    case 512: return dispatch_a_flags<512>(a, flags, batch, s);
    case 1024: return dispatch_a_flags<1024>(a, flags, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_pass_b(const PassBArgs& a, int mode, int batch, cudaStream_t s) {
  const float scale = a.scale;
  switch (a.ny) {
    case 64: return dispatch_b_mode<64>(a, mode, scale, batch, s);
    case 128: return dispatch_b_mode<128>(a, mode, scale, batch, s);
    case 256: return dispatch_b_mode<256>(a, mode, scale, batch, s);
    case 512: return dispatch_b_mode<512>(a, mode, scale, batch, s);
    case 1024: return dispatch_b_mode<1024>(a, mode, scale, batch, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ms
