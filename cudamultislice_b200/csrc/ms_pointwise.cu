// ms_pointwise.cu -- element-wise kernels (plain path, finite differences,
// probe, read-out).  Launch shape is the reference's: 32 x 8 threads per
// block, one thread per pixel, row-major index y*nx + x.
#include <cmath>

#include "ms_ctf.cuh"
#include "ms_philox.h"
#include "ms_pointwise.cuh"

namespace ms {

namespace {

constexpr int kBX = 32, kBY = 8;

inline dim3 grid_of(Grid2 g) { return dim3((g.nx + kBX - 1) / kBX, (g.ny + kBY - 1) / kBY); }

#define PW_INDEX                                         \
  const int x = blockIdx.x * kBX + threadIdx.x;          \
  const int y = blockIdx.y * kBY + threadIdx.y;          \
  if (x >= g.nx || y >= g.ny) return;                    \
  const long long i = (long long)y * g.nx + x;

// initializingKernel U.cu:305-319
__global__ void k_fill(float2* a, Grid2 g, float2 v) {
  PW_INDEX
  a[i] = v;
}

// transmission exp(i sigma V) as written by binnedAtomPKernel3 (U.cu:651-652)
__global__ void k_transmission(const float* V, float sigma, float2* t, Grid2 g) {
  PW_INDEX
  float s, c;
  sincosf(fmul_x(sigma, V[i]), &s, &c);
  t[i] = make_float2(c, s);
}

// multiplicationKernel U.cu:385-397
__global__ void k_cmul(const float2* a, const float2* b, float2* out, float scale, Grid2 g) {
  PW_INDEX
  out[i] = cscale(cmul(a[i], b[i]), scale);
}

// normalisingKernel U.cu:430-443
__global__ void k_scale(float2* a, float scale, Grid2 g) {
  PW_INDEX
  a[i] = cscale(a[i], scale);
}

// CreatePropsKernel U.cu:399-428; the phase pi*dz*lambda*k^2 in FP64.
__global__ void k_props(const float* kx, const float* ky, float dz, float wavel, float kmax, float2* P,
                        Grid2 g) {
  PW_INDEX
  const float k0x = fmul_x(kx[x], kx[x]), k0y = fmul_x(ky[y], ky[y]);
  if (fsqrt_x(fadd_x(k0x, k0y)) < kmax) {
    const double kk = (double)kx[x] * kx[x] + (double)ky[y] * ky[y];
    const double ph = 3.14159265 * (double)dz * (double)wavel * kk;
    const double twopi = 6.283185307179586;
    float s, c;
    sincosf((float)(ph - twopi * rint(ph / twopi)), &s, &c);
    P[i] = make_float2(c, -s);
  } else {
    P[i] = make_float2(0.f, 0.f);
  }
}

// BandLimitKernel U.cu:1025-1042 (keep k <= kmax), with a scale folded in.
__global__ void k_bandlimit(float2* F, const float* kx, const float* ky, float kmax, float scale, Grid2 g) {
  PW_INDEX
  const float k = fsqrt_x(fadd_x(fmul_x(kx[x], kx[x]), fmul_x(ky[y], ky[y])));
  F[i] = (k <= kmax) ? cscale(F[i], scale) : make_float2(0.f, 0.f);
}

// gradKernel U.cu:948-962: F *= scale * (-4 pi^2 k^2), pi = 3.14159.
__global__ void k_laplacian(float2* F, const float* kx, const float* ky, float scale, Grid2 g) {
  PW_INDEX
  const float k2 = kx[x] * kx[x] + ky[y] * ky[y];
  F[i] = cscale(F[i], scale * k2);
}

// finiteDifferenceKernel U.cu:995-1023 with its coefficients precomputed:
// psi+ = rc * (2 psi - dz^2 grad - kv V psi) - ratio * psi-.
struct FdCoef {
  float2 rc, ratio;
  float dz2, kv;
};
__global__ void k_fd_update(const float2* grad, const float2* psim, float2* psip, const float2* psi,
                            const float2* V, FdCoef c, Grid2 g) {
  PW_INDEX
  const float2 p = psi[i], gr = grad[i], m = psim[i];
  const float v = V[i].x;
  const float2 A = make_float2(2.f * p.x - c.dz2 * gr.x - c.kv * v * p.x, 2.f * p.y - c.dz2 * gr.y - c.kv * v * p.y);
  psip[i] = csub(cmul(c.rc, A), cmul(c.ratio, m));
}

// STEMinitializingKernel U.cu:354-383: exp(i(2 pi k.r0 - chi)) inside the
// condenser aperture; both phases in FP64.
__global__ void k_probe(float2* P, const float* kx, const float* ky, int px, int py, float apert, float ps,
                        float df, float Cs, float wavel, Grid2 g) {
  PW_INDEX
  const float kf = fsqrt_x(fadd_x(fmul_x(kx[x], kx[x]), fmul_x(ky[y], ky[y])));
  if (kf < apert) {
    const double kxd = kx[x], kyd = ky[y], k2 = kxd * kxd + kyd * kyd, lam = wavel;
    const double chi = 3.14159265 * lam * k2 * ((double)Cs * lam * lam * k2 * 0.5 + (double)df);
    const double phi = 2.0 * 3.14159265 * (kxd * px * (double)ps + kyd * py * (double)ps);
    const double ph = phi - chi, twopi = 6.283185307179586;
    float s, c;
    sincosf((float)(ph - twopi * rint(ph / twopi)), &s, &c);
    P[i] = make_float2(c, s);
  } else {
    P[i] = make_float2(0.f, 0.f);
  }
}

// k_probe for a batch: blockIdx.z selects the probe position.
__global__ void k_probe_batch(float2* P, long long stride, const float* kx, const float* ky, const int* pxs,
                              const int* pys, float apert, float ps, float df, float Cs, float wavel, Grid2 g) {
  PW_INDEX
  const int b = blockIdx.z;
  const float kf = fsqrt_x(fadd_x(fmul_x(kx[x], kx[x]), fmul_x(ky[y], ky[y])));
  float2 v = make_float2(0.f, 0.f);
  if (kf < apert) {
    const double kxd = kx[x], kyd = ky[y], k2 = kxd * kxd + kyd * kyd, lam = wavel;
    const double chi = 3.14159265 * lam * k2 * ((double)Cs * lam * lam * k2 * 0.5 + (double)df);
    const double phi = 2.0 * 3.14159265 * (kxd * pxs[b] * (double)ps + kyd * pys[b] * (double)ps);
    const double ph = phi - chi, twopi = 6.283185307179586;
    float sn, cs;
    sincosf((float)(ph - twopi * rint(ph / twopi)), &sn, &cs);
    v = make_float2(cs, sn);
  }
  P[b * stride + i] = v;
}

// makeComplex U.cu:322-336
__global__ void k_real_to_complex(const float* in, float2* out, Grid2 g) {
  PW_INDEX
  out[i] = make_float2(in[i], 0.f);
}

// CentreKernel U.cu:964-993 + conjugationKernel mode 1, accumulated.
__global__ void k_centre_abs_acc(const float2* F, float* acc, float scale, Grid2 g) {
  PW_INDEX
  int x2 = x + g.nx / 2, y2 = y + g.ny / 2;
  if (x >= g.nx / 2) x2 = x - g.nx / 2;
  if (y >= g.ny / 2) y2 = y - g.ny / 2;
  const float2 v = F[(long long)y2 * g.nx + x2];
  acc[i] += sqrtf(v.x * v.x + v.y * v.y) * scale;
}

__global__ void k_centre(const float2* F, float2* out, Grid2 g) {
  PW_INDEX
  int x2 = x + g.nx / 2, y2 = y + g.ny / 2;
  if (x >= g.nx / 2) x2 = x - g.nx / 2;
  if (y >= g.ny / 2) y2 = y - g.ny / 2;
  out[i] = F[(long long)y2 * g.nx + x2];
}

__global__ void k_transpose(const float2* in, float2* out, Grid2 g) {
  PW_INDEX
  out[(long long)x * g.ny + y] = in[i];
}

__global__ void k_abs2(const float2* a, float* out, float scale, Grid2 g) {
  PW_INDEX
  const float2 v = a[i];
  out[i] = (v.x * v.x + v.y * v.y) * scale;
}

// One term of MultisliceStepRS's series (RSMS U.cu:849-877 over
// DifferentialXKernel + DifferentialYKernel U.cu:797-847, as written):
//   m = 1:  out = 1 + i pre V
//   m > 1:  out = w + i pre (L w + V w),
//   L w = inv_ps2 (4/3 (w[+1] + w[-1] - w) - 1/12 (w[+2] + w[-2] - w)) per direction,
// neighbours beyond an edge read at index 0 of the line ((i>0)*(i-1) indices).
__global__ void k_rs_term(const float2* w, float2* out, const float* V, float pre, float inv_ps2, int m, Grid2 g) {
  PW_INDEX
  if (m == 1) {
    out[i] = make_float2(1.0f, pre * V[i]);
    return;
  }
  const int p1 = (x > 0) * (x - 1), p2 = (x > 1) * (x - 2);
  const int n1 = (x < g.nx - 1) * (x + 1), n2 = (x < g.nx - 2) * (x + 2);
  const int q1 = (y > 0) * (y - 1), q2 = (y > 1) * (y - 2);
  const int o1 = (y < g.ny - 1) * (y + 1), o2 = (y < g.ny - 2) * (y + 2);
  const long long row = (long long)y * g.nx;
  const float2 c = w[i];
  const float2 dx1 = csub(cadd(w[row + n1], w[row + p1]), c), dx2 = csub(cadd(w[row + n2], w[row + p2]), c);
  const float2 dy1 = csub(cadd(w[(long long)o1 * g.nx + x], w[(long long)q1 * g.nx + x]), c);
  const float2 dy2 = csub(cadd(w[(long long)o2 * g.nx + x], w[(long long)q2 * g.nx + x]), c);
  const float lx = inv_ps2 * (4.0f * dx1.x / 3.0f - dx2.x / 12.0f) + inv_ps2 * (4.0f * dy1.x / 3.0f - dy2.x / 12.0f);
  const float ly = inv_ps2 * (4.0f * dx1.y / 3.0f - dx2.y / 12.0f) + inv_ps2 * (4.0f * dy1.y / 3.0f - dy2.y / 12.0f);
  const float v = V[i];
  out[i] = make_float2(c.x - pre * (ly + v * c.y), c.y + pre * (lx + v * c.x));
}

// Detector transfer of the noisy image chain (DQEFunc/DQEKernel/NTFKernel,
// U.cu:1120-1186): the table entry at floor(sqrtf(dx^2 + dy^2) / binning), dx,
// dy the frequency-index distances to the nearest corner, 0.0001 beyond the
// table; the square root of it for the DQE stage.  `scale` carries the FFT
// normalisations of both transforms around the filter.
__global__ void k_detector_filter(float2* F, const float* tab, int n, int binning, int use_sqrt, float scale, Grid2 g) {
  PW_INDEX
  const int xd = x - (x < g.nx / 2 ? 0 : g.nx), yd = y - (y < g.ny / 2 ? 0 : g.ny);
  const float rad = sqrtf((float)(xd * xd + yd * yd)) / binning;
  const int r2 = (int)floorf(rad);
  float v = r2 <= n - 1 ? tab[r2] : 0.0001f;
  if (use_sqrt) v = sqrtf(v);
  F[i] = cscale(cscale(F[i], v), scale);
}

// Shot noise of the chain (U.cu:2383-2409): counts = round(dose a + sqrt(|dose a|) z)
// with a = |F| and z the clipped normal of Philox4x32-10 at counter
// (pixel, serial, 0x5407, 0) under key (seed lo, seed hi).
__global__ void k_shot_noise(const float2* F, float* counts, float dose, uint32_t k0, uint32_t k1, uint32_t serial,
                             Grid2 g) {
  PW_INDEX
  const float a = sqrtf(F[i].x * F[i].x + F[i].y * F[i].y);
  const uint32_t ctr[4] = {(uint32_t)i, serial, 0x5407u, 0u}, key[2] = {k0, k1};
  uint32_t r[4];
  philox4x32_10(ctr, key, r);
  const double z = clipped_normal(r[0], r[1]);
  const float na = dose * a;
  counts[i] = (float)round((double)na + (double)sqrtf(fabsf(na)) * z);
}

__global__ void k_abs(const float2* a, float* out, Grid2 g) {
  PW_INDEX
  out[i] = sqrtf(a[i].x * a[i].x + a[i].y * a[i].y);
}

// Transmission exp(i sigma V) of n values with the fused row pass's sincos
// (identical values to the on-the-fly transmission).
__global__ void k_transmission_stack(const float* V, float sigma, float2* t, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float sn, cs;
  sincos_red(fmul_x(sigma, V[i]), &sn, &cs);
  t[i] = make_float2(cs, sn);
}

// acc += scale * sum_b in[b * stride + i] (batched images into one sum)
__global__ void k_add_batch(const float* in, long long stride, int nb, float* acc, float scale, Grid2 g) {
  PW_INDEX
  float s = 0.0f;
  for (int b = 0; b < nb; ++b) s += in[(long long)b * stride + i];
  acc[i] += scale * s;
}

__global__ void k_ctf(float2* F, const float* kx, const float* ky, double wavel, double Cs, double df, double A2,
                      double phi2, double beta, double delta, float objap2, float scale, Grid2 g) {
  PW_INDEX
  F[i] = cmul(F[i], ctf_weight(wavel, Cs, df, A2, phi2, 0.0, 0.0, beta, delta, objap2, kx[x], ky[y], scale));
}

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1024;

__device__ __forceinline__ double block_sum_d(double v) {
  __shared__ double s[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < kRedThreads / 32) ? s[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_abs(const float2* a, long long n, double* partial) {
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads) {
    const float2 v = a[i];
    acc += sqrt((double)v.x * v.x + (double)v.y * v.y);
  }
  const double r = block_sum_d(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_abs_batch(const float2* a, long long n, long long stride,
                                                               double* partial) {
  const float2* ab = a + blockIdx.y * stride;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads) {
    const float2 v = ab[i];
    acc += sqrt((double)v.x * v.x + (double)v.y * v.y);
  }
  const double r = block_sum_d(acc);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = r;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_partials_batch(const double* partial, int nb, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += kRedThreads) acc += partial[blockIdx.x * nb + i];
  const double r = block_sum_d(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kRedThreads) k_annular(const float2* F, const float* kx, const float* ky,
                                                         float kin2, float kout2, Grid2 g, double* partial) {
  const long long n = (long long)g.nx * g.ny;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads) {
    const int x = (int)(i % g.nx), y = (int)(i / g.nx);
    const float k2 = fadd_x(fmul_x(kx[x], kx[x]), fmul_x(ky[y], ky[y]));
    if (k2 >= kin2 && k2 < kout2) {
      const float2 v = F[i];
      acc += (double)v.x * v.x + (double)v.y * v.y;
    }
  }
  const double r = block_sum_d(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_partials(const double* partial, int nb, double scale,
                                                              double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += kRedThreads) acc += partial[i];
  const double r = block_sum_d(acc);
  if (threadIdx.x == 0) *out = r * scale;
}

}  // namespace

#define PW_LAUNCH(kern, ...)                                            \
  do {                                                                  \
    kern<<<grid_of(g), dim3(kBX, kBY), 0, s>>>(__VA_ARGS__);            \
    if (count) ++*count;                                                \
    return cudaGetLastError();                                          \
  } while (0)

cudaError_t pw_fill(float2* a, Grid2 g, float2 v, cudaStream_t s, long long* count) { PW_LAUNCH(k_fill, a, g, v); }
cudaError_t pw_transmission(const float* V, float sigma, float2* t, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_transmission, V, sigma, t, g);
}
cudaError_t pw_cmul(const float2* a, const float2* b, float2* out, float scale, Grid2 g, cudaStream_t s,
                    long long* count) {
  PW_LAUNCH(k_cmul, a, b, out, scale, g);
}
cudaError_t pw_scale(float2* a, float scale, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_scale, a, scale, g);
}
cudaError_t pw_props(const float* kx, const float* ky, float dz, float wavel, float kmax, float2* P, Grid2 g,
                     cudaStream_t s, long long* count) {
  PW_LAUNCH(k_props, kx, ky, dz, wavel, kmax, P, g);
}
cudaError_t pw_bandlimit(float2* F, const float* kx, const float* ky, float kmax, float scale, Grid2 g,
                         cudaStream_t s, long long* count) {
  PW_LAUNCH(k_bandlimit, F, kx, ky, kmax, scale, g);
}
cudaError_t pw_laplacian(float2* F, const float* kx, const float* ky, float scale, Grid2 g, cudaStream_t s,
                         long long* count) {
  const float coef = (float)(-4.0 * 3.14159 * 3.14159) * scale;
  PW_LAUNCH(k_laplacian, F, kx, ky, coef, g);
}
cudaError_t pw_fd_update(const float2* grad, const float2* psim, float2* psip, const float2* psi,
                         const float2* V, float sigma, float wavel, float dz, Grid2 g, cudaStream_t s,
                         long long* count) {
  // coefficients of finiteDifferenceKernel (U.cu:1006-1010) in FP64, pi = 3.14159
  const double a = 2.0 * 3.14159 * (double)dz / (double)wavel;
  const double den = 1.0 + a * a;
  FdCoef c;
  c.rc = make_float2((float)(1.0 / den), (float)(-a / den));
  c.ratio = make_float2((float)((1.0 - a * a) / den), (float)(-2.0 * a / den));
  c.dz2 = (float)((double)dz * dz);
  c.kv = (float)((double)dz * dz * 4.0 * 3.14159 * (double)sigma / (double)wavel);
  PW_LAUNCH(k_fd_update, grad, psim, psip, psi, V, c, g);
}
cudaError_t pw_probe(float2* P, const float* kx, const float* ky, int px, int py, float apert, float ps,
                     float df, float Cs, float wavel, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_probe, P, kx, ky, px, py, apert, ps, df, Cs, wavel, g);
}
cudaError_t pw_real_to_complex(const float* in, float2* out, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_real_to_complex, in, out, g);
}
cudaError_t pw_centre_abs_acc(const float2* F, float* acc, float scale, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_centre_abs_acc, F, acc, scale, g);
}
cudaError_t pw_centre(const float2* F, float2* out, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_centre, F, out, g);
}
cudaError_t pw_transpose(const float2* in, float2* out, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_transpose, in, out, g);
}
cudaError_t pw_abs2(const float2* a, float* out, float scale, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_abs2, a, out, scale, g);
}
cudaError_t pw_add_batch(const float* in, long long stride, int nb, float* acc, float scale, Grid2 g, cudaStream_t s,
                         long long* count) {
  PW_LAUNCH(k_add_batch, in, stride, nb, acc, scale, g);
}
cudaError_t pw_detector_filter(float2* F, const float* tab, int n, int binning, bool use_sqrt, float scale, Grid2 g,
                               cudaStream_t s, long long* count) {
  PW_LAUNCH(k_detector_filter, F, tab, n, binning, use_sqrt ? 1 : 0, scale, g);
}
cudaError_t pw_shot_noise(const float2* F, float* counts, float dose, uint64_t seed, uint32_t serial, Grid2 g,
                          cudaStream_t s, long long* count) {
  PW_LAUNCH(k_shot_noise, F, counts, dose, (uint32_t)seed, (uint32_t)(seed >> 32), serial, g);
}
cudaError_t pw_abs(const float2* a, float* out, Grid2 g, cudaStream_t s, long long* count) {
  PW_LAUNCH(k_abs, a, out, g);
}
cudaError_t pw_transmission_stack(const float* V, float sigma, float2* t, long long n, cudaStream_t s,
                                  long long* count) {
  k_transmission_stack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(V, sigma, t, n);
  if (count) ++*count;
  return cudaGetLastError();
}
cudaError_t pw_rs_term(const float2* w, float2* out, const float* V, float pre, float inv_ps2, int m, Grid2 g,
                       cudaStream_t s, long long* count) {
  PW_LAUNCH(k_rs_term, w, out, V, pre, inv_ps2, m, g);
}
cudaError_t pw_ctf(float2* F, const float* kx, const float* ky, double wavel, double Cs, double df, double A2,
                   double phi2, double beta, double delta, float objap2, float scale, Grid2 g, cudaStream_t s,
                   long long* count) {
  PW_LAUNCH(k_ctf, F, kx, ky, wavel, Cs, df, A2, phi2, beta, delta, objap2, scale, g);
}

int pw_reduce_blocks(long long n) {
  long long b = (n + kRedThreads - 1) / kRedThreads;
  return (int)(b < kRedMaxBlocks ? (b < 1 ? 1 : b) : kRedMaxBlocks);
}

cudaError_t pw_sum_abs(const float2* a, long long n, double* partial, double* out, cudaStream_t s,
                       long long* count) {
  const int nb = pw_reduce_blocks(n);
  k_sum_abs<<<nb, kRedThreads, 0, s>>>(a, n, partial);
  k_sum_partials<<<1, kRedThreads, 0, s>>>(partial, nb, 1.0, out);
  if (count) *count += 2;
  return cudaGetLastError();
}

cudaError_t pw_probe_batch(float2* P, long long stride, int nb, const float* kx, const float* ky, const int* px,
                           const int* py, float apert, float ps, float df, float Cs, float wavel, Grid2 g,
                           cudaStream_t s, long long* count) {
  dim3 grid = grid_of(g);
  grid.z = nb;
  k_probe_batch<<<grid, dim3(kBX, kBY), 0, s>>>(P, stride, kx, ky, px, py, apert, ps, df, Cs, wavel, g);
  if (count) ++*count;
  return cudaGetLastError();
}

cudaError_t pw_sum_abs_batch(const float2* a, long long n, long long stride, int nb, double* partial, double* out,
                             cudaStream_t s, long long* count) {
  const int blocks = pw_reduce_blocks(n);
  k_sum_abs_batch<<<dim3(blocks, nb), kRedThreads, 0, s>>>(a, n, stride, partial);
  k_sum_partials_batch<<<nb, kRedThreads, 0, s>>>(partial, blocks, out);
  if (count) *count += 2;
  return cudaGetLastError();
}

cudaError_t pw_annular(const float2* F, const float* kx, const float* ky, float kin2, float kout2, double scale,
                       Grid2 g, double* partial, double* out, cudaStream_t s, long long* count) {
  const int nb = pw_reduce_blocks((long long)g.nx * g.ny);
  k_annular<<<nb, kRedThreads, 0, s>>>(F, kx, ky, kin2, kout2, g, partial);
  k_sum_partials<<<1, kRedThreads, 0, s>>>(partial, nb, scale, out);
  if (count) *count += 2;
  return cudaGetLastError();
}

}  // namespace ms
