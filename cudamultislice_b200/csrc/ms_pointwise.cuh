// ms_pointwise.cuh -- element-wise kernels: the plain (one kernel per
// operation) slice path, finite differences, probe generation, read-out.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "ms_common.cuh"

namespace ms {

struct Grid2 {
  int nx, ny;
};

// Each launcher returns cudaGetLastError() and counts one launch in *count.
cudaError_t pw_fill(float2* a, Grid2 g, float2 v, cudaStream_t s, long long* count);
cudaError_t pw_transmission(const float* V, float sigma, float2* t, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_cmul(const float2* a, const float2* b, float2* out, float scale, Grid2 g, cudaStream_t s,
                    long long* count);
cudaError_t pw_scale(float2* a, float scale, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_props(const float* kx, const float* ky, float dz, float wavel, float kmax, float2* P, Grid2 g,
                     cudaStream_t s, long long* count);
cudaError_t pw_bandlimit(float2* F, const float* kx, const float* ky, float kmax, float scale, Grid2 g,
                         cudaStream_t s, long long* count);
cudaError_t pw_laplacian(float2* F, const float* kx, const float* ky, float scale, Grid2 g, cudaStream_t s,
                         long long* count);
cudaError_t pw_fd_update(const float2* grad, const float2* psim, float2* psip, const float2* psi,
                         const float2* V, float sigma, float wavel, float dz, Grid2 g, cudaStream_t s,
                         long long* count);
cudaError_t pw_probe(float2* P, const float* kx, const float* ky, int px, int py, float apert, float ps,
                     float df, float Cs, float wavel, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_real_to_complex(const float* in, float2* out, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_centre_abs_acc(const float2* F, float* acc, float scale, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_centre(const float2* F, float2* out, Grid2 g, cudaStream_t s, long long* count);
cudaError_t pw_abs2(const float2* a, float* out, float scale, Grid2 g, cudaStream_t s, long long* count);
// Noisy image chain (see .cu): radial detector transfer, seeded shot noise, |.|.
cudaError_t pw_detector_filter(float2* F, const float* tab, int n, int binning, bool use_sqrt, float scale, Grid2 g,
                               cudaStream_t s, long long* count);
cudaError_t pw_shot_noise(const float2* F, float* counts, float dose, uint64_t seed, uint32_t serial, Grid2 g,
                          cudaStream_t s, long long* count);
cudaError_t pw_abs(const float2* a, float* out, Grid2 g, cudaStream_t s, long long* count);
// t = exp(i sigma V) over n values, with the fused row pass's sincos.
cudaError_t pw_transmission_stack(const float* V, float sigma, float2* t, long long n, cudaStream_t s,
                                  long long* count);
// Term m of the real-space (RS) series, as written in the reference (see .cu).
cudaError_t pw_rs_term(const float2* w, float2* out, const float* V, float pre, float inv_ps2, int m, Grid2 g,
                       cudaStream_t s, long long* count);
// acc += scale * sum over nb instances (stride apart) of in.
cudaError_t pw_add_batch(const float* in, long long stride, int nb, float* acc, float scale, Grid2 g, cudaStream_t s,
                         long long* count);
// out[x][y] = in[y][x] (one-time layout changes).
cudaError_t pw_transpose(const float2* in, float2* out, Grid2 g, cudaStream_t s, long long* count);
// CTF multiply for the plain path (same weight as the fused column pass).
cudaError_t pw_ctf(float2* F, const float* kx, const float* ky, double wavel, double Cs, double df, double A2,
                   double phi2, double beta, double delta, float objap2, float scale, Grid2 g, cudaStream_t s,
                   long long* count);
// Sum of |a| (FP64 accumulation, deterministic two-stage tree).  `partial`
// holds pw_reduce_blocks(n) doubles.
int pw_reduce_blocks(long long n);
cudaError_t pw_sum_abs(const float2* a, long long n, double* partial, double* out, cudaStream_t s,
                       long long* count);
// Batched probes: probe b at pixel (px[b], py[b]) into P + b*stride (gridDim.z = b).
cudaError_t pw_probe_batch(float2* P, long long stride, int nb, const float* kx, const float* ky, const int* px,
                           const int* py, float apert, float ps, float df, float Cs, float wavel, Grid2 g,
                           cudaStream_t s, long long* count);
// Per-instance sum of |a| for nb instances of n points: out[b] (FP64).
// `partial` holds nb * pw_reduce_blocks(n) doubles.
cudaError_t pw_sum_abs_batch(const float2* a, long long n, long long stride, int nb, double* partial, double* out,
                             cudaStream_t s, long long* count);
// Annular detector sum over kin2 <= k^2 < kout2 of |F|^2 * scale (FP64).
cudaError_t pw_annular(const float2* F, const float* kx, const float* ky, float kin2, float kout2, double scale,
                       Grid2 g, double* partial, double* out, cudaStream_t s, long long* count);

}  // namespace ms
