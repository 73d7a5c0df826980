// ms_slice.cuh -- launch interface of the fused slice-step passes.
//
// One slice step psi <- IFFT2(P * FFT2(t * psi)) / N is split into two
// line-local passes, because IFFT2 = IFFT_rows o IFFT_cols and consecutive
// steps meet row-to-row:
//   pass A (rows):    [IFFT_row] -> x t = exp(i sigma V) -> FFT_row
//   pass B (columns): FFT_col -> x P(k)/N (band-limited) -> IFFT_col
// Between steps the wave stays in the "row-frequency" domain; a final pass A
// with only IFFT_row returns it to real space.  Each pass reads and writes the
// wave once (8 MB at 1024^2: L2-resident on B200) and pass A streams V.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "ms_common.cuh"

namespace ms {

enum PassAFlags : int {
  A_INV = 1,        // IFFT_row of the input line
  A_MULT_T = 2,     // x exp(i sigma V)
  A_FWD = 4,        // FFT_row
  A_INTENSITY = 8,  // store |.|^2 * scale as float
  A_REAL = 16,      // store the real part * scale as float
  A_FD = 32,        // finite-difference stencil (see PassAArgs.fd_*)
  A_SAVE = 64,      // store the real-space line (before x t) to out2
  A_RESID = 128,    // focal-series residual: I = |.|^2, r = I - T, loss += r^2,
                    // line <- 2 r line (I to out_f when not null)
  A_ADJ = 256,      // adjoint of x t: dV = -2 sigma Im(conj(h) t psi) to out_f
                    // (psi from in2), line <- conj(t) line
  A_MULT_TC = 512,  // x t from a precomputed transmission slice (PassAArgs.tr)
};
enum PassBMode : int {
  B_FWD_ONLY = 0,    // FFT_col
  B_INV_ONLY = 1,    // IFFT_col
  B_PROPAGATE = 2,   // FFT_col, x Px*Py (band-limited), IFFT_col
  B_CTF = 3,         // FFT_col, x CTF(k)/N (objective aperture), IFFT_col
  B_CBED = 4,        // FFT_col, accumulate |.| fftshifted into a float map
  B_DETECT = 5,      // FFT_col, band limit of P, sum |.|^2 over an annulus per instance
  B_BANDLIMIT = 6,   // FFT_col, keep k <= kmax (x scale), IFFT_col
  B_FD = 7,          // FFT_col = Q; spec <- BL Q + fd_c k^2 spec; IFFT_col(spec) * scale
  B_PROPAGATE_ADJ = 8,  // FFT_col, x conj(Px*Py) * scale (band-limited), IFFT_col
  B_CTF_ADJ = 9,        // FFT_col, x conj(CTF(k)) * scale, IFFT_col; out += when accumulate
};

struct PassAArgs {
  const float2* in;   // wave read (may alias out)
  float2* out;        // wave written
  float* out_f;       // intensity output (A_INTENSITY), else unused
  const float* V;     // potential slice [ny][nx] (A_MULT_T)
  float sigma;        // interaction constant
  float scale;        // applied to the result of the line (1 = none)
  // A_FD: the input line is the row-frequency state of psi_n; the pass stores
  // psi_n (real space) to out2 and FFT_row(q) to out, with
  // q = fd_rc * (2 - fd_kv V) psi_n - fd_ratio * psi_{n-1} (psi_{n-1} from in2),
  // the three-level update of finiteDifferenceKernel (U.cu:995-1023) without
  // its Laplacian term, which the column pass adds in k-space.
  const float2* in2;
  float2* out2;
  float2 fd_rc, fd_ratio;
  float fd_kv;
  const float2* tr;   // A_MULT_TC: transmission exp(i sigma V) [ny][nx] (instance stride batch_stride_V)
  const float* T;     // A_RESID: target intensity [ny][nx] (instance stride batch_stride_V)
  double* loss;       // A_RESID: FP64 sum of r^2 (atomic)
  const float2* tw;   // twiddle table for nx
  int nx, ny;
  long long batch_stride_wave;  // elements between instances (blockIdx.y)
  long long batch_stride_V;
};

struct CtfParams {
  double wavel, Cs, df, A2, phi2, A3, phi3, beta, delta;  // beta in rad
  float objap2;                                          // FP32 aperture decision
};

struct PassBArgs {
  const float2* in;
  float2* out;
  float* acc;          // B_CBED accumulation map [ny][nx]
  const float2* tw;    // twiddle table for ny
  const float2* px;    // propagator factor per column (scaled 1/N)
  const float2* py;    // propagator factor per row
  const float* kx;     // FP32 reference frequencies (decisions)
  const float* ky;
  float kmax;
  // the band-limit decisions as thresholds on k^2 = fadd(kx^2, ky^2), set by
  // band_limit_thresholds(): sqrt_rn(k^2) < kmax  <=>  k^2 < k2_lt and
  // sqrt_rn(k^2) <= kmax  <=>  k^2 < k2_le (sqrt_rn is monotone)
  float k2_lt, k2_le;
  CtfParams ctf;
  float scale;         // B_CTF: factor on the weight; B_CBED: factor on |.|
  double* sig;         // B_DETECT: one FP64 sum per instance (blockIdx.y)
  float2* spec;        // B_FD: band-limited spectrum FFT2(psi_n) in, FFT2(psi_{n+1}) out,
                       //       stored column-major [nx][ny] (coalesced in this pass)
  float2 fd_c;         // B_FD: rc dz^2 4 pi^2 (pi = 3.14159, gradKernel U.cu:959)
  float kin2, kout2;   // B_DETECT: annulus kin^2 <= kx^2+ky^2 < kout^2 (FP32 decision)
  int accumulate;      // B_CTF_ADJ: add to out instead of storing
  int nx, ny;
  long long batch_stride_wave;
  // columns of 2048 and 4096 points, propagation, one instance: when set, the
  // column pass stages its columns through shared memory with tensor copies
  // (k_pass_b_tma), and a wait for them that runs out sets this word
  int* err;
};

// The smallest FP32 k^2 with sqrt_rn(k^2) >= kmax (k2_lt) and with
// sqrt_rn(k^2) > kmax (k2_le), found from kmax^2 by stepping one ulp at a time
// against the host's correctly rounded sqrtf, so that a comparison of k^2
// with them takes exactly the decisions of the rounded square root.
void band_limit_thresholds(float kmax, float* k2_lt, float* k2_le);

// (cos, sin) as the FP32 pair within one ulp of each component whose modulus
// is nearest 1 (ties: nearest angle).  Unit factors applied once per transform
// or per slice (twiddles, propagator) then scale the wave by |(c, s)|^S over a
// stack of S slices only to that pair's remaining modulus error, far below the
// plain rounding's, which adds up coherently when the slices repeat (crystals).
float2 unit_fp32(double c, double s);

// Line lengths 64..4096 (powers of two) in both directions.
bool fused_supported(int nx, int ny);
// Number of FFT plan variants per line length (autotuned by the engine).
int plan_variants();
// Twiddle table of plan `variant` for lines of n points into host_out
// (at most 2n entries); returns its length.
int make_twiddles(int n, int variant, float2* host_out);
cudaError_t launch_pass_a(const PassAArgs& a, int variant, int flags, int batch, cudaStream_t s);
cudaError_t launch_pass_b(const PassBArgs& a, int variant, int mode, int batch, cudaStream_t s);

// ---- persistent slice loop (ms_slice_loop.cuh) ----
struct LoopSync {
  unsigned int* count;          // grid-barrier arrivals, zeroed before the launch
  int* error;                   // 0, or kLoopTimeout after a wait ran out
  unsigned long long limit_ns;  // bound on each wait
  unsigned int expect_extra;    // added to every barrier's target: a target the
                                // grid cannot reach (tests of the bound)
};
constexpr int kLoopTimeout = 1;

struct LoopArgs {
  PassAArgs a;          // row phase (twiddles, sigma; the wave set below)
  PassBArgs b;          // column phase (twiddles, propagator, band limit)
  const float2* psi0;   // initial wave (real space), read by slice 1
  float2* wave;         // the wave, left in row-frequency form
  const float* Vstack;  // potentials [S][ny][nx]
  long long vstride;    // floats between slices of the stack
  int S;                // slices
  LoopSync sync;
};
// Batched persistent loop: B instances of one or two square grid sizes
// stepped through the same S slices by one cooperative launch.
struct LoopGroup {
  int n;                   // grid (n x n): 256, 512 or 1024; 0 = group absent
  int B;                   // instances
  float2* wave;            // [B][n][n]: real space on entry, row-frequency form after the loop
  const float* Vstack;     // per-instance potentials (x exp(i sigma V) on the fly), or null
  const float2* tstack;    // transmissions (x t), used when Vstack is null
  long long inst_stride;   // elements between instances' stacks (0: one stack shared by all)
  long long slice_stride;  // elements between slices of a stack
  PassAArgs a;             // row tables (twiddles, sigma)
  PassBArgs b;             // column tables (twiddles, propagator, band limit; detector annulus)
  double* sig;             // last slice: annular-detector sum per instance (then no propagation)
};
struct BatchLoopArgs {
  LoopGroup g[2];
  int S;
  LoopSync sync;
};
// Grids (n0 >= n1; n1 = 0 for one group, n1 = n0 for two of one size) the
// batched loop is provided for.
bool batch_loop_supported(int n0, int n1);
// FFT plan variant (twiddle tables) of the batched loop for lines of n points.
int batch_loop_plan(int n);
// tc: the groups multiply by stored transmissions (else exp(i sigma V) from V).
cudaError_t batch_loop_prepare(int n0, int n1, bool tc, int* grid);
cudaError_t launch_batch_loop(const BatchLoopArgs& L, int grid, cudaStream_t s);

// Grids the persistent loop is provided for (square 256, 512, 1024), and the
// FFT plan variant (twiddle tables) that loop kernel variant `variant` uses.
bool slice_loop_supported(int nx, int ny);
int slice_loop_plan(int n, int variant);
// Kernel variants of the loop (column unit width, grid-barrier form), and the
// columns per unit of one variant.
int slice_loop_variants();
int slice_loop_columns(int variant);
// Raises a loop variant's shared-memory limit and returns its grid (one CTA
// per SM, all resident).
cudaError_t slice_loop_prepare(int n, int variant, int* grid);
// Cooperative launch of the whole slice loop (kernel variant `variant`).
cudaError_t launch_slice_loop(const LoopArgs& L, int variant, int grid, cudaStream_t s);

}  // namespace ms
