// ms_atoms.cu -- bit-exact atom binning and the potential-build kernels.
#include <algorithm>
#include <cmath>

#include "ms_atoms.cuh"

namespace ms {

namespace {

// ---------------------------------------------------------------------------
// Atom binning.  atombin2 (U.cu:277-303) computes, per atom and in FP32,
//   bidx = floor((x - minx) / (maxx - minx) * 50), bidy likewise,
//   zid  = floor((maxz - z) / 1);
// the reference host code then gathers the atoms into a CSR ordered
// slice -> y-bin -> x-bin, stable in input order (U.cu:1444-1525).  Here the
// whole index is built on the device: keys + counts, exclusive scan, scatter,
// a per-bin insertion sort that restores input order, and a gather that
// stores positions shifted by the box minimum.  Every rounding is explicit
// (no FMA contraction), so bins agree bit for bit with the host definition.
// ---------------------------------------------------------------------------
__global__ void k_bin_keys(const float* __restrict__ x, const float* __restrict__ y,
                           const float* __restrict__ z, int n, Box b, int nz,
                           int* __restrict__ key, int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float qx = fdiv_x(fsub_x(x[i], b.MinX), fsub_x(b.MaxX, b.MinX));
  const float qy = fdiv_x(fsub_x(y[i], b.MinY), fsub_x(b.MaxY, b.MinY));
  int bx = (int)floorf(fmul_x(qx, (float)kBins));
  int by = (int)floorf(fmul_x(qy, (float)kBins));
  int bz = (int)floorf(fdiv_x(fsub_x(b.MaxZ, z[i]), 1.0f));
  // The +-2 A box padding keeps imported atoms in range; displaced thermal
  // positions are clamped to the edge bins.
  bx = min(max(bx, 0), kBins - 1);
  by = min(max(by, 0), kBins - 1);
  bz = min(max(bz, 0), nz - 1);
  const int k = bz * kBins2 + by * kBins + bx;
  key[i] = k;
  atomicAdd(count + k, 1);
}

__global__ void k_scatter(const int* __restrict__ key, int n, int* __restrict__ cursor,
                          int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  idx[atomicAdd(cursor + key[i], 1)] = i;
}

// Restores input order inside each bin (bins hold a handful of atoms).
__global__ void k_sort_bins(const int* __restrict__ off, int nbins, int* __restrict__ idx) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const int s = off[b], e = off[b + 1];
  for (int i = s + 1; i < e; ++i) {
    const int v = idx[i];
    int j = i - 1;
    while (j >= s && idx[j] > v) {
      idx[j + 1] = idx[j];
      --j;
    }
    idx[j + 1] = v;
  }
}

__global__ void k_gather(const int* __restrict__ idx, int n, const int* __restrict__ Z,
                         const float* __restrict__ x, const float* __restrict__ y,
                         const float* __restrict__ z, Box b, float4* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = idx[j];
  out[j] = make_float4(fsub_x(x[i], b.MinX), fsub_x(y[i], b.MinY), fsub_x(z[i], b.MinZ),
                       __int_as_float(Z[i]));
}

// ---- exclusive scan of int counts (nbins) into offsets (nbins + 1) ----
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    s_warp[lane] = wi - w;
    if (lane == 31) s_warp[32] = wi;
  }
  __syncthreads();
  const int r = s_warp[warp] + incl - v;
  *total = s_warp[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int* __restrict__ in, int n,
                                                             int* __restrict__ out, int* __restrict__ tile_sums) {
  __shared__ int s_warp[33];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems], sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    sum += v[k];
  }
  int total;
  int run = block_exclusive_scan(sum, s_warp, &total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile sums in place; writes the grand total.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int* __restrict__ sums, int ntiles,
                                                            int* __restrict__ total_out) {
  __shared__ int s_warp[33];
  int carry = 0;
  for (int base = 0; base < ntiles; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const int v = (i < ntiles) ? sums[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, s_warp, &total);
    if (i < ntiles) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ tile_sums) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] += tile_sums[i / kScanTile];
}

// ---------------------------------------------------------------------------
// Potential build.  One CTA covers a 32 x 8 pixel tile (the reference's
// thread-block shape).  The atoms that can reach the tile (xy bins within
// sqrt(5) A plus one bin of margin, z-bins of the window) form a list of
// contiguous CSR segments; the CTA stages them in shared memory in chunks and
// every thread accumulates its pixel with the reference's exact cut-off
// r^2 < 5 A^2 evaluated in non-contracted FP32.
// ---------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 8, kPotThreads = kTX * kTY;

// Pixel of thread `tid` in the 32 x 8 tile: each warp covers an 8 x 4 patch
// (patches 4 across, 2 down), so that the lanes of a warp lie close together
// and agree on which atoms and sub-planes pass the cut-off.
__device__ __forceinline__ void tile_pixel(int tid, int& tx, int& ty) {
  const int w = tid >> 5, l = tid & 31;
  tx = (w & 3) * 8 + (l & 7);
  ty = (w >> 2) * 4 + (l >> 3);
}
constexpr int kChunk = 256;
constexpr int kMaxSeg = 512;

// v(r) of vatom (U.cu:160-193) from precomputed per-Z coefficients:
// c[0..2] = 150.4121417 a_i, c[3..5] = 2 pi sqrt(b_i) log2(e),
// c[6..8] = 266.5157269 c_i d_i^-1.5, c[9..11] = pi^2 / d_i log2(e).
__device__ __forceinline__ float vatom_f(const float* __restrict__ c, float r2) {
  float r = sqrtf(fabsf(r2));
  if (r < 0.25f) r = 0.25f;
  const float rinv = __frcp_rn(r);
  const float L = c[0] * exp2f(-c[3] * r) + c[1] * exp2f(-c[4] * r) + c[2] * exp2f(-c[5] * r);
  const float rr = r * r;
  const float G = c[6] * exp2f(-c[9] * rr) + c[7] * exp2f(-c[10] * rr) + c[8] * exp2f(-c[11] * rr);
  return L * rinv + G;
}

// K0 of bessk0 (U.cu:77-111): the small-argument series (which cancels) in FP64,
// the asymptotic branch in FP32.
__device__ __forceinline__ float bessk0_f(float x) {
  const float ax = fabsf(x);
  if (ax > 2.0f) {
    const float t = 2.0f / ax;
    float s = 0.00053208f;
    s = s * t - 0.00251540f;
    s = s * t + 0.00587872f;
    s = s * t - 0.01062446f;
    s = s * t + 0.02189568f;
    s = s * t - 0.07832358f;
    s = s * t + 1.25331414f;
    return expf(-ax) * s * rsqrtf(ax);
  }
  if (ax > 0.0f) {
    const double xd = ax, h = xd / 2.0, x2 = h * h;
    double s = 0.00000740;
    s = s * x2 + 0.00010750;
    s = s * x2 + 0.00262698;
    s = s * x2 + 0.03488590;
    s = s * x2 + 0.23069756;
    s = s * x2 + 0.42278420;
    s = s * x2 - 0.57721566;
    double t = xd / 3.75;
    t = t * t;
    double i0 = 0.0045813;
    i0 = i0 * t + 0.0360768;
    i0 = i0 * t + 0.2659732;
    i0 = i0 * t + 1.2067492;
    i0 = i0 * t + 3.0899424;
    i0 = i0 * t + 3.5156229;
    i0 = i0 * t + 1.0;
    return (float)(-log(h) * i0 + s);
  }
  return 1.0e20f;
}

// vz(r) of vzatom2 (U.cu:119-152): c[12..14] = 300.8242834 a_i,
// c[15..17] = 2 pi sqrt(b_i), c[18..20] = 150.4121417 c_i / d_i,
// c[21..23] = pi^2 / d_i log2(e).
__device__ __forceinline__ float vzatom2_f(const float* __restrict__ c, float r2) {
  float r = sqrtf(fabsf(r2));
  if (r < 0.25f) r = 0.25f;
  const float L = c[12] * bessk0_f(c[15] * r) + c[13] * bessk0_f(c[16] * r) + c[14] * bessk0_f(c[17] * r);
  const float rr = r * r;
  const float G = c[18] * exp2f(-c[21] * rr) + c[19] * exp2f(-c[22] * rr) + c[20] * exp2f(-c[23] * rr);
  return L + G;
}

template <int KIND>
__global__ void __launch_bounds__(kPotThreads) k_potential(PotArgs a) {
  constexpr int NSUB = (KIND == POT_CONVENTIONAL) ? 20 : (KIND == POT_RS) ? 10 : 1;
  __shared__ float4 s_at[kChunk];
  __shared__ int s_start[kMaxSeg];
  __shared__ int s_pref[kMaxSeg + 1];
  __shared__ int s_warp[33];
  __shared__ int s_wcnt[kPotThreads / 32];

  // (coefficients are read through L1 per atom: a tile meets few elements, and
  // staging the whole 103-element table cost more than the plane's terms)

  int tx, ty;
  tile_pixel(threadIdx.x, tx, ty);
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int x = x0 + tx, y = y0 + ty;
  const bool inside = (x < a.nx) && (y < a.ny);

  // pixel position, rounded exactly as the host definition (no FMA)
  const float px = fadd_x(a.xoff, fmul_x((float)x, a.ps));
  const float py = fadd_x(a.yoff, fmul_x((float)y, a.ps));
  // Values are evaluated at the exact positions (the cut-off decisions use the
  // FP32 ones above, as the reference rounds them): the pixel's offset from
  // its rounded position, and per sub-plane the height's (zsub_lo).  Deep in a
  // thick slab or far across the grid the rounding is 1e-6..1e-5 A, which next
  // to a core moves V by ~1e-5 of its value -- the same in every repeat of a
  // crystal's slices, so it would add up over the stack.
  const float px_lo = (float)(((double)a.xoff + (double)x * (double)a.ps) - (double)px);
  const float py_lo = (float)(((double)a.yoff + (double)y * (double)a.ps) - (double)py);
  // the tile's pixel rectangle (the extreme pixel positions, as rounded above)
  const float tx_lo = fadd_x(a.xoff, fmul_x((float)x0, a.ps));
  const float tx_hi = fadd_x(a.xoff, fmul_x((float)(x0 + kTX - 1), a.ps));
  const float ty_lo = fadd_x(a.yoff, fmul_x((float)y0, a.ps));
  const float ty_hi = fadd_x(a.yoff, fmul_x((float)(y0 + kTY - 1), a.ps));

  // candidate bins of the tile (conservative: sqrt(5) + one bin)
  const float xlo = a.xoff + x0 * a.ps - 2.2361f, xhi = a.xoff + (x0 + kTX - 1) * a.ps + 2.2361f;
  const float ylo = a.yoff + y0 * a.ps - 2.2361f, yhi = a.yoff + (y0 + kTY - 1) * a.ps + 2.2361f;
  const int bxl = max((int)floorf(xlo / a.bw_x) - 1, 0);
  const int bxh = min((int)floorf(xhi / a.bw_x) + 1, kBins - 1);
  const int byl = max((int)floorf(ylo / a.bw_y) - 1, 0);
  const int byh = min((int)floorf(yhi / a.bw_y) + 1, kBins - 1);
  const int nyb = byh - byl + 1;

  float acc = 0.0f;
  if (bxl <= bxh && byl <= byh && a.kt <= a.kb) {
    const int kstep = max(kMaxSeg / nyb, 1);
    for (int kg = a.kt; kg <= a.kb; kg += kstep) {
      const int kend = min(kg + kstep - 1, a.kb);
      const int nseg = (kend - kg + 1) * nyb;
      // segment lengths and their exclusive prefix
      int len0 = 0, len1 = 0, st0 = 0, st1 = 0;
      // thread t holds the adjacent segments 2t and 2t + 1, so that the scan of
      // their summed lengths gives every segment its prefix in segment order
      const int s0 = 2 * (int)threadIdx.x, s1 = s0 + 1;
      if (s0 < nseg) {
        const int k = kg + s0 / nyb, j = byl + s0 % nyb;
        const int b = k * kBins2 + j * kBins;
        st0 = a.off[b + bxl];
        len0 = a.off[b + bxh + 1] - st0;
      }
      if (s1 < nseg) {
        const int k = kg + s1 / nyb, j = byl + s1 % nyb;
        const int b = k * kBins2 + j * kBins;
        st1 = a.off[b + bxl];
        len1 = a.off[b + bxh + 1] - st1;
      }
      int total;
      const int ex = block_exclusive_scan(len0 + len1, s_warp, &total);
      if (s0 < nseg) { s_start[s0] = st0; s_pref[s0] = ex; }
      if (s1 < nseg) { s_start[s1] = st1; s_pref[s1] = ex + len0; }
      if (threadIdx.x == 0) s_pref[nseg] = total;
      __syncthreads();

      for (int base = 0; base < total; base += kChunk) {
        const int nload = min(kChunk, total - base);
        // this chunk of candidates, kept when some pixel of the tile can take
        // a term from them: within sqrt(5) A of the tile's pixel rectangle
        // with the nearest sub-plane (margin far above FP32 rounding), and in
        // the slab for the projected form.  Kept atoms stay in order, so every
        // pixel sums the same terms in the same order.
        bool keep = false;
        float4 at = make_float4(0.f, 0.f, 0.f, 0.f);
        if (threadIdx.x < nload) {
          const int gidx = base + threadIdx.x;
          int lo = 0, hi = nseg - 1;  // last segment with s_pref <= gidx
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_pref[mid] <= gidx) lo = mid; else hi = mid - 1;
          }
          at = a.atoms[s_start[lo] + (gidx - s_pref[lo])];
          const float ddx = fmaxf(0.0f, fmaxf(tx_lo - at.x, at.x - tx_hi));
          const float ddy = fmaxf(0.0f, fmaxf(ty_lo - at.y, at.y - ty_hi));
          float reach = ddx * ddx + ddy * ddy;
          if constexpr (KIND == POT_PROJECTED) {
            keep = (int)floorf(fdiv_x(fsub_x(a.top, at.z), a.slab_dz)) == a.slab && reach < 5.0005f;
          } else {
            float dz2 = 1e30f;
#pragma unroll
            for (int m = 0; m < NSUB; ++m) {
              const float dz = a.zsub[m] - at.z;
              dz2 = fminf(dz2, dz * dz);
            }
            keep = reach + dz2 < 5.0005f;
          }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if ((threadIdx.x & 31) == 0) s_wcnt[threadIdx.x >> 5] = __popc(bal);
        __syncthreads();
        int pos = 0, cnt = 0;
#pragma unroll
        for (int w = 0; w < kPotThreads / 32; ++w) {
          if (w < (int)(threadIdx.x >> 5)) pos += s_wcnt[w];
          cnt += s_wcnt[w];
        }
        if (keep) s_at[pos + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = at;
        __syncthreads();
        for (int i = 0; i < cnt; ++i) {
          const float4 at = s_at[i];
          const float dx = fsub_x(px, at.x), dy = fsub_x(py, at.y);
          const float dxy = fadd_x(fmul_x(dx, dx), fmul_x(dy, dy));
          const float dxv = dx + px_lo, dyv = dy + py_lo;
          const float dxyv = fmaf(dxv, dxv, dyv * dyv);
          if (!(dxy < 5.0f)) continue;
          const float* c = a.coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
          if constexpr (KIND == POT_PROJECTED) {
            const int slab = (int)floorf(fdiv_x(fsub_x(a.top, at.z), a.slab_dz));
            if (slab == a.slab) acc += vzatom2_f(c, dxy);
          } else {
#pragma unroll
            for (int m = 0; m < NSUB; ++m) {
              const float dz = fsub_x(a.zsub[m], at.z);
              const float r2 = fadd_x(dxy, fmul_x(dz, dz));
              if (r2 < 5.0f) acc += a.wsub * vatom_f(c, r2);
            }
          }
        }
        __syncthreads();
      }
    }
  }
  if (inside) a.V[(long long)y * a.nx + x] = acc;
}

// exp2 on the MUFU (PTX ex2.approx.ftz.f32; relative error about 2^-22).
__device__ __forceinline__ float ex2_fast(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ f2p ex2_pair(f2p a) {
  float lo, hi;
  up2(a, lo, hi);
  return pk2(ex2_fast(lo), ex2_fast(hi));
}

// Conventional potential (binnedAtomPKernel3 semantics) with per-atom work
// hoisted out of the pixel loop.  For each staged atom the 20 sub-plane offsets
// dz_m^2 (rounded exactly as in the cut-off test) and the Gaussian factors
// exp(-pi^2 dz_m^2 / d_i) are computed once per CTA; a pixel then needs
// exp(-pi^2 rho^2 / d_i) once per atom and, per sub-plane inside the cut-off,
// one rsqrt and three exp2 for the Lorentzian terms.  Inside r < 0.25 A (the
// clamp) the full vatom is evaluated.  Cut-offs stay non-contracted FP32.
// Staging drops the candidates that no pixel of the tile can reach (kept
// atoms keep their order, so every pixel sums the same terms in the same
// order), and each warp (an 8 x 4 pixel patch) walks only the sub-planes that
// its nearest pixel can reach.
constexpr int kConvChunk = 64;

// Tile shapes of the conventional kernel (TX x TY pixels, 256 threads, warps
// on 8 x 4 patches): 32 x 8, 16 x 16, 64 x 4 -- tuned per specimen and grid by
// the engine (a squarer tile stages fewer candidate atoms per pixel, a wider
// one fewer bins per row of CTAs).
template <int TX, int TY>
__device__ __forceinline__ void tile_pixel_t(int tid, int& tx, int& ty) {
  constexpr int PX = TX / 8;  // patches across
  const int w = tid >> 5, l = tid & 31;
  tx = (w % PX) * 8 + (l & 7);
  ty = (w / PX) * 4 + (l >> 3);
}

template <int TX, int TY>
__global__ void __launch_bounds__(kPotThreads) k_potential_conv(PotArgs a) {
  static_assert(TX * TY == kPotThreads && TX % 8 == 0 && TY % 4 == 0, "tile of 8 x 4 warp patches");
  __shared__ float4 s_at[kConvChunk];
  __shared__ __align__(8) float s_dz2[kConvChunk][20];
  __shared__ __align__(8) float s_dz2v[kConvChunk][20];
  __shared__ __align__(8) float s_g[kConvChunk][3][20];
  __shared__ int s_mlo[kConvChunk], s_mhi[kConvChunk];
  __shared__ float s_dzmin[kConvChunk];
  __shared__ int s_wcnt[kPotThreads / 32];
  __shared__ float s_coef[103 * kCoefPerZ];
  __shared__ int s_start[kMaxSeg];
  __shared__ int s_pref[kMaxSeg + 1];
  __shared__ int s_warp[33];

  for (int i = threadIdx.x; i < 103 * kCoefPerZ; i += kPotThreads) s_coef[i] = a.coef[i];

  int tx, ty;
  tile_pixel_t<TX, TY>(threadIdx.x, tx, ty);
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool inside = (x < a.nx) && (y < a.ny);
  const float px = fadd_x(a.xoff, fmul_x((float)x, a.ps));
  const float py = fadd_x(a.yoff, fmul_x((float)y, a.ps));
  // Values are evaluated at the exact positions (the cut-off decisions use the
  // FP32 ones above, as the reference rounds them): the pixel's offset from
  // its rounded position, and per sub-plane the height's (zsub_lo).  Deep in a
  // thick slab or far across the grid the rounding is 1e-6..1e-5 A, which next
  // to a core moves V by ~1e-5 of its value -- the same in every repeat of a
  // crystal's slices, so it would add up over the stack.
  const float px_lo = (float)(((double)a.xoff + (double)x * (double)a.ps) - (double)px);
  const float py_lo = (float)(((double)a.yoff + (double)y * (double)a.ps) - (double)py);
  // the tile's pixel rectangle (the extreme pixel positions, as rounded above)
  const float tx_lo = fadd_x(a.xoff, fmul_x((float)x0, a.ps));
  const float tx_hi = fadd_x(a.xoff, fmul_x((float)(x0 + TX - 1), a.ps));
  const float ty_lo = fadd_x(a.yoff, fmul_x((float)y0, a.ps));
  const float ty_hi = fadd_x(a.yoff, fmul_x((float)(y0 + TY - 1), a.ps));
  // sub-plane m sits at zsub[0] - m h: its index from a height, for the
  // per-warp sub-plane window below
  const float zs0 = a.zsub[0], inv_h = 19.0f / (a.zsub[0] - a.zsub[19]);
  const float xlo = a.xoff + x0 * a.ps - 2.2361f, xhi = a.xoff + (x0 + TX - 1) * a.ps + 2.2361f;
  const float ylo = a.yoff + y0 * a.ps - 2.2361f, yhi = a.yoff + (y0 + TY - 1) * a.ps + 2.2361f;
  const int bxl = max((int)floorf(xlo / a.bw_x) - 1, 0);
  const int bxh = min((int)floorf(xhi / a.bw_x) + 1, kBins - 1);
  const int byl = max((int)floorf(ylo / a.bw_y) - 1, 0);
  const int byh = min((int)floorf(yhi / a.bw_y) + 1, kBins - 1);
  const int nyb = byh - byl + 1;

  float acc = 0.0f;
  if (bxl <= bxh && byl <= byh && a.kt <= a.kb) {
    const int kstep = max(kMaxSeg / nyb, 1);
    for (int kg = a.kt; kg <= a.kb; kg += kstep) {
      const int kend = min(kg + kstep - 1, a.kb);
      const int nseg = (kend - kg + 1) * nyb;
      int len0 = 0, len1 = 0, st0 = 0, st1 = 0;
      // thread t holds the adjacent segments 2t and 2t + 1, so that the scan of
      // their summed lengths gives every segment its prefix in segment order
      const int s0 = 2 * (int)threadIdx.x, s1 = s0 + 1;
      if (s0 < nseg) {
        const int b = (kg + s0 / nyb) * kBins2 + (byl + s0 % nyb) * kBins;
        st0 = a.off[b + bxl];
        len0 = a.off[b + bxh + 1] - st0;
      }
      if (s1 < nseg) {
        const int b = (kg + s1 / nyb) * kBins2 + (byl + s1 % nyb) * kBins;
        st1 = a.off[b + bxl];
        len1 = a.off[b + bxh + 1] - st1;
      }
      int total;
      const int ex = block_exclusive_scan(len0 + len1, s_warp, &total);
      if (s0 < nseg) { s_start[s0] = st0; s_pref[s0] = ex; }
      if (s1 < nseg) { s_start[s1] = st1; s_pref[s1] = ex + len0; }
      if (threadIdx.x == 0) s_pref[nseg] = total;
      __syncthreads();

      for (int base = 0; base < total; base += kConvChunk) {
        const int nload = min(kConvChunk, total - base);
        // this chunk of candidates, kept when some sub-plane can pass the
        // cut-off (dz_m^2 < 5) and the atom lies within sqrt(5) A of the tile's
        // pixel rectangle (with a margin far above FP32 rounding, so that every
        // dropped atom fails r^2 < 5 at every pixel); kept atoms stay in order
        bool keep = false;
        float4 at = make_float4(0.f, 0.f, 0.f, 0.f);
        int amlo = 20, amhi = -1;
        float dmin = 1e30f;
        if (threadIdx.x < nload) {
          const int gidx = base + threadIdx.x;
          int lo = 0, hi = nseg - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_pref[mid] <= gidx) lo = mid; else hi = mid - 1;
          }
          at = a.atoms[s_start[lo] + (gidx - s_pref[lo])];
          // sub-planes that can pass the cut-off for some pixel (dz_m^2 < 5: an
          // interval of m, since the non-contracted dz and dz^2 are monotone in
          // the plane height) and the smallest dz_m^2 (the clamp test below)
          for (int m = 0; m < 20; ++m) {
            const float dz = fsub_x(a.zsub[m], at.z);
            const float dz2 = fmul_x(dz, dz);
            if (dz2 < 5.0f) {
              amlo = min(amlo, m);
              amhi = m;
            }
            dmin = fminf(dmin, dz2);
          }
          const float ddx = fmaxf(0.0f, fmaxf(tx_lo - at.x, at.x - tx_hi));
          const float ddy = fmaxf(0.0f, fmaxf(ty_lo - at.y, at.y - ty_hi));
          keep = amlo <= amhi && ddx * ddx + ddy * ddy < 5.0005f;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if ((threadIdx.x & 31) == 0) s_wcnt[threadIdx.x >> 5] = __popc(bal);
        __syncthreads();
        int pos = 0, cnt = 0;
        for (int w = 0; w < kConvChunk / 32; ++w) {
          if (w < (int)(threadIdx.x >> 5)) pos += s_wcnt[w];
          cnt += s_wcnt[w];
        }
        if (keep) {
          pos += __popc(bal & ((1u << (threadIdx.x & 31)) - 1u));
          s_at[pos] = at;
          s_mlo[pos] = amlo;
          s_mhi[pos] = amhi;
          s_dzmin[pos] = dmin;
        }
        __syncthreads();
        // per (atom, sub-plane): dz^2 as the cut-off rounds it, the exact
        // height's dz^2 for the values, Gaussian factors
        for (int q = threadIdx.x; q < cnt * 20; q += kPotThreads) {
          const int i = q / 20, m = q % 20;
          const float4 at = s_at[i];
          const float dz = fsub_x(a.zsub[m], at.z);
          const float dz2 = fmul_x(dz, dz);
          s_dz2[i][m] = dz2;
          const float dzv = dz + a.zsub_lo[m];
          const float dz2v = dzv * dzv;
          s_dz2v[i][m] = dz2v;
          const float* c = s_coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
          s_g[i][0][m] = ex2_fast(-c[9] * dz2v);
          s_g[i][1][m] = ex2_fast(-c[10] * dz2v);
          s_g[i][2][m] = ex2_fast(-c[11] * dz2v);
        }
        __syncthreads();
        for (int i = 0; i < cnt; ++i) {
          const float4 at = s_at[i];
          const float dx = fsub_x(px, at.x), dy = fsub_x(py, at.y);
          const float dxy = fadd_x(fmul_x(dx, dx), fmul_x(dy, dy));
          const float dxv = dx + px_lo, dyv = dy + py_lo;
          const float dxyv = fmaf(dxv, dxv, dyv * dyv);
          // the warp's nearest pixel bounds the sub-planes any lane can use:
          // |zsub[m] - z| < sqrt(5 - min dxy), widened by one plane each side
          // (dxy >= 0, so its bits order as the values do)
          const float wmin = __int_as_float(__reduce_min_sync(0xffffffffu, __float_as_int(dxy)));
          if (!(wmin < 5.0f)) continue;
          if (!(dxy < 5.0f)) continue;
          const float w5 = 5.0f - wmin, zr = w5 * rsqrtf(w5);  // (approximate: one plane of margin)
          const int mlo = max(s_mlo[i], __float2int_rd((zs0 - at.z - zr) * inv_h) - 1);
          const int mhi = min(s_mhi[i], __float2int_ru((zs0 - at.z + zr) * inv_h) + 1);
          const float* c = s_coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
          const float g0 = c[6] * ex2_fast(-c[9] * dxyv), g1 = c[7] * ex2_fast(-c[10] * dxyv),
                      g2 = c[8] * ex2_fast(-c[11] * dxyv);
          // (a margin over 0.0625: the clamp is decided on the exact-position
          // value r^2 in the sub-plane loop below)
          if (!(fadd_x(dxy, s_dzmin[i]) < 0.0627f)) {
            // No sub-plane reaches the 0.25 A clamp for this pixel: sub-planes in
            // pairs (m, m+1) on the packed FP32x2 pipe.  add.rn.f32x2 rounds each
            // lane as fadd_x does, so the r^2 < 5 decisions are unchanged; sub-
            // planes outside [mlo, mhi] have dz^2 >= 5 and fail the test.
            const f2p d2 = pk2(dxy, dxy), d2v = pk2(dxyv, dxyv);
            const f2p c0 = pk2(c[0], c[0]), c1 = pk2(c[1], c[1]), c2 = pk2(c[2], c[2]);
            const f2p n3 = pk2(-c[3], -c[3]), n4 = pk2(-c[4], -c[4]), n5 = pk2(-c[5], -c[5]);
            const f2p q0 = pk2(g0, g0), q1 = pk2(g1, g1), q2 = pk2(g2, g2);
            f2p acc2 = pk2(0.0f, 0.0f);
            // one pair (m, m+1) into acc; pairs with no sub-plane inside the
            // cut-off for this pixel add nothing
            auto pair = [&](int m, f2p& acc) {
              const f2p r2 = add2(d2, *reinterpret_cast<const f2p*>(&s_dz2[i][m]));
              float ra, rb;
              up2(r2, ra, rb);
              const bool ka = ra < 5.0f, kb = rb < 5.0f;
              if (!(ka || kb)) return;
              const f2p r2v = add2(d2v, *reinterpret_cast<const f2p*>(&s_dz2v[i][m]));
              float va2, vb2;
              up2(r2v, va2, vb2);
              const f2p ri = pk2(rsqrtf(va2), rsqrtf(vb2));
              const f2p r = mul2(r2v, ri);
              f2p L = mul2(c0, ex2_pair(mul2(n3, r)));
              L = fma2(c1, ex2_pair(mul2(n4, r)), L);
              L = fma2(c2, ex2_pair(mul2(n5, r)), L);
              f2p G = mul2(q0, *reinterpret_cast<const f2p*>(&s_g[i][0][m]));
              G = fma2(q1, *reinterpret_cast<const f2p*>(&s_g[i][1][m]), G);
              G = fma2(q2, *reinterpret_cast<const f2p*>(&s_g[i][2][m]), G);
              float va, vb;
              up2(fma2(L, ri, G), va, vb);
              acc = fma2(pk2(ka ? a.wsub : 0.0f, kb ? a.wsub : 0.0f), pk2(va, vb), acc);
            };
            // two pairs per step into two sums: independent chains for the
            // scheduler (the even pair's sum, then the odd pair's, per lane)
            f2p acc2b = pk2(0.0f, 0.0f);
            int m = mlo & ~1;
            for (; m + 2 <= mhi; m += 4) {
              pair(m, acc2);
              pair(m + 2, acc2b);
            }
            if (m <= mhi) pair(m, acc2);
            acc2 = add2(acc2, acc2b);
            float ea, eb;
            up2(acc2, ea, eb);
            acc += ea + eb;
          } else {
            for (int m = mlo; m <= mhi; ++m) {
              const float r2 = fadd_x(dxy, s_dz2[i][m]);
              if (!(r2 < 5.0f)) continue;
              const float r2v = dxyv + s_dz2v[i][m];
              float v;
              if (r2v < 0.0625f) {
                v = vatom_f(c, r2v);  // inside the 0.25 A clamp
              } else {
                const float ri = rsqrtf(r2v), r = r2v * ri;
                const float L =
                    c[0] * ex2_fast(-c[3] * r) + c[1] * ex2_fast(-c[4] * r) + c[2] * ex2_fast(-c[5] * r);
                const float G = g0 * s_g[i][0][m] + g1 * s_g[i][1][m] + g2 * s_g[i][2][m];
                v = L * ri + G;
              }
              acc += a.wsub * v;
            }
          }
        }
        __syncthreads();
      }
    }
  }
  if (inside) a.V[(long long)y * a.nx + x] = acc;
}

// ---------------------------------------------------------------------------
// Separable conventional potential.  Each Gaussian of an element's expansion
// v(r) ~= sum_j w_j exp(-alpha_j r^2) factorises over r^2 = rho^2 + dz_m^2, so
// an atom's sub-plane sum at a pixel is
//   sum_{m valid} wsub v(rho^2 + dz_m^2) ~= sum_j exp(-alpha_j rho^2) T_K[j],
//   T_K[j] = wsub sum_{k < K} w_j exp(-alpha_j dz_(k)^2),
// where the valid sub-planes (r^2 < 5 in the reference's FP32 rounding) are the
// K with the smallest dz^2: for a fixed pixel the decision is monotone in dz^2.
// k_atom_tables forms the T rows once per atom and slice; the pixel kernel
// finds K with a five-step search over the atom's ascending thresholds (the
// reference's own FP32 test, sub-plane by sub-plane) and takes kGaussJ
// exponentials per (pixel, atom) instead of four per (pixel, atom, sub-plane).
// Inside the 0.25 A clamp, where v is constant and the expansion does not
// hold, the pixel sums vatom over its K sub-planes directly.
// ---------------------------------------------------------------------------
constexpr int kTabAtoms = 16;  // atoms per CTA of the table kernel, 16 threads each

// The cut-off test fadd(dxy, q) < 5 (round to nearest even) holds exactly when
// the real sum dxy + q < 5 - 2^-22 (the midpoint below 5 rounds up to the even
// 5); for a float dxy that is dxy < t with t the FP32 value of 5 - 2^-22 - q
// rounded up (the difference is exact in FP64 wherever it can decide the
// rounding).  So one comparison per search step decides as the reference does.
__device__ __forceinline__ float cutoff_threshold(float q) {
  return __double2float_ru(4.999999761581421 - (double)q);
}

__global__ void __launch_bounds__(256) k_atom_tables(PotArgs a) {
  __shared__ float s_d2[kTabAtoms][20];
  __shared__ float s_qv[kTabAtoms][20];
  __shared__ float s_e[kTabAtoms][20][kGaussJ];
  __shared__ int s_n[kTabAtoms];
  if (a.kt > a.kb || a.kt < 0 || a.kb >= a.nz) return;  // (no z-bin in the window)
  // (this instance's index and tables; a itself stays in parameter space,
  // where a.zsub is read)
  const float4* atoms = a.atoms + blockIdx.y * a.b_atoms;
  const int* off = a.off + blockIdx.y * a.b_off;
  float* tabs = a.tab + blockIdx.y * a.b_tab;
  const int a0 = off[a.kt * kBins2], na = off[(a.kb + 1) * kBins2] - a0;
  const int la = threadIdx.x >> 4, j = threadIdx.x & 15;
  for (int base = blockIdx.x * kTabAtoms; base < na; base += gridDim.x * kTabAtoms) {
    const bool valid = base + la < na;
    float* tab = tabs + (size_t)(base + la) * kTabStride;
    float4 at = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      at = atoms[a0 + base + la];
      // dz_m^2 as the cut-off rounds it (16 lanes, two planes for the first 4)
      for (int m = j; m < 20; m += 16) {
        const float dz = fsub_x(a.zsub[m], at.z);
        s_d2[la][m] = fmul_x(dz, dz);
      }
    }
    __syncthreads();
    const float* g = a.gauss + (valid ? __float_as_int(at.w) - 1 : 0) * 2 * kGaussJ;
    if (valid) {
      // each lane places its sub-planes by rank (ascending dz^2, ties by m);
      // the planes with dz^2 < 5 are the first n of that order
      int cnt = 0;
      for (int m = 0; m < 20; ++m) cnt += s_d2[la][m] < 5.0f;
      if (j == 0) s_n[la] = cnt;
      for (int m = j; m < 20; m += 16) {
        const float d = s_d2[la][m];
        if (!(d < 5.0f)) continue;
        int r = 0;
        for (int k = 0; k < 20; ++k) {
          const float e = s_d2[la][k];
          r += (e < d) || (e == d && k < m);
        }
        const float dzv = fsub_x(a.zsub[m], at.z) + a.zsub_lo[m];
        const float qv = dzv * dzv;
        tab[kTabQ + r] = cutoff_threshold(d);
        tab[kTabQV + r] = qv;
        s_qv[la][r] = qv;
      }
      for (int k = cnt + j; k < 32; k += 16) tab[kTabQ + k] = -1e30f;
    }
    __syncthreads();
    if (valid) {
      // w_j exp(-alpha_j dzv_k^2) for every (sub-plane, Gaussian), independent
      const int nk = s_n[la];
      for (int q = j; q < nk * kGaussJ; q += 16) {
        const int k = q / kGaussJ, jj = q - k * kGaussJ;
        s_e[la][k][jj] = g[kGaussJ + jj] * exp2f(-g[jj] * s_qv[la][k]);
      }
    }
    __syncthreads();
    if (valid && j < kGaussJ) {
      // running sums over the sub-planes in ascending dz^2 (FP64, rounded once)
      const int nk = s_n[la];
      double sum = 0.0;
      for (int k = 0; k < nk; ++k) {
        sum += (double)s_e[la][k][j];
        tab[kTabT + k * kGaussJ + j] = (float)((double)a.wsub * sum);
      }
    }
    __syncthreads();
  }
}

// Each thread sums RY pixels of one column (rows y, y + 4, ...): a warp covers
// an 8 x 4RY patch, and the per-atom work of a warp (staged atom, element,
// table row base, loop) is shared by RY pixels per lane.  Each warp walks
// only the staged atoms that can reach its own patch.
template <int TX, int TY, int RY>
__global__ void __launch_bounds__(kPotThreads, RY >= 4 ? 5 : 6) k_potential_sep(PotArgs a) {
  static_assert(TX * TY == kPotThreads * RY && TX % 8 == 0 && TY % (4 * RY) == 0, "tile of 8 x 4RY warp patches");
  __shared__ float4 s_at[kConvChunk];
  __shared__ __align__(16) float s_t[kConvChunk][32];
  __shared__ __align__(16) float s_al[kConvChunk][kGaussJ];
  __shared__ int s_l[kConvChunk];
  __shared__ int s_wcnt[kPotThreads / 32];
  __shared__ int s_start[kMaxSeg];
  __shared__ int s_pref[kMaxSeg + 1];
  __shared__ int s_warp[33];

  constexpr int PX = TX / 8;  // patches across
  // (this instance's index, tables and output)
  const float4* atoms = a.atoms + blockIdx.z * a.b_atoms;
  const int* off = a.off + blockIdx.z * a.b_off;
  const float* tabs = a.tab + blockIdx.z * a.b_tab;
  float* V = a.V + blockIdx.z * a.b_V;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int wx0 = x0 + (w % PX) * 8, wy0 = y0 + (w / PX) * 4 * RY;  // this warp's patch
  const int x = wx0 + (lane & 7);
  const float px = fadd_x(a.xoff, fmul_x((float)x, a.ps));
  // values at the exact positions, decisions at the reference's FP32 ones (as
  // in k_potential_conv)
  const float px_lo = (float)(((double)a.xoff + (double)x * (double)a.ps) - (double)px);
  float py[RY], py_lo[RY], acc[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    const int y = wy0 + (lane >> 3) + 4 * r;
    py[r] = fadd_x(a.yoff, fmul_x((float)y, a.ps));
    py_lo[r] = (float)(((double)a.yoff + (double)y * (double)a.ps) - (double)py[r]);
    acc[r] = 0.0f;
  }
  const float tx_lo = fadd_x(a.xoff, fmul_x((float)x0, a.ps));
  const float tx_hi = fadd_x(a.xoff, fmul_x((float)(x0 + TX - 1), a.ps));
  const float ty_lo = fadd_x(a.yoff, fmul_x((float)y0, a.ps));
  const float ty_hi = fadd_x(a.yoff, fmul_x((float)(y0 + TY - 1), a.ps));
  const float wx_lo = fadd_x(a.xoff, fmul_x((float)wx0, a.ps)), wx_hi = fadd_x(a.xoff, fmul_x((float)(wx0 + 7), a.ps));
  const float wy_lo = fadd_x(a.yoff, fmul_x((float)wy0, a.ps));
  const float wy_hi = fadd_x(a.yoff, fmul_x((float)(wy0 + 4 * RY - 1), a.ps));
  const float xlo = a.xoff + x0 * a.ps - 2.2361f, xhi = a.xoff + (x0 + TX - 1) * a.ps + 2.2361f;
  const float ylo = a.yoff + y0 * a.ps - 2.2361f, yhi = a.yoff + (y0 + TY - 1) * a.ps + 2.2361f;
  const int bxl = max((int)floorf(xlo / a.bw_x) - 1, 0);
  const int bxh = min((int)floorf(xhi / a.bw_x) + 1, kBins - 1);
  const int byl = max((int)floorf(ylo / a.bw_y) - 1, 0);
  const int byh = min((int)floorf(yhi / a.bw_y) + 1, kBins - 1);
  const int nyb = byh - byl + 1;
  const bool window = a.kt <= a.kb && a.kt >= 0 && a.kb < a.nz;
  const int a0 = window ? off[a.kt * kBins2] : 0;

  if (bxl <= bxh && byl <= byh && window) {
    const int kstep = max(kMaxSeg / nyb, 1);
    for (int kg = a.kt; kg <= a.kb; kg += kstep) {
      const int kend = min(kg + kstep - 1, a.kb);
      const int nseg = (kend - kg + 1) * nyb;
      int len0 = 0, len1 = 0, st0 = 0, st1 = 0;
      // thread t holds the adjacent segments 2t and 2t + 1, so that the scan of
      // their summed lengths gives every segment its prefix in segment order
      const int s0 = 2 * (int)threadIdx.x, s1 = s0 + 1;
      if (s0 < nseg) {
        const int b = (kg + s0 / nyb) * kBins2 + (byl + s0 % nyb) * kBins;
        st0 = off[b + bxl];
        len0 = off[b + bxh + 1] - st0;
      }
      if (s1 < nseg) {
        const int b = (kg + s1 / nyb) * kBins2 + (byl + s1 % nyb) * kBins;
        st1 = off[b + bxl];
        len1 = off[b + bxh + 1] - st1;
      }
      int total;
      const int ex = block_exclusive_scan(len0 + len1, s_warp, &total);
      if (s0 < nseg) { s_start[s0] = st0; s_pref[s0] = ex; }
      if (s1 < nseg) { s_start[s1] = st1; s_pref[s1] = ex + len0; }
      if (threadIdx.x == 0) s_pref[nseg] = total;
      __syncthreads();

      for (int base = 0; base < total; base += kConvChunk) {
        const int nload = min(kConvChunk, total - base);
        // candidates kept when the nearest sub-plane can pass the cut-off
        // within sqrt(5) A of the tile's pixel rectangle (margin far above
        // FP32 rounding); kept atoms stay in CSR order
        bool keep = false;
        float4 at = make_float4(0.f, 0.f, 0.f, 0.f);
        int li = 0;
        if (threadIdx.x < nload) {
          const int gidx = base + threadIdx.x;
          int lo = 0, hi = nseg - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_pref[mid] <= gidx) lo = mid; else hi = mid - 1;
          }
          const int l = s_start[lo] + (gidx - s_pref[lo]);
          at = atoms[l];
          li = l - a0;
          const float t0 = tabs[(size_t)li * kTabStride + kTabQ];
          const float ddx = fmaxf(0.0f, fmaxf(tx_lo - at.x, at.x - tx_hi));
          const float ddy = fmaxf(0.0f, fmaxf(ty_lo - at.y, at.y - ty_hi));
          keep = ddx * ddx + ddy * ddy < t0 + 0.0005f;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wcnt[w] = __popc(bal);
        __syncthreads();
        int pos = 0, cnt = 0;
        for (int ww = 0; ww < kConvChunk / 32; ++ww) {
          if (ww < w) pos += s_wcnt[ww];
          cnt += s_wcnt[ww];
        }
        if (keep) {
          pos += __popc(bal & ((1u << lane) - 1u));
          s_at[pos] = at;
          s_l[pos] = li;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < cnt * 32; q += kPotThreads)
          s_t[q >> 5][q & 31] = tabs[(size_t)s_l[q >> 5] * kTabStride + kTabQ + (q & 31)];
        for (int q = threadIdx.x; q < cnt * kGaussJ; q += kPotThreads) {
          const int i = q / kGaussJ, jj = q - i * kGaussJ;
          s_al[i][jj] = -a.gauss[(__float_as_int(s_at[i].w) - 1) * 2 * kGaussJ + jj];
        }
        __syncthreads();
        // each warp walks the staged atoms that can reach its own patch
        for (int c0 = 0; c0 < cnt; c0 += 32) {
          bool reach = false;
          if (c0 + lane < cnt) {
            const float4 ar = s_at[c0 + lane];
            const float ddx = fmaxf(0.0f, fmaxf(wx_lo - ar.x, ar.x - wx_hi));
            const float ddy = fmaxf(0.0f, fmaxf(wy_lo - ar.y, ar.y - wy_hi));
            reach = ddx * ddx + ddy * ddy < s_t[c0 + lane][0] + 0.0005f;
          }
          unsigned mask = __ballot_sync(0xffffffffu, reach);
          while (mask) {
            const int i = c0 + __ffs(mask) - 1;
            mask &= mask - 1u;
            const float4 at = s_at[i];
            const float* t = s_t[i];
            const float* tab = tabs + (size_t)s_l[i] * kTabStride;
            const float4* A = reinterpret_cast<const float4*>(&s_al[i][0]);
            const float dx = fsub_x(px, at.x);
            const float dx2 = fmul_x(dx, dx);
            const float dxv = dx + px_lo;
#pragma unroll
            for (int r = 0; r < RY; ++r) {
              const float dy = fsub_x(py[r], at.y);
              const float dxy = fadd_x(dx2, fmul_x(dy, dy));
              // K = the sub-planes with r^2 = dxy + dz^2 < 5 (the reference's test)
              int K = 0;
#pragma unroll
              for (int st = 16; st >= 1; st >>= 1)
                if (dxy < t[K + st - 1]) K += st;
              if (K == 0) continue;
              const float dyv = dy + py_lo[r];
              const float dxyv = fmaf(dxv, dxv, dyv * dyv);
              if (dxy < t[0] - 4.9373f) {
                // a sub-plane can reach the 0.25 A clamp (dxy + dz^2 < 0.0627;
                // the clamp itself is decided on the exact r^2 inside vatom_f):
                // the direct sum
                const float* c = a.coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
                float v = 0.0f;
                for (int k = 0; k < K; ++k) v += vatom_f(c, dxyv + __ldg(tab + kTabQV + k));
                acc[r] += a.wsub * v;
              } else {
                // sum_j exp(-alpha_j rho^2) T_K[j]: per pair of Gaussians one
                // packed multiply, two ex2, one packed fused multiply-add
                const ulonglong2* T = reinterpret_cast<const ulonglong2*>(tab + kTabT + (K - 1) * kGaussJ);
                const ulonglong2* A2 = reinterpret_cast<const ulonglong2*>(A);
                const f2p rr = pk2(dxyv, dxyv);
                f2p s2 = pk2(0.0f, 0.0f);
#pragma unroll
                for (int g = 0; g < kGaussJ / 4; ++g) {
                  const ulonglong2 al = A2[g];
                  const ulonglong2 tt = __ldg(T + g);
                  s2 = fma2(ex2_pair(mul2(al.x, rr)), tt.x, s2);
                  s2 = fma2(ex2_pair(mul2(al.y, rr)), tt.y, s2);
                }
                float e0, e1;
                up2(s2, e0, e1);
                acc[r] += e0 + e1;
              }
            }
          }
        }
        // (no barrier here: the next round writes the staged arrays only after
        // its first barrier, which every warp reaches after this loop)
      }
    }
  }
  if (x < a.nx) {
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int y = wy0 + (lane >> 3) + 4 * r;
      if (y < a.ny) V[(long long)y * a.nx + x] = acc[r];
    }
  }
}

// Adjoint of k_potential_conv with respect to the atoms' x and y.  For slice
// potential V(p) = sum_atoms sum_m wsub v(r^2), r^2 = (p - X)^2 + dz_m^2, and
// the slice's dL/dV field G:
//   dL/dX = sum_p G(p) wsub sum_m v'(r^2) (-2 (px - X)),  likewise for Y,
// over exactly the (pixel, atom, sub-plane) triples the forward kept (the same
// non-contracted FP32 cut-off tests on the same stored positions; the forward
// visits every atom of the z-window within sqrt(5) A of a pixel).  Inside the
// 0.25 A clamp v is constant and contributes nothing.  blockIdx.x picks the
// atom of the window, blockIdx.y one of gridDim.y interleaved row sets of its
// +-2.3 A pixel square (so that a window of few atoms still fills the GPU);
// each CTA's sums (FP64 across threads) are added atomically to the atom's
// entry in input order.
//   v'(r^2) = sum_i c_i e^{-b_i r} (-b_i r - 1) / (2 r^3)
//             - ln2 sum_k c9_k c6_k 2^{-c9_k r^2}     (c layout of vatom_f).
__global__ void __launch_bounds__(kPotThreads) k_potential_conv_adjoint(PotArgs a, const float* __restrict__ G,
                                                                        const int* __restrict__ perm, int a0,
                                                                        double* __restrict__ dxy) {
  __shared__ float s_dz2[20];
  __shared__ float s_gz[3][20];
  __shared__ double s_red[2][kPotThreads / 32];
  constexpr float kLn2 = 0.6931471805599453f;
  const int l = a0 + blockIdx.x;
  const float4 at = a.atoms[l];
  const float* c = a.coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
  if (threadIdx.x < 20) {
    const int m = threadIdx.x;
    const float dz = fsub_x(a.zsub[m], at.z);
    const float dz2 = fmul_x(dz, dz);
    s_dz2[m] = dz2;
    s_gz[0][m] = ex2_fast(-c[9] * dz2);
    s_gz[1][m] = ex2_fast(-c[10] * dz2);
    s_gz[2][m] = ex2_fast(-c[11] * dz2);
  }
  __syncthreads();
  const float b0 = c[3] * kLn2, b1 = c[4] * kLn2, b2 = c[5] * kLn2;
  const float h0 = -kLn2 * c[9] * c[6], h1 = -kLn2 * c[10] * c[7], h2 = -kLn2 * c[11] * c[8];
  const int xl = max((int)floorf((at.x - 2.3f - a.xoff) / a.ps), 0);
  const int xh = min((int)ceilf((at.x + 2.3f - a.xoff) / a.ps), a.nx - 1);
  const int yl = max((int)floorf((at.y - 2.3f - a.yoff) / a.ps), 0);
  const int yh = min((int)ceilf((at.y + 2.3f - a.yoff) / a.ps), a.ny - 1);
  const int wx = xh - xl + 1, wy = yh - yl + 1;
  const int ns = gridDim.y, js = blockIdx.y;
  float gx = 0.0f, gy = 0.0f;
  if (wx > 0 && wy > js) {
    const int npx = wx * ((wy - js + ns - 1) / ns);
    for (int w = threadIdx.x; w < npx; w += kPotThreads) {
      const int x = xl + w % wx, y = yl + js + (w / wx) * ns;
      const float px = fadd_x(a.xoff, fmul_x((float)x, a.ps));
      const float py = fadd_x(a.yoff, fmul_x((float)y, a.ps));
      const float dx = fsub_x(px, at.x), dy = fsub_x(py, at.y);
      const float dxy = fadd_x(fmul_x(dx, dx), fmul_x(dy, dy));
      if (!(dxy < 5.0f)) continue;
      const float gp = G[(long long)y * a.nx + x];
      const float g0 = h0 * ex2_fast(-c[9] * dxy), g1 = h1 * ex2_fast(-c[10] * dxy), g2 = h2 * ex2_fast(-c[11] * dxy);
      float D = 0.0f;
#pragma unroll 4
      for (int m = 0; m < 20; ++m) {
        const float r2 = fadd_x(dxy, s_dz2[m]);
        if (!(r2 < 5.0f) || r2 < 0.0625f) continue;
        const float ri = rsqrtf(r2), r = r2 * ri;
        const float L = c[0] * ex2_fast(-c[3] * r) * fmaf(-b0, r, -1.0f) +
                        c[1] * ex2_fast(-c[4] * r) * fmaf(-b1, r, -1.0f) +
                        c[2] * ex2_fast(-c[5] * r) * fmaf(-b2, r, -1.0f);
        D += 0.5f * L * ri * ri * ri + g0 * s_gz[0][m] + g1 * s_gz[1][m] + g2 * s_gz[2][m];
      }
      gx += gp * D * dx;
      gy += gp * D * dy;
    }
  }
  double sx = gx, sy = gy;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sy += __shfl_down_sync(0xffffffffu, sy, o);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_red[0][warp] = sx;
    s_red[1][warp] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tx = 0.0, ty = 0.0;
    for (int k = 0; k < kPotThreads / 32; ++k) {
      tx += s_red[0][k];
      ty += s_red[1][k];
    }
    const double f = -2.0 * (double)a.wsub;
    const int i = perm[l];
    atomicAdd(dxy + 2 * i, f * tx);
    atomicAdd(dxy + 2 * i + 1, f * ty);
  }
}

// v'(r^2) of vatom_f, as k_potential_conv_adjoint evaluates it term by term
// (zero inside the 0.25 A clamp, where v is constant).
__device__ __forceinline__ float vatom_deriv_f(const float* __restrict__ c, float r2) {
  if (r2 < 0.0625f) return 0.0f;
  constexpr float kLn2 = 0.6931471805599453f;
  const float ri = rsqrtf(r2), r = r2 * ri;
  const float L = c[0] * ex2_fast(-c[3] * r) * fmaf(-c[3] * kLn2, r, -1.0f) +
                  c[1] * ex2_fast(-c[4] * r) * fmaf(-c[4] * kLn2, r, -1.0f) +
                  c[2] * ex2_fast(-c[5] * r) * fmaf(-c[5] * kLn2, r, -1.0f);
  const float G = c[9] * c[6] * ex2_fast(-c[9] * r2) + c[10] * c[7] * ex2_fast(-c[10] * r2) +
                  c[11] * c[8] * ex2_fast(-c[11] * r2);
  return 0.5f * L * ri * ri * ri - kLn2 * G;
}

// Adjoint of the separable potential with respect to the atoms' x and y: for
// the slice's dL/dV field G and V(p) = sum_atoms sum_j exp(-alpha_j rho^2)
// T_K(p)[j] (the same K, the same exact-position values as k_potential_sep),
//   dL/dX = 2 sum_p G(p) (px - X) sum_j alpha_j exp(-alpha_j rho^2) T_K[j],
// likewise for Y (the cut-off decisions are not differentiated, as in the
// per-sub-plane adjoint).  Pixels with a sub-plane inside the 0.25 A clamp
// take the per-sub-plane derivative.  blockIdx.x: the atom of the window (its
// table row), blockIdx.y: one of gridDim.y interleaved row sets of its
// +-2.3 A pixel square; FP64 block sums, added atomically in input order.
__global__ void __launch_bounds__(kPotThreads) k_potential_sep_adjoint(PotArgs a, const float* __restrict__ G,
                                                                       const int* __restrict__ perm, int a0,
                                                                       double* __restrict__ dxy) {
  __shared__ float s_t[32];
  __shared__ float s_qv[20];
  __shared__ __align__(16) float s_al[kGaussJ];
  __shared__ double s_red[2][kPotThreads / 32];
  constexpr float kLn2 = 0.6931471805599453f;
  const int l = a0 + blockIdx.x;
  const float4 at = a.atoms[l];
  const float* tab = a.tab + (size_t)blockIdx.x * kTabStride;
  const float* c = a.coef + (__float_as_int(at.w) - 1) * kCoefPerZ;
  if (threadIdx.x < 32) s_t[threadIdx.x] = tab[kTabQ + threadIdx.x];
  if (threadIdx.x < 20) s_qv[threadIdx.x] = tab[kTabQV + threadIdx.x];
  if (threadIdx.x < kGaussJ) s_al[threadIdx.x] = a.gauss[(__float_as_int(at.w) - 1) * 2 * kGaussJ + threadIdx.x];
  __syncthreads();
  const int xl = max((int)floorf((at.x - 2.3f - a.xoff) / a.ps), 0);
  const int xh = min((int)ceilf((at.x + 2.3f - a.xoff) / a.ps), a.nx - 1);
  const int yl = max((int)floorf((at.y - 2.3f - a.yoff) / a.ps), 0);
  const int yh = min((int)ceilf((at.y + 2.3f - a.yoff) / a.ps), a.ny - 1);
  const int wx = xh - xl + 1, wy = yh - yl + 1;
  const int ns = gridDim.y, js = blockIdx.y;
  const float t0 = s_t[0];
  float gx = 0.0f, gy = 0.0f;
  if (wx > 0 && wy > js) {
    const int npx = wx * ((wy - js + ns - 1) / ns);
    for (int w = threadIdx.x; w < npx; w += kPotThreads) {
      const int x = xl + w % wx, y = yl + js + (w / wx) * ns;
      const float px = fadd_x(a.xoff, fmul_x((float)x, a.ps));
      const float py = fadd_x(a.yoff, fmul_x((float)y, a.ps));
      const float dx = fsub_x(px, at.x), dy = fsub_x(py, at.y);
      const float dxy2 = fadd_x(fmul_x(dx, dx), fmul_x(dy, dy));
      int K = 0;
#pragma unroll
      for (int st = 16; st >= 1; st >>= 1)
        if (dxy2 < s_t[K + st - 1]) K += st;
      if (K == 0) continue;
      const float dxv = dx + (float)(((double)a.xoff + (double)x * (double)a.ps) - (double)px);
      const float dyv = dy + (float)(((double)a.yoff + (double)y * (double)a.ps) - (double)py);
      const float dxyv = fmaf(dxv, dxv, dyv * dyv);
      const float gp = G[(long long)y * a.nx + x];
      float D;  // d/d(rho^2) of the atom's value at this pixel
      if (dxy2 < t0 - 4.9373f) {
        D = 0.0f;
        for (int k = 0; k < K; ++k) D += vatom_deriv_f(c, dxyv + s_qv[k]);
        D *= a.wsub;
      } else {
        const float4* T = reinterpret_cast<const float4*>(tab + kTabT + (K - 1) * kGaussJ);
        float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
        for (int g = 0; g < kGaussJ / 4; ++g) {
          const float4 al = *reinterpret_cast<const float4*>(&s_al[4 * g]);
          const float4 tt = __ldg(T + g);
          e0 = fmaf(al.x * ex2_fast(-al.x * dxyv), tt.x, e0);
          e1 = fmaf(al.y * ex2_fast(-al.y * dxyv), tt.y, e1);
          e0 = fmaf(al.z * ex2_fast(-al.z * dxyv), tt.z, e0);
          e1 = fmaf(al.w * ex2_fast(-al.w * dxyv), tt.w, e1);
        }
        D = -kLn2 * (e0 + e1);  // (s_al holds alpha_j log2(e))
      }
      gx += gp * D * dxv;
      gy += gp * D * dyv;
    }
  }
  double sx = gx, sy = gy;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sy += __shfl_down_sync(0xffffffffu, sy, o);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_red[0][warp] = sx;
    s_red[1][warp] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tx = 0.0, ty = 0.0;
    for (int k = 0; k < kPotThreads / 32; ++k) {
      tx += s_red[0][k];
      ty += s_red[1][k];
    }
    const int i = perm[l];
    atomicAdd(dxy + 2 * i, -2.0 * tx);
    atomicAdd(dxy + 2 * i + 1, -2.0 * ty);
  }
}

}  // namespace

cudaError_t launch_potential_adjoint(const PotArgs& a, const float* G, const int* perm, int a0, int a1, double* dxy,
                                     cudaStream_t s, bool separable) {
  if (a1 <= a0) return cudaSuccess;
  // about 8 CTAs per SM (148 SMs) in all, at most 16 row sets per atom
  const int na = a1 - a0;
  const int ns = std::min(16, std::max(1, (8 * 148 + na - 1) / na));
  if (separable) {
    if (!a.tab || !a.gauss) return cudaErrorInvalidValue;
    // the slice's per-atom tables (a0 is the window's first atom, as there)
    k_atom_tables<<<148 * 8, 256, 0, s>>>(a);
    k_potential_sep_adjoint<<<dim3(na, ns), kPotThreads, 0, s>>>(a, G, perm, a0, dxy);
    return cudaGetLastError();
  }
  k_potential_conv_adjoint<<<dim3(na, ns), kPotThreads, 0, s>>>(a, G, perm, a0, dxy);
  return cudaGetLastError();
}

size_t bin_scratch_blocks(int nbins) { return (size_t)(nbins + kScanTile - 1) / kScanTile + 1; }

cudaError_t build_atom_index(const int* dZ, const float* dx, const float* dy, const float* dz, int n,
                             const Box& box, int nz, AtomIndex& out, BinScratch& scr, cudaStream_t s) {
  const int nbins = nz * kBins2;
  cudaError_t e;
  if ((e = cudaMemsetAsync(scr.cursor, 0, sizeof(int) * nbins, s)) != cudaSuccess) return e;
  const int tb = 256;
  k_bin_keys<<<(n + tb - 1) / tb, tb, 0, s>>>(dx, dy, dz, n, box, nz, scr.key, scr.cursor);
  // offsets = exclusive scan of the counts; off[nbins] = n
  const int ntiles = (nbins + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<ntiles, kScanThreads, 0, s>>>(scr.cursor, nbins, out.off, scr.blocksum);
  k_scan_sums<<<1, kScanThreads, 0, s>>>(scr.blocksum, ntiles, out.off + nbins);
  k_scan_add<<<(nbins + tb - 1) / tb, tb, 0, s>>>(out.off, nbins, scr.blocksum);
  if ((e = cudaMemcpyAsync(scr.cursor, out.off, sizeof(int) * nbins, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return e;
  k_scatter<<<(n + tb - 1) / tb, tb, 0, s>>>(scr.key, n, scr.cursor, scr.idx);
  k_sort_bins<<<(nbins + tb - 1) / tb, tb, 0, s>>>(out.off, nbins, scr.idx);
  k_gather<<<(n + tb - 1) / tb, tb, 0, s>>>(scr.idx, n, dZ, dx, dy, dz, box, out.atoms);
  out.n = n;
  out.nz = nz;
  return cudaGetLastError();
}

int potential_tiles() { return 3; }
int potential_tiles_separable() { return 4; }

cudaError_t launch_atom_tables(const PotArgs& a, cudaStream_t s, int nbatch) {
  if (!a.tab || !a.gauss || nbatch < 1 || nbatch > 65535) return cudaErrorInvalidValue;
  // the window's atoms (read on the device) in 16-atom rounds
  k_atom_tables<<<dim3(nbatch > 1 ? 296 : 148 * 8, nbatch), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_potential_from_tables(const PotArgs& a, cudaStream_t s, int tile, int nbatch) {
  if (!a.tab || !a.gauss || nbatch < 1 || nbatch > 65535) return cudaErrorInvalidValue;
  // tiles of two or four pixels per thread: 16 x 32, 32 x 16, 16 x 64, 32 x 32
  const int nb = nbatch;
  switch (tile) {
    case 0: k_potential_sep<16, 32, 2><<<dim3((a.nx + 15) / 16, (a.ny + 31) / 32, nb), kPotThreads, 0, s>>>(a); break;
    case 1: k_potential_sep<32, 16, 2><<<dim3((a.nx + 31) / 32, (a.ny + 15) / 16, nb), kPotThreads, 0, s>>>(a); break;
    case 2: k_potential_sep<16, 64, 4><<<dim3((a.nx + 15) / 16, (a.ny + 63) / 64, nb), kPotThreads, 0, s>>>(a); break;
    case 3: k_potential_sep<32, 32, 4><<<dim3((a.nx + 31) / 32, (a.ny + 31) / 32, nb), kPotThreads, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_potential(const PotArgs& a, int kind, cudaStream_t s, int tile, bool separable, int nbatch) {
  dim3 grid((a.nx + kTX - 1) / kTX, (a.ny + kTY - 1) / kTY);
  if (kind == POT_CONVENTIONAL && separable) {
    if (!a.tab || !a.gauss || nbatch < 1 || nbatch > 65535) return cudaErrorInvalidValue;
    // the window's atoms (read on the device) in 16-atom rounds
    k_atom_tables<<<dim3(nbatch > 1 ? 296 : 148 * 8, nbatch), 256, 0, s>>>(a);
    // tiles of two or four pixels per thread: 16 x 32, 32 x 16, 16 x 64, 32 x 32
    const int nb = nbatch;
    switch (tile) {
      case 0: k_potential_sep<16, 32, 2><<<dim3((a.nx + 15) / 16, (a.ny + 31) / 32, nb), kPotThreads, 0, s>>>(a); break;
      case 1: k_potential_sep<32, 16, 2><<<dim3((a.nx + 31) / 32, (a.ny + 15) / 16, nb), kPotThreads, 0, s>>>(a); break;
      case 2: k_potential_sep<16, 64, 4><<<dim3((a.nx + 15) / 16, (a.ny + 63) / 64, nb), kPotThreads, 0, s>>>(a); break;
      case 3: k_potential_sep<32, 32, 4><<<dim3((a.nx + 31) / 32, (a.ny + 31) / 32, nb), kPotThreads, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  }
  if (nbatch != 1) return cudaErrorInvalidValue;
  if (kind == POT_CONVENTIONAL) {
    switch (tile) {
      case 0: k_potential_conv<32, 8><<<grid, kPotThreads, 0, s>>>(a); break;
      case 1: k_potential_conv<16, 16><<<dim3((a.nx + 15) / 16, (a.ny + 15) / 16), kPotThreads, 0, s>>>(a); break;
      case 2: k_potential_conv<64, 4><<<dim3((a.nx + 63) / 64, (a.ny + 3) / 4), kPotThreads, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  }
  switch (kind) {
    case POT_FD: k_potential<POT_FD><<<grid, kPotThreads, 0, s>>>(a); break;
    case POT_PROJECTED: k_potential<POT_PROJECTED><<<grid, kPotThreads, 0, s>>>(a); break;
    case POT_RS: k_potential<POT_RS><<<grid, kPotThreads, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ms
