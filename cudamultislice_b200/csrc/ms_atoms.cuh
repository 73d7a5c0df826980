// ms_atoms.cuh -- atom index (bit-exact binning) and projected-potential build.
#pragma once
#include <cuda_runtime.h>
#include "ms_common.cuh"

namespace ms {

// Box as computed by LoadAtomFile (U.cu:1350-1355).
struct Box {
  float MaxX, MinX, MaxY, MinY, MaxZ, MinZ;
};

// Device atom index: atoms sorted slice -> y-bin -> x-bin, stable in input
// order, positions shifted by the box minimum (U.cu:1444-1525).
struct AtomIndex {
  float4* atoms;   // (x, y, z, Z as int bits), shifted frame
  int* off;        // CSR offsets, nz * 2500 + 1
  int n;           // atoms
  int nz;          // 1-A z-bins
};

// Scratch for building the index (all sized by n or by the bin count).
struct BinScratch {
  int* key;      // n
  int* idx;      // n
  int* cursor;   // nbins
  int* blocksum; // scan partials
};

size_t bin_scratch_blocks(int nbins);
cudaError_t build_atom_index(const int* dZ, const float* dx, const float* dy, const float* dz, int n,
                             const Box& box, int nz, AtomIndex& out, BinScratch& scr, cudaStream_t s);

// Per-Z coefficients of vatom / vzatom2 derived from one fparams row on the
// host in FP64: 12 floats for vatom, then 12 for vzatom2 (see engine).
constexpr int kCoefPerZ = 24;

enum PotKind : int { POT_CONVENTIONAL = 0, POT_FD = 1, POT_PROJECTED = 2, POT_RS = 3 };

struct PotArgs {
  const float4* atoms;
  const int* off;
  const float* coef;     // [103][kCoefPerZ]
  float* V;              // [ny][nx] output (V*A, not yet exponentiated)
  int nx, ny, nz;
  float ps, xoff, yoff;  // pixel (x,y) sits at (xoff + x*ps, yoff + y*ps) in the shifted frame
  float bw_x, bw_y;      // bin widths (MaxX-MinX)/50, (MaxY-MinY)/50
  int kt, kb;            // inclusive z-bin window
  int nsub;              // sub-planes (20 conventional, 1 finite difference)
  float zsub[20];        // sub-plane z (shifted frame), FP32 as the reference
  float zsub_lo[20];     // exact height minus zsub (values only; the cut-off
                         // decisions use zsub as the reference rounds it)
  float wsub;            // weight per sub-plane
  // projected mode: atoms with floorf((top - z)/dz) == slab
  float top, slab_dz;
  int slab;
  long long batch_stride_V;
  // separable conventional kernel: per-atom tables of the slice (written by
  // the table kernel, kTabStride floats per atom of the z-window, in CSR
  // order) and the Gaussian expansions [103][2][kGaussJ] (alpha_j log2(e),
  // then w_j)
  float* tab;
  const float* gauss;
  // batched separable builds (one instance per blockIdx.z of the pixel kernel,
  // blockIdx.y of the table kernel): element strides of atoms, off, tab and V
  // between instances (0 for one instance)
  long long b_atoms, b_off, b_tab, b_V;
};

// Gaussian expansion of vatom per element: v(r) ~= sum_j w_j exp(-alpha_j r^2)
// for 0.25 A <= r <= 2.2365 A (positive weights).
constexpr int kGaussJ = 12;
// Per-atom table of one slice (floats): for the sub-planes that can pass the
// cut-off, in ascending reference-rounded dz_m^2, the thresholds t_k with
// "fadd(dxy, dz_k^2) < 5 exactly when dxy < t_k", padded with -1e30 to 32;
// the exact-height dz_m^2 in the same order; then row k = 0..19:
// wsub sum_{k' <= k} w_j exp(-alpha_j dzv_k'^2), j < kGaussJ.
constexpr int kTabQ = 0, kTabQV = 32, kTabT = 56, kTabStride = 304;

// tile: the conventional kernel's tile shape variant (0: 32 x 8, 1: 16 x 16,
// 2: 64 x 4 pixels; other kinds take 32 x 8).
// separable: conventional kind only, through the per-atom tables (a.tab,
// a.gauss set) instead of the per-sub-plane sum.
cudaError_t launch_potential(const PotArgs& a, int kind, cudaStream_t s, int tile = 0, bool separable = false,
                             int nbatch = 1);
int potential_tiles();
int potential_tiles_separable();
// The separable conventional kernel's two launches apart (launch_potential
// with separable = true enqueues both on one stream): the per-atom tables of
// the slice into a.tab, then the potential from them.
cudaError_t launch_atom_tables(const PotArgs& a, cudaStream_t s, int nbatch = 1);
cudaError_t launch_potential_from_tables(const PotArgs& a, cudaStream_t s, int tile, int nbatch = 1);

// Adjoint of the conventional potential of one slice with respect to atom x, y:
// dxy[2 perm[l] + {0,1}] += dL/d{x,y} of sorted atoms l in [a0, a1) (the CSR
// range of the slice's z-window), G = dL/dV of the slice [ny][nx].
// separable: through the per-atom tables of the separable kernel (a.tab,
// a.gauss set; a0 must be the first atom of the slice's z-window).
cudaError_t launch_potential_adjoint(const PotArgs& a, const float* G, const int* perm, int a0, int a1, double* dxy,
                                     cudaStream_t s, bool separable = false);

}  // namespace ms
