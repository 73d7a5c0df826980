// ms_engine.cu -- host engine and C ABI of the B200 multislice library.
//
// ms::Engine is the B200-native counterpart of the reference class
// UnmanagedMultisliceSimulation (GUI Simulation/unmanagedGUISimulation.cuh:62-200,
// GUI Simulation/UnmanagedGUISimulation.cu = "U.cu").  Set-up scalars that the
// reference computes on the host in FP32 (wavelength, interaction constant,
// finite-difference step, frequencies, kmax, slice planes) are computed here
// with the same FP32 operations in the same order, so the engine solves exactly
// the reference's problem; the heavy numerics run in the CUDA kernels of
// ms_atoms.cu (binning, potentials), ms_slice.cu (fused slice passes) and
// ms_pointwise.cu (plain path, finite differences, probe, read-out).
#include <cufft.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mslice.h"
#include "ms_atoms.cuh"
#include "ms_philox.h"
#include "ms_tiff.h"
#include "ms_pointwise.cuh"
#include "ms_slice.cuh"

// Inside Engine members: return an ms_status with the message set.
#define MS_TRY(expr)                                    \
  do {                                                  \
    cudaError_t _e = (expr);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
  } while (0)
#define MS_TRY_FFT(expr)                                                                 \
  do {                                                                                   \
    cufftResult _r = (expr);                                                             \
    if (_r != CUFFT_SUCCESS) return fail(MS_ERR_CUDA, std::string("cuFFT failed: ") + #expr); \
  } while (0)

namespace ms {

// Gaussian expansions of vatom per element for the separable potential kernel
// (kGaussFit[Z-1] = {J, alpha_j..., w_j...}), fitted offline to the stock
// fparams.dat and re-checked against the loaded table before use.
#include "ms_gauss_fit.inc"

// ---------------------------------------------------------------------------
// small utilities
// ---------------------------------------------------------------------------
struct Status {
  int code;
  std::string msg;
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t resize(size_t count) {
    if (count == n && p) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
};

// Element symbols for Z = 1..103 (the rows of fparams.dat).
static const char* const kElements[103] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar",
    "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe",
    "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf",
    "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr"};

// GetZNum U.cu:1188-1243: the reference knows 25 symbols; any other maps to 1.
static int znum(const std::string& s, bool full) {
  static const int ref_known[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 12, 14, 15, 16, 17, 20, 24, 35, 26, 38, 44, 57, 62, 73, 74};
  if (full) {
    for (int z = 1; z <= 103; ++z)
      if (s == kElements[z - 1]) return z;
    return 1;
  }
  for (int z : ref_known)
    if (s == kElements[z - 1]) return z;
  return 1;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
class Engine {
 public:
  explicit Engine(int device) : device_(device) {}
  ~Engine() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (fd_graph_) cudaGraphExecDestroy(fd_graph_);
    if (h_loop_err_) cudaFreeHost(h_loop_err_);
    if (have_plan_) cufftDestroy(plan_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    for (int k = 0; k < kPixStreams; ++k)
      for (cudaEvent_t e : {ev_tab_[k], ev_pix_[k], ev_pjoin_[k]})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_fork_, ev_fork2_, ev_join_, ev_dv_, ev_adj_[0], ev_adj_[1]})
      if (e) cudaEventDestroy(e);
    if (side_) cudaStreamDestroy(side_);
    for (int k = 1; k < kPixStreams; ++k)
      if (pix_[k]) cudaStreamDestroy(pix_[k]);
    if (pass_) cudaStreamDestroy(pass_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  std::string err;
  long long launches = 0;

  int init() {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(MS_ERR_CUDA, "no CUDA device available");
    if (device_ < 0 || device_ >= ndev) return fail(MS_ERR_INVALID, "device index out of range");
    MS_TRY(cudaSetDevice(device_));
    MS_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    MS_TRY(cudaEventCreate(&ev0_));
    MS_TRY(cudaEventCreate(&ev1_));
    // the side stream of the potential stack (tables of the next slice while
    // the current slice's potential runs) and its ordering events
    // (the side stream's tables and the pass stream's slice steps are short
    // launches on the critical path: their CTAs are scheduled ahead of the
    // pixel streams' potentials)
    int prio_lo = 0, prio_hi = 0;
    MS_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    MS_TRY(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, prio_hi));
    pix_[0] = stream_;
    for (int k = 1; k < kPixStreams; ++k) MS_TRY(cudaStreamCreateWithFlags(&pix_[k], cudaStreamNonBlocking));
    MS_TRY(cudaStreamCreateWithPriority(&pass_, cudaStreamNonBlocking, prio_hi));
    for (int k = 0; k < kPixStreams; ++k)
      for (cudaEvent_t* e : {&ev_tab_[k], &ev_pix_[k], &ev_pjoin_[k]})
        MS_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (cudaEvent_t* e : {&ev_fork_, &ev_fork2_, &ev_join_, &ev_dv_, &ev_adj_[0], &ev_adj_[1]})
      MS_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    MS_TRY(d_loop_sync_.resize(2));
    MS_TRY(d_pass_err_.resize(1));
    MS_TRY(cudaMemsetAsync(d_pass_err_.p, 0, sizeof(int), stream_));
    MS_TRY(cudaHostAlloc((void**)&h_loop_err_, sizeof(unsigned int), cudaHostAllocDefault));
    *h_loop_err_ = 0;
    return MS_OK;
  }

  // ---- options ----
  int set_option(int opt, int value) {
    switch (opt) {
      case MS_OPT_SLICE_PATH:
        if (value != 0 && value != 1) return fail(MS_ERR_INVALID, "slice path must be 0 (fused) or 1 (plain)");
        force_plain_ = value == 1;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_ELEMENT_TABLE:
        if (value != 0 && value != 1) return fail(MS_ERR_INVALID, "element table must be 0 or 1");
        full_table_ = value == 1;
        return MS_OK;
      case MS_OPT_POTENTIAL:
        if (value != 0 && value != 1) return fail(MS_ERR_INVALID, "potential mode must be 0 or 1");
        pot_mode_ = value;
        stack_valid_ = false;
    fd_stack_valid_ = false;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_CHECKPOINT:
        if (value < 0) return fail(MS_ERR_INVALID, "checkpoint stride must be 0 (automatic) or >= 1");
        ckpt_ = value;
        return MS_OK;
      case MS_OPT_FFT_PLAN:
        if (value < -1 || value >= plan_variants()) return fail(MS_ERR_INVALID, "FFT plan must be -1 (tuned) or a variant index");
        forced_plan_ = value;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_SLICE_LOOP:
        if (value != 0 && value != 1) return fail(MS_ERR_INVALID, "slice loop must be 0 (persistent) or 1 (per pass)");
        loop_off_ = value == 1;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_LOOP_WAIT_US:
        if (value < 1) return fail(MS_ERR_INVALID, "wait bound must be >= 1 microsecond");
        loop_limit_ns_ = 1000ull * (unsigned long long)value;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_LOOP_VARIANT:
        if (value < -1 || value >= slice_loop_variants())
          return fail(MS_ERR_INVALID, "loop variant must be -1 (tuned) or a variant index");
        forced_loop_ = value;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_POTENTIAL_TILE:
        if (value < -1 || value >= std::max(potential_tiles(), potential_tiles_separable()))
          return fail(MS_ERR_INVALID, "tile must be -1 (tuned) or a tile index of the potential kernels");
        pot_tile_ = value;
        pot_tile_forced_ = value >= 0;
        stack_valid_ = false;
        fd_stack_valid_ = false;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_POTENTIAL_SUM:
        if (value < 0 || value > 2) return fail(MS_ERR_INVALID, "potential sum must be 0 (auto), 1 or 2");
        pot_sum_ = value;
        if (!pot_tile_forced_) pot_tile_ = -1;  // (the tile is tuned per kernel)
        stack_valid_ = false;
        fd_stack_valid_ = false;
        invalidate_graph();
        return MS_OK;
      case MS_OPT_BUILD_OVERLAP:
        if (value != 0 && value != 1) return fail(MS_ERR_INVALID, "build overlap must be 0 or 1");
        overlap_build_ = value == 1;
        return MS_OK;
      case MS_OPT_LOOP_WAIT_TEST:
        if (value < 0) return fail(MS_ERR_INVALID, "test arrivals must be >= 0");
        loop_extra_ = (unsigned int)value;
        invalidate_graph();
        return MS_OK;
      default:
        return fail(MS_ERR_INVALID, "unknown option");
    }
  }

  // ---- structure ----
  int import_atoms(const char* path) {
    if (!path) return fail(MS_ERR_INVALID, "null path");
    std::ifstream in(path);
    if (!in) return fail(MS_ERR_IO, std::string("cannot open structure file ") + path);
    // LoadAtomFile reads the count, discards the rest of that line (its
    // comment) and then reads "symbol x y z" records (U.cu:1309-1321).  A
    // separate comment line, as in the common .xyz layout, would be read by the
    // reference as an atom; here a line that is not an atom record is skipped.
    int n = 0;
    if (!(in >> n) || n <= 0) return fail(MS_ERR_IO, "structure file: bad atom count");
    std::string line;
    std::getline(in, line);
    std::vector<int> Z;
    std::vector<float> x, y, z;
    Z.reserve(n);
    x.reserve(n);
    y.reserve(n);
    z.reserve(n);
    bool first = true;
    while ((int)Z.size() < n && std::getline(in, line)) {
      std::istringstream ls(line);
      std::string sym;
      float a, b, c;
      if (!(ls >> sym >> a >> b >> c)) {
        if (first && line.find_first_not_of(" \t\r") != std::string::npos) {
          first = false;  // a comment line after the count
          continue;
        }
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        return fail(MS_ERR_IO, "structure file: malformed atom record");
      }
      first = false;
      Z.push_back(znum(sym, full_table_));
      x.push_back(a);
      y.push_back(b);
      z.push_back(c);
    }
    if ((int)Z.size() < n) return fail(MS_ERR_IO, "structure file: truncated atom list");
    return set_atoms(Z.data(), x.data(), y.data(), z.data(), n);
  }

  int set_atoms(const int* Z, const float* x, const float* y, const float* z, int n) {
    if (n <= 0 || !Z || !x || !y || !z) return fail(MS_ERR_INVALID, "no atoms");
    for (int i = 0; i < n; ++i) {
      if (Z[i] < 1 || Z[i] > 103) return fail(MS_ERR_INVALID, "atomic number out of range 1..103");
      if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i]))
        return fail(MS_ERR_INVALID, "non-finite atom position");
    }
    hZ_.assign(Z, Z + n);
    zpresent_.assign(104, 0);
    for (int i = 0; i < n; ++i) zpresent_[Z[i]] = 1;
    hx_.assign(x, x + n);
    hy_.assign(y, y + n);
    hz_.assign(z, z + n);
    // bounding box as LoadAtomFile (U.cu:1326-1355): extreme atoms, +-2 A in FP32
    float x1 = hx_[0], x0 = hx_[0], y1 = hy_[0], y0 = hy_[0], z1 = hz_[0], z0 = hz_[0];
    for (int i = 1; i < n; ++i) {
      x1 = std::max(x1, hx_[i]);
      x0 = std::min(x0, hx_[i]);
      y1 = std::max(y1, hy_[i]);
      y0 = std::min(y0, hy_[i]);
      z1 = std::max(z1, hz_[i]);
      z0 = std::min(z0, hz_[i]);
    }
    box_.MaxX = x1 + 2;
    box_.MinX = x0 - 2;
    box_.MaxY = y1 + 2;
    box_.MinY = y0 - 2;
    box_.MaxZ = z1 + 2;
    box_.MinZ = z0 - 2;
    have_atoms_ = true;
    have_index_ = false;
    stack_valid_ = false;
    fd_stack_valid_ = false;  // (the slice-loop graph depends on the stack's allocation only)
    return MS_OK;
  }

  int upload_binned(bool tds, uint64_t seed, uint32_t pass, float sigma) {
    if (!have_atoms_) return fail(MS_ERR_STATE, "no atoms: call ms_import_atoms or ms_set_atoms first");
    const int n = (int)hx_.size();
    std::vector<float> x = hx_, y = hy_, z = hz_;
    if (tds) {
      if (!(sigma >= 0) || !std::isfinite(sigma)) return fail(MS_ERR_INVALID, "bad thermal displacement sigma");
      tds_displace(hx_.data(), hy_.data(), hz_.data(), n, seed, pass, sigma, x.data(), y.data(), z.data());
    }
    // nSlices = ceil((MaximumZ-MinimumZ)/dz), dz = 1 (U.cu:1409-1411); the
    // extent is range-checked before the conversion to int
    const float zext = std::ceil((box_.MaxZ - box_.MinZ) / (float)1);
    if (!std::isfinite(zext) || zext < 0.0f || (double)zext * kBins2 > (double)(INT_MAX - 1))
      return fail(MS_ERR_INVALID, "structure too deep for the atom index: " + std::to_string(zext) + " z-bins");
    int nz = (int)zext;
    nz += (nz == 0);
    const int nbins = nz * kBins2;
    MS_TRY(d_Zin_.resize(n));
    MS_TRY(d_xin_.resize(n));
    MS_TRY(d_yin_.resize(n));
    MS_TRY(d_zin_.resize(n));
    MS_TRY(d_atoms_.resize(n));
    if (d_tab_.n < (size_t)n * kTabStride) MS_TRY(d_tab_.resize((size_t)n * kTabStride));
    MS_TRY(d_off_.resize(nbins + 1));
    MS_TRY(d_key_.resize(n));
    MS_TRY(d_idx_.resize(n));
    MS_TRY(d_cursor_.resize(nbins));
    MS_TRY(d_blocksum_.resize(bin_scratch_blocks(nbins)));
    MS_TRY(cudaMemcpyAsync(d_Zin_.p, hZ_.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemcpyAsync(d_xin_.p, x.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemcpyAsync(d_yin_.p, y.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemcpyAsync(d_zin_.p, z.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
    AtomIndex idx{d_atoms_.p, d_off_.p, 0, 0};
    BinScratch scr{d_key_.p, d_idx_.p, d_cursor_.p, d_blocksum_.p};
    MS_TRY(build_atom_index(d_Zin_.p, d_xin_.p, d_yin_.p, d_zin_.p, n, box_, nz, idx, scr, stream_));
    launches += 8;
    MS_TRY(cudaStreamSynchronize(stream_));
    natoms_ = n;
    nzb_ = nz;
    have_index_ = true;
    hzoff_.clear();
    stack_valid_ = false;
    fd_stack_valid_ = false;
    return MS_OK;
  }

  // fparams.dat, U.cu:1718-1747: rows of 12 numbers, row Z-1.
  int get_parameterisation(const char* path) {
    if (!path) return fail(MS_ERR_INVALID, "null path");
    std::ifstream in(path);
    if (!in) return fail(MS_ERR_IO, std::string("cannot open parameterisation file ") + path);
    std::vector<double> fp;
    double v[12];
    while (fp.size() < 103 * 12) {
      int k = 0;
      for (; k < 12; ++k)
        if (!(in >> v[k])) break;
      if (k < 12) break;
      fp.insert(fp.end(), v, v + 12);
    }
    if (fp.empty()) return fail(MS_ERR_IO, "parameterisation file holds no complete row");
    nrows_fp_ = (int)(fp.size() / 12);
    for (double d : fp)
      if (!std::isfinite(d)) return fail(MS_ERR_IO, "parameterisation file holds a non-finite value");
    // Per-Z coefficients in FP64, rounded once (layout in ms_atoms.cu).
    const double pi = 3.141592654, log2e = 1.4426950408889634;
    std::vector<float> coef(103 * kCoefPerZ, 0.0f);
    for (int r = 0; r < nrows_fp_; ++r) {
      const double* f = &fp[r * 12];
      float* c = &coef[r * kCoefPerZ];
      bool ok = true;
      for (int i = 0; i < 3; ++i) {
        const double a = f[2 * i], b = f[2 * i + 1], cc = f[6 + 2 * i], d = f[7 + 2 * i];
        if (!(b >= 0) || !(d > 0)) { ok = false; break; }
        c[i] = (float)(150.4121417 * a);
        c[3 + i] = (float)(2.0 * pi * std::sqrt(b) * log2e);
        c[6 + i] = (float)(266.5157269 * cc * std::pow(d, -1.5));
        c[9 + i] = (float)(pi * pi / d * log2e);
        c[12 + i] = (float)(300.8242834 * a);
        c[15 + i] = (float)(2.0 * pi * std::sqrt(b));
        c[18 + i] = (float)(150.4121417 * cc / d);
        c[21 + i] = (float)(pi * pi / d * log2e);
      }
      if (!ok) return fail(MS_ERR_IO, "parameterisation row with b < 0 or d <= 0");
    }
    MS_TRY(d_coef_.resize(coef.size()));
    MS_TRY(copy_sync(d_coef_.p, coef.data(), sizeof(float) * coef.size(), cudaMemcpyHostToDevice));
    // the Gaussian expansions, in the kernel's FP32 form (alpha_j log2(e), w_j)
    std::vector<float> gauss(103 * 2 * kGaussJ, 0.0f);
    for (int r = 0; r < 103; ++r) {
      if ((int)kGaussFit[r][0] != kGaussJ) continue;
      for (int j = 0; j < kGaussJ; ++j) {
        gauss[(r * 2) * kGaussJ + j] = (float)(kGaussFit[r][1 + j] * log2e);
        gauss[(r * 2 + 1) * kGaussJ + j] = (float)kGaussFit[r][1 + kGaussJ + j];
      }
    }
    MS_TRY(d_gauss_.resize(gauss.size()));
    MS_TRY(copy_sync(d_gauss_.p, gauss.data(), sizeof(float) * gauss.size(), cudaMemcpyHostToDevice));
    hfp_ = fp;
    hgauss_ = gauss;
    gauss_row_ok_.assign(103, -1);
    have_fp_ = true;
    stack_valid_ = false;
    fd_stack_valid_ = false;
    invalidate_graph();
    return MS_OK;
  }

  int apply_microscope(float kV, float df, float A2, float phi2, float Cs, float beta, float delta, float ap) {
    const float v[8] = {kV, df, A2, phi2, Cs, beta, delta, ap};
    for (float f : v)
      if (!std::isfinite(f)) return fail(MS_ERR_INVALID, "non-finite microscope parameter");
    if (!(kV > 0)) return fail(MS_ERR_INVALID, "accelerating voltage must be positive");
    kV_ = kV; df_ = df; A2_ = A2; phi2_ = phi2; Cs_ = Cs; beta_ = beta; delta_ = delta; aperture_ = ap;
    have_micro_ = true;
    return MS_OK;
  }

  // SetCalculationVariables U.cu:1763-1875 (stem = false) and
  // STEMSetCalculationVariables U.cu:2567-2670 (stem = true).
  int set_calc(float ps, float df, int nx, int ny, float sizeZ, float xoff, float yoff, bool stem) {
    if (!have_micro_) return fail(MS_ERR_STATE, "microscope parameters not applied");
    if (!have_atoms_) return fail(MS_ERR_STATE, "no atoms");
    if (nx < 2 || ny < 2 || nx > 16384 || ny > 16384) return fail(MS_ERR_INVALID, "grid size out of range 2..16384");
    if (!(ps > 0) || !std::isfinite(ps) || !std::isfinite(df) || !std::isfinite(xoff) || !std::isfinite(yoff))
      return fail(MS_ERR_INVALID, "bad pixel size, defocus or offset");
    nx_ = nx; ny_ = ny; ps_ = ps; df_ = df; stem_ = stem;
    xoff_ = stem ? 0.0f : xoff;
    yoff_ = stem ? 0.0f : yoff;
    const float ksizex = ps * nx, ksizey = ps * ny;
    const float Pi = 3.1415926f;
    const float V = kV_;
    const float echarge = 1.6e-019f;
    wavel_ = 6.63e-034f * 3e+008f / std::sqrt((echarge * V * 1000 * (2 * 9.11e-031f * 9e+016f + echarge * V * 1000))) *
             1e+010f;
    sigma2_ = (2 * Pi / (wavel_ * V * 1000)) *
              ((9.11e-031f * 9e+016f + echarge * V * 1000) / (2 * 9.11e-031f * 9e+016f + echarge * V * 1000));
    const float V2 = V * 1000;
    const float fnkx = (float)nx, fnky = (float)ny;
    const float p1 = fnkx / (2 * ksizex), p2 = fnky / (2 * ksizey);
    const float p12 = p1 * p1, p22 = p2 * p2;
    const float ke2 = (.666666f) * (p12 + p22);
    const float qA = (ke2 * ke2 * 16 * Pi * Pi * Pi * Pi) - (32 * Pi * Pi * Pi * ke2 * sigma2_ * V2 / wavel_) +
                     (16 * Pi * Pi * sigma2_ * sigma2_ * V2 * V2 / (wavel_ * wavel_));
    const float qB = 16 * Pi * Pi * (ke2 - (sigma2_ * V2 / (Pi * wavel_)) - (1 / (4 * wavel_ * wavel_)));
    const float qC = 3;
    const float disc = qB * qB - 4 * qA * qC;
    float msd = (-qB + std::sqrt(disc)) / (2 * qA);
    msd = (float)(0.99 * (double)std::sqrt(msd));
    if (stem && msd > 0.06) msd = (float)0.06;
    int nFD = (int)std::ceil(sizeZ / msd);
    nFD += (nFD == 0);
    fd_stable_ = disc >= 0 && msd > 0 && std::isfinite(msd);
    dzFD_ = msd;
    nFD_ = fd_stable_ ? nFD : -1;
    lbz_ = (int)std::ceil(std::sqrt(5.0f) / (float)1);  // consts[2], U.cu:1859
    have_calc_ = true;
    have_freq_ = false;
    have_waves_ = false;
    stack_valid_ = false;
    fd_stack_valid_ = false;
    invalidate_graph();
    return MS_OK;
  }

  // PreCalculateFrequencies U.cu:1877-1964 (the unused doubled grids are not built).
  int precalc() {
    if (!have_calc_) return fail(MS_ERR_STATE, "calculation variables not set");
    const int nx = nx_, ny = ny_;
    const float ksizex = ps_ * nx, ksizey = ps_ * ny;
    const int imidx = (int)std::floor(nx / 2 + 0.5), imidy = (int)std::floor(ny / 2 + 0.5);
    hkx_.resize(nx);
    hky_.resize(ny);
    for (int i = 1; i <= nx; ++i) hkx_[i - 1] = ((i - 1) > imidx) ? ((i - 1) - nx) / ksizex : (i - 1) / ksizex;
    for (int i = 1; i <= ny; ++i) hky_[i - 1] = ((i - 1) > imidy) ? ((i - 1) - ny) / ksizey : (i - 1) / ksizey;
    const float kmaxx = (float)std::pow((double)(hkx_[imidx - 1] * 1 / 2), 2);
    const float kmaxy = (float)std::pow((double)(hky_[imidy - 1] * 1 / 2), 2);
    kmax_ = std::sqrt((kmaxy <= kmaxx) ? kmaxy : kmaxx);
    const size_t N = (size_t)nx * ny;
    MS_TRY(d_kx_.resize(nx));
    MS_TRY(d_ky_.resize(ny));
    MS_TRY(copy_sync(d_kx_.p, hkx_.data(), sizeof(float) * nx, cudaMemcpyHostToDevice));
    MS_TRY(copy_sync(d_ky_.p, hky_.data(), sizeof(float) * ny, cudaMemcpyHostToDevice));
    // wave buffers
    MS_TRY(d_psi0_.resize(N));
    MS_TRY(d_psi_.resize(N));
    MS_TRY(d_psim_.resize(N));
    MS_TRY(d_t1_.resize(N));
    MS_TRY(d_t2_.resize(N));
    MS_TRY(d_V_.resize(N));
    MS_TRY(d_f_.resize(N));
    MS_TRY(d_grad_.resize(N));
    MS_TRY(d_partial_.resize(1024 + 8));
    // cuFFT plan for the plain path, as U.cu:1961 (ny rows of nx)
    if (have_plan_) {
      cufftDestroy(plan_);
      have_plan_ = false;
    }
    if (cufftPlan2d(&plan_, ny, nx, CUFFT_C2C) != CUFFT_SUCCESS) return fail(MS_ERR_CUDA, "cufftPlan2d failed");
    if (cufftSetStream(plan_, stream_) != CUFFT_SUCCESS) return fail(MS_ERR_CUDA, "cufftSetStream failed");
    have_plan_ = true;
    fused_ok_ = fused_supported(nx, ny);
    tuned_.clear();
    raster_batch_.clear();
    loop_grid_ = 0;
    if (!pot_tile_forced_) pot_tile_ = -1;
    if (fused_ok_) {
      std::vector<float2> tw(2 * (size_t)std::max(nx, ny));
      for (int v = 0; v < plan_variants(); ++v) {
        const int sx = make_twiddles(nx, v, tw.data());
        MS_TRY(d_twx_[v].resize(std::max(sx, 1)));
        MS_TRY(copy_sync(d_twx_[v].p, tw.data(), sizeof(float2) * sx, cudaMemcpyHostToDevice));
        const int sy = make_twiddles(ny, v, tw.data());
        MS_TRY(d_twy_[v].resize(std::max(sy, 1)));
        MS_TRY(copy_sync(d_twy_[v].p, tw.data(), sizeof(float2) * sy, cudaMemcpyHostToDevice));
      }
    }
    prop_dz_ = -1.0f;
    have_freq_ = true;
    have_waves_ = false;
    stack_valid_ = false;
    fd_stack_valid_ = false;
    invalidate_graph();
    return MS_OK;
  }

  // ---- wavefunctions ----
  int init_waves(float conv_dz) {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    if (conv_dz > 0 && !std::isfinite(conv_dz)) return fail(MS_ERR_INVALID, "bad slice thickness");
    const float dz = conv_dz > 0 ? conv_dz : 1.0f;  // U.cu:1968 / U.cu:2005
    if (dz != convdz_) {
      stack_valid_ = false;
    fd_stack_valid_ = false;
      invalidate_graph();
    }
    convdz_ = dz;
    const Grid2 g{nx_, ny_};
    MS_TRY(pw_fill(d_psi0_.p, g, make_float2(1.f, 0.f), stream_, &launches));
    return finish_init();
  }

  int stem_init_waves(int px, int py) {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    const Grid2 g{nx_, ny_};
    const float apert = (float)((double)aperture_ * 0.001 / (double)wavel_);
    MS_TRY(pw_probe(d_t1_.p, d_kx_.p, d_ky_.p, px, py, apert, ps_, df_, Cs_, wavel_, g, stream_, &launches));
    // unnormalised inverse FFT (U.cu:2693), then divide by sum |psi| (U.cu:2698-2705)
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_psi0_.p, CUFFT_INVERSE));
    MS_TRY(pw_sum_abs(d_psi0_.p, (long long)nx_ * ny_, d_partial_.p, d_partial_.p + 1024, stream_, &launches));
    double l1 = 0;
    MS_TRY(cudaMemcpyAsync(&l1, d_partial_.p + 1024, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    if (!(l1 > 0)) return fail(MS_ERR_NUMERIC, "probe is empty (aperture smaller than one frequency pixel)");
    MS_TRY(pw_scale(d_psi0_.p, (float)(1.0 / l1), g, stream_, &launches));
    return finish_init();
  }

  int set_fd_dz(float dz) {
    if (!have_calc_) return fail(MS_ERR_STATE, "calculation variables not set");
    if (!(dz > 0) || !std::isfinite(dz)) return fail(MS_ERR_INVALID, "bad finite-difference step");
    dzFD_ = dz;
    int n = (int)std::ceil((box_.MaxZ - box_.MinZ) / dz);
    nFD_ = n + (n == 0);
    fd_stable_ = true;
    fd_stack_valid_ = false;
    invalidate_graph();
    return MS_OK;
  }

  // ---- steps ----
  int step_conventional(int it) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (it < 1) return fail(MS_ERR_INVALID, "iteration counts from 1");
    if (int rc = require_potential_inputs()) return rc;
    const float* V = nullptr;
    if (stack_valid_ && it <= nstack_) {
      V = d_stack_.p + (size_t)(it - 1) * nx_ * ny_;
    } else {
      if (int rc = potential_slice(pot_mode_ == 1 ? POT_PROJECTED : POT_CONVENTIONAL, it, d_V_.p)) return rc;
      V = d_V_.p;
    }
    return transmit_propagate(V, it == 1);
  }

  int step_fd(int it) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (it < 1) return fail(MS_ERR_INVALID, "iteration counts from 1");
    if (!fd_stable_) return fail(MS_ERR_NUMERIC, "no stable finite-difference step for these conditions");
    if (int rc = require_potential_inputs()) return rc;
    if (use_fused()) return step_fd_fused(it);
    if (int rc = ensure_real()) return rc;
    const Grid2 g{nx_, ny_};
    const float nf = 1.0f / std::sqrt((float)(nx_ * ny_));
    // V at the plane, band-limited (U.cu:2053-2063)
    if (int rc = potential_slice(POT_FD, it, d_f_.p)) return rc;
    MS_TRY(pw_real_to_complex(d_f_.p, d_t1_.p, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_bandlimit(d_t2_.p, d_kx_.p, d_ky_.p, kmax_, nf * nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t1_.p, CUFFT_INVERSE));  // t1 = band-limited V
    // spectral Laplacian of psi (U.cu:2066-2069)
    MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_laplacian(d_t2_.p, d_kx_.p, d_ky_.p, nf * nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_grad_.p, CUFFT_INVERSE));  // grad
    // three-level update (U.cu:2073) into t2
    MS_TRY(pw_fd_update(d_grad_.p, d_psim_.p, d_t2_.p, d_psi_.p, d_t1_.p, sigma2_, wavel_, dzFD_, g, stream_,
                        &launches));
    // band-limit psi+ (U.cu:2075-2078)
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t1_.p, CUFFT_FORWARD));
    MS_TRY(pw_bandlimit(d_t1_.p, d_kx_.p, d_ky_.p, kmax_, nf * nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_INVERSE));
    // rotate psi- <- psi <- psi+ (U.cu:2081-2082) by swapping buffers
    std::swap(d_psim_.p, d_psi_.p);  // psim = old psi
    std::swap(d_psi_.p, d_t2_.p);    // psi = psi+
    invalidate_graph();
    return MS_OK;
  }

  // MultisliceStepRS (U.cu:2126-2178) as written: the RS potential of the
  // plane (not exponentiated), ten series terms w <- w + i pre_m (L w + V w)
  // restarting from w = 1 (ping-pong buffers), then PsiMinus = w * Psi for
  // iterations after the first and Psi = w.  The reference does not expose
  // this step through its managed wrapper.
  int step_rs(int it) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (it < 1) return fail(MS_ERR_INVALID, "iteration counts from 1");
    if (int rc = require_potential_inputs()) return rc;
    if (int rc = ensure_real()) return rc;
    fd_state_ = false;
    const Grid2 g{nx_, ny_};
    if (int rc = potential_slice(POT_RS, it, d_f_.p)) return rc;
    const float pre0 = wavel_ * 1.0f / (4.0f * 3.1415927f);
    const float ips2 = 1.0f / (ps_ * ps_);
    float2* bufs[2] = {d_t1_.p, d_t2_.p};
    for (int m = 1; m <= 10; ++m)
      MS_TRY(pw_rs_term(bufs[m % 2], bufs[(m + 1) % 2], d_f_.p, (1.0f / (float)m) * pre0, ips2, m, g, stream_,
                        &launches));
    float2* w = bufs[11 % 2];
    if (it > 1) MS_TRY(pw_cmul(w, d_psi_.p, d_psim_.p, 1.0f, g, stream_, &launches));
    MS_TRY(cudaMemcpyAsync(d_psi_.p, w, sizeof(float2) * nx_ * ny_, cudaMemcpyDeviceToDevice, stream_));
    domain_ = 0;
    invalidate_graph();
    return MS_OK;
  }

  // Finite-difference step on the fused passes.  Between steps the state is
  // X (row-frequency form of psi_n, IFFT_row(X) = psi_n), the band-limited
  // spectrum FFT2(psi_n) (column-major) and psi_{n-1} in real space.
  // MultisliceStep (U.cu:2040-2083) becomes one row pass (IFFT_row, the
  // three-level stencil without its Laplacian, FFT_row) and one column pass
  // (FFT_col, + rc dz^2 4 pi^2 k^2 FFT2(psi_n), band limit, IFFT_col).
  // `Vplane`: the step's band-limited potential plane from the FD stack
  // (run_fd), or null to build it here.
  int step_fd_fused(int it, const float* Vplane = nullptr) {
    const Grid2 g{nx_, ny_};
    const long long N = (long long)nx_ * ny_;
    MS_TRY(d_fdX_.resize(N));
    MS_TRY(d_fdQ_.resize(N));
    MS_TRY(d_fdS_.resize(N));
    if (!fd_state_) {
      if (int rc = ensure_real()) return rc;
      // spectrum FFT2(psi_n) = FFT_col(FFT_row(psi_n)) stored column-major,
      // X = FFT_row(psi_n) / nx (so that IFFT_row(X) = psi_n)
      MS_TRY(pass_a(passa_args(d_psi_.p, d_t2_.p, 0), A_FWD, 1));
      MS_TRY(pass_b(passb_args(d_t2_.p, d_t1_.p, 0), B_FWD_ONLY, 1));
      MS_TRY(pw_transpose(d_t1_.p, d_fdS_.p, g, stream_, &launches));
      PassAArgs x0 = passa_args(d_psi_.p, d_fdX_.p, 0);
      x0.scale = 1.0f / (float)nx_;
      MS_TRY(pass_a(x0, A_FWD, 1));
      launches += 3;
      fd_state_ = true;
    }
    // V at the plane, band-limited (U.cu:2053-2063), real part kept
    if (!Vplane) {
      if (int rc = fd_plane_fused(it, d_f_.p)) return rc;
      Vplane = d_f_.p;
    }
    // coefficients of finiteDifferenceKernel (U.cu:1006-1012), pi = 3.14159
    const double dz = dzFD_, lam = wavel_, aa = 2.0 * 3.14159 * dz / lam, den = 1.0 + aa * aa;
    const double rcx = 1.0 / den, rcy = -aa / den;
    PassAArgs a = passa_args(d_fdX_.p, d_fdQ_.p, 0);
    a.in2 = d_psim_.p;
    a.out2 = d_psi_.p;
    a.V = Vplane;
    a.fd_rc = make_float2((float)rcx, (float)rcy);
    a.fd_ratio = make_float2((float)((1.0 - aa * aa) / den), (float)(-2.0 * aa / den));
    a.fd_kv = (float)(dz * dz * 4.0 * 3.14159 * (double)sigma2_ / lam);
    MS_TRY(pass_a(a, A_INV | A_FD | A_FWD, 1));
    PassBArgs b = passb_args(d_fdQ_.p, d_fdX_.p, 0);
    b.spec = d_fdS_.p;
    const double cf = dz * dz * 4.0 * 3.14159 * 3.14159;
    b.fd_c = make_float2((float)(rcx * cf), (float)(rcy * cf));
    b.scale = 1.0f / (float)N;
    MS_TRY(pass_b(b, B_FD, 1));
    launches += 2;
    std::swap(d_psim_.p, d_psi_.p);  // psi_n becomes psi_{n-1}
    domain_ = 2;                      // current wave held as X
    if (!capturing_) invalidate_graph();  // a single step leaves the FD run's graph stale too
    return MS_OK;
  }

  // The band-limited FD potential plane of step `it` (binnedAtomPKernelFD,
  // then BandLimitKernel in k-space, U.cu:2051-2063) on the fused passes, real
  // part into out (ny x nx floats).
  int fd_plane_fused(int it, float* out) {
    const Grid2 g{nx_, ny_};
    const long long N = (long long)nx_ * ny_;
    if (int rc = potential_slice(POT_FD, it, d_f_.p)) return rc;
    MS_TRY(pw_real_to_complex(d_f_.p, d_t1_.p, g, stream_, &launches));
    MS_TRY(pass_a(passa_args(d_t1_.p, d_t1_.p, 0), A_FWD, 1));
    PassBArgs bl = passb_args(d_t1_.p, d_t1_.p, 0);
    bl.scale = 1.0f / (float)N;
    MS_TRY(pass_b(bl, B_BANDLIMIT, 1));
    PassAArgs vr = passa_args(d_t1_.p, nullptr, 0);
    vr.out_f = out;
    MS_TRY(pass_a(vr, A_INV | A_REAL, 1));
    launches += 3;
    return MS_OK;
  }

  // ---- finite differences as a whole run ----
  // The band-limited potential planes of FD steps 1..S, kept resident like the
  // conventional stack (rebuilt when the structure, grid or FD step changes):
  // real planes for the fused passes, complex ones for the plain path (whose
  // update kernel reads complex V, as finiteDifferenceKernel U.cu:995-1023).
  int build_fd_stack(int S) {
    const bool fused = use_fused();
    if (fd_stack_valid_ && fd_nstack_ >= S && fd_stack_dz_ == dzFD_ && fd_stack_fused_ == fused) return MS_OK;
    const size_t N = (size_t)nx_ * ny_;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
        (double)N * S * (fused ? sizeof(float) : sizeof(float2)) > 0.5 * (double)free_b)
      return fail(MS_ERR_NOMEM, "the FD potential stack of " + std::to_string(S) +
                                    " planes would take more than half the free device memory");
    fd_stack_valid_ = false;
    if (fused) {
      d_fdstack_c_.release();
      MS_TRY(d_fdstack_.resize(N * S));
      for (int it = 1; it <= S; ++it)
        if (int rc = fd_plane_fused(it, d_fdstack_.p + (size_t)(it - 1) * N)) return rc;
    } else {
      d_fdstack_.release();
      MS_TRY(d_fdstack_c_.resize(N * S));
      const Grid2 g{nx_, ny_};
      const float nf = 1.0f / std::sqrt((float)(nx_ * ny_));
      for (int it = 1; it <= S; ++it) {
        float2* plane = d_fdstack_c_.p + (size_t)(it - 1) * N;
        if (int rc = potential_slice(POT_FD, it, d_f_.p)) return rc;
        MS_TRY(pw_real_to_complex(d_f_.p, d_t1_.p, g, stream_, &launches));
        MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_FORWARD));
        MS_TRY(pw_bandlimit(d_t2_.p, d_kx_.p, d_ky_.p, kmax_, nf * nf, g, stream_, &launches));
        MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, plane, CUFFT_INVERSE));
      }
    }
    MS_TRY(cudaStreamSynchronize(stream_));
    fd_nstack_ = S;
    fd_stack_dz_ = dzFD_;
    fd_stack_fused_ = fused;
    fd_stack_valid_ = true;
    return MS_OK;
  }

  // FD steps 1..S (S <= 0: the structure's FD step count) from the initial
  // waves over the resident band-limited potential stack: on the fused path
  // one captured CUDA graph (two passes per step), replayed while the stack,
  // the step count and the wave buffers stay the same; on the plain path the
  // reference's per-step launch sequence without the potential build.  Device
  // time in ms_get_last_device_ms.
  int run_fd(int nsteps, int* out_steps) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!fd_stable_) return fail(MS_ERR_NUMERIC, "no stable finite-difference step for these conditions");
    if (int rc = require_potential_inputs()) return rc;
    const int S = nsteps > 0 ? nsteps : nFD_;
    if (S < 1 || S > 100000) return fail(MS_ERR_INVALID, "need 1 <= steps <= 100000");
    if (int rc = build_fd_stack(S)) return rc;
    const size_t N = (size_t)nx_ * ny_;
    if (use_fused()) {
      if (int rc = ensure_real()) return rc;
      plan_for(1);  // tune outside the capture
      MS_TRY(d_fdX_.resize(N));
      MS_TRY(d_fdQ_.resize(N));
      MS_TRY(d_fdS_.resize(N));
      if (!fd_graph_ || fd_graph_S_ != S || fd_graph_stack_ != d_fdstack_.p || fd_graph_psi_ != d_psi_.p ||
          fd_graph_psim_ != d_psim_.p) {
        drop_fd_graph();
        float2* psi0 = d_psi_.p;
        float2* psim0 = d_psim_.p;
        fd_state_ = false;
        capturing_ = true;
        MS_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        int rc = MS_OK;
        for (int it = 1; it <= S && rc == MS_OK; ++it) rc = step_fd_fused(it, d_fdstack_.p + (size_t)(it - 1) * N);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream_, &graph);
        capturing_ = false;
        // nothing ran: the waves are still in the buffers the capture started on
        fd_graph_psi_end_ = d_psi_.p;
        fd_graph_psim_end_ = d_psim_.p;
        d_psi_.p = psi0;
        d_psim_.p = psim0;
        domain_ = 0;
        fd_state_ = false;
        if (rc != MS_OK) {
          if (graph) cudaGraphDestroy(graph);
          return rc;
        }
        if (e != cudaSuccess) return fail(MS_ERR_CUDA, std::string("FD graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&fd_graph_, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          fd_graph_ = nullptr;
          return fail(MS_ERR_CUDA, std::string("FD graph instantiate: ") + cudaGetErrorString(e));
        }
        fd_graph_S_ = S;
        fd_graph_stack_ = d_fdstack_.p;
        fd_graph_psi_ = psi0;
        fd_graph_psim_ = psim0;
      }
      MS_TRY(cudaEventRecord(ev0_, stream_));
      MS_TRY(cudaGraphLaunch(fd_graph_, stream_));
      MS_TRY(cudaEventRecord(ev1_, stream_));
      launches += 4 + 2LL * S;
      d_psi_.p = fd_graph_psi_end_;
      d_psim_.p = fd_graph_psim_end_;
      fd_state_ = true;
      domain_ = 2;
    } else {
      if (int rc = ensure_real()) return rc;
      MS_TRY(cudaEventRecord(ev0_, stream_));
      for (int it = 1; it <= S; ++it)
        if (int rc = step_fd_plain(d_fdstack_c_.p + (size_t)(it - 1) * N)) return rc;
      MS_TRY(cudaEventRecord(ev1_, stream_));
    }
    MS_TRY(cudaStreamSynchronize(stream_));
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    drop_conv_graph();  // the conventional loop's graph holds the old wave buffers
    if (out_steps) *out_steps = S;
    return MS_OK;
  }

  // One plain-path FD step on a band-limited complex potential plane: the
  // spectral Laplacian, the three-level update and the band limit of psi+
  // (U.cu:2066-2082), cuFFT plus one kernel per operation.
  int step_fd_plain(const float2* Vc) {
    const Grid2 g{nx_, ny_};
    const float nf = 1.0f / std::sqrt((float)(nx_ * ny_));
    MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_laplacian(d_t2_.p, d_kx_.p, d_ky_.p, nf * nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_grad_.p, CUFFT_INVERSE));
    MS_TRY(pw_fd_update(d_grad_.p, d_psim_.p, d_t2_.p, d_psi_.p, Vc, sigma2_, wavel_, dzFD_, g, stream_,
                        &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t1_.p, CUFFT_FORWARD));
    MS_TRY(pw_bandlimit(d_t1_.p, d_kx_.p, d_ky_.p, kmax_, nf * nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_INVERSE));
    std::swap(d_psim_.p, d_psi_.p);
    std::swap(d_psi_.p, d_t2_.p);
    domain_ = 0;
    fd_state_ = false;
    return MS_OK;
  }

  void drop_fd_graph() {
    if (fd_graph_) cudaGraphExecDestroy(fd_graph_);
    fd_graph_ = nullptr;
    fd_graph_S_ = -1;
  }

  // ---- queries ----
  int get_slices(bool conventional, int* out) {
    if (!have_atoms_) return fail(MS_ERR_STATE, "no atoms");
    if (conventional) {
      *out = (int)std::ceil((box_.MaxZ - box_.MinZ) / convdz_);  // ManagedMultislice.cpp:108
    } else {
      if (!have_calc_) return fail(MS_ERR_STATE, "calculation variables not set");
      if (!fd_stable_) return fail(MS_ERR_NUMERIC, "no stable finite-difference step for these conditions");
      *out = nFD_;
    }
    return MS_OK;
  }

  // ---- read-out ----
  int get_exit_wave(bool stem_view) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (int rc = ensure_real()) return rc;
    const size_t N = (size_t)nx_ * ny_;
    ew_.resize(N);
    if (stem_view) {
      // GetSTEMExitWave U.cu:2180-2229: centred FFT(psi)
      const Grid2 g{nx_, ny_};
      MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
      MS_TRY(pw_centre(d_t1_.p, d_t2_.p, g, stream_, &launches));
      MS_TRY(cudaMemcpyAsync(ew_.data(), d_t2_.p, N * sizeof(float2), cudaMemcpyDeviceToHost, stream_));
    } else {
      MS_TRY(cudaMemcpyAsync(ew_.data(), d_psi_.p, N * sizeof(float2), cudaMemcpyDeviceToHost, stream_));
    }
    MS_TRY(cudaStreamSynchronize(stream_));
    if (int rc = check_pass_err()) return rc;
    float mn = INFINITY, mx = -INFINITY;
    for (const float2& v : ew_) {
      const float a = std::sqrt(v.x * v.x + v.y * v.y);
      mn = std::min(mn, a);
      mx = std::max(mx, a);
    }
    ew_min_ = mn;
    ew_max_ = mx;
    have_ew_ = true;
    return MS_OK;
  }

  int free_exit_wave() {
    ew_.clear();
    ew_.shrink_to_fit();
    have_ew_ = false;
    return MS_OK;
  }

  int ew_value(int x, int y, int which, float* out) {
    if (!have_ew_) return fail(MS_ERR_STATE, "exit wave not fetched (ms_get_exit_wave)");
    if (x < 0 || y < 0 || x >= nx_ || y >= ny_) return fail(MS_ERR_INVALID, "pixel index out of range");
    const float2 v = ew_[(size_t)y * nx_ + x];
    *out = which == 0 ? std::sqrt(v.x * v.x + v.y * v.y) : which == 1 ? v.x : v.y;
    return MS_OK;
  }

  int copy_exit_wave(float* dst) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!dst) return fail(MS_ERR_INVALID, "null destination");
    if (int rc = ensure_real()) return rc;
    MS_TRY(cudaMemcpyAsync(dst, d_psi_.p, sizeof(float2) * nx_ * ny_, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return check_pass_err();
  }

  int alloc_tds() {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    MS_TRY(d_tds_.resize((size_t)nx_ * ny_));
    MS_TRY(cudaMemsetAsync(d_tds_.p, 0, sizeof(float) * nx_ * ny_, stream_));
    have_tds_ = true;
    return MS_OK;
  }

  // AddTDSWaves U.cu:2734-2766: tds += |centre(FFT(psi))|, unnormalised FFT.
  int add_tds() {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!have_tds_) return fail(MS_ERR_STATE, "TDS buffer not allocated (ms_alloc_tds)");
    if (domain_ == 2)
      if (int rc = ensure_real()) return rc;
    const Grid2 g{nx_, ny_};
    if (use_fused() && domain_ == 1) {
      PassBArgs b = passb_args(d_psi_.p, d_psi_.p, 0);
      b.acc = d_tds_.p;
      b.scale = (float)nx_;  // FFT_rows(psi) = nx * X for the row-frequency state X
      MS_TRY(pass_b(b, B_CBED, 1));
      ++launches;
    } else if (use_fused()) {
      PassAArgs a = passa_args(d_psi_.p, d_t1_.p, 0);
      MS_TRY(pass_a(a, A_FWD, 1));
      PassBArgs b = passb_args(d_t1_.p, d_t1_.p, 0);
      b.acc = d_tds_.p;
      b.scale = 1.0f;
      MS_TRY(pass_b(b, B_CBED, 1));
      launches += 2;
    } else {
      MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
      MS_TRY(pw_centre_abs_acc(d_t1_.p, d_tds_.p, 1.0f, g, stream_, &launches));
    }
    tds_host_valid_ = false;
    return MS_OK;
  }

  int tds_host() {
    if (!have_tds_) return fail(MS_ERR_STATE, "TDS buffer not allocated (ms_alloc_tds)");
    if (tds_host_valid_) return MS_OK;
    htds_.resize((size_t)nx_ * ny_);
    MS_TRY(cudaMemcpyAsync(htds_.data(), d_tds_.p, sizeof(float) * htds_.size(), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    tds_host_valid_ = true;
    return MS_OK;
  }

  int tds_query(int which, int x, int y, float* out) {
    if (int rc = tds_host()) return rc;
    if (which == 0) {
      // GetTDSMin U.cu:2768-2777
      float m = FLT_MAX_;
      for (float v : htds_) m = std::min(m, v);
      *out = m;
    } else if (which == 1) {
      // GetTDSMax U.cu:2778-2787 (starts from FLT_MIN as the reference)
      float m = 1.17549435e-38f;
      for (float v : htds_) m = std::max(m, v);
      *out = m;
    } else {
      if (x < 0 || y < 0 || x >= nx_ || y >= ny_) return fail(MS_ERR_INVALID, "pixel index out of range");
      *out = htds_[(size_t)y * nx_ + x];
    }
    return MS_OK;
  }

  int copy_tds(float* dst) {
    if (!dst) return fail(MS_ERR_INVALID, "null destination");
    if (int rc = tds_host()) return rc;
    std::memcpy(dst, htds_.data(), sizeof(float) * htds_.size());
    return MS_OK;
  }

  int alloc_host_image() {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    image_.assign((size_t)nx_ * ny_, 0.0f);
    have_image_buf_ = true;
    return MS_OK;
  }

  // SimulateImage U.cu:2311-2343: the CTF image, and with a detector model
  // (ms_set_detector) the noisy chain of U.cu:2345-2437.
  int simulate_image(float dose = 0.0f) {
    if (det_n_ > 0 && !(dose >= 0 && std::isfinite(dose))) return fail(MS_ERR_INVALID, "bad dose per pixel");
    image_noisy_ = false;
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!have_image_buf_) alloc_host_image();
    if (domain_ == 2)
      if (int rc = ensure_real()) return rc;
    const Grid2 g{nx_, ny_};
    const size_t N = (size_t)nx_ * ny_;
    const float wavel = wavel_, objap = aperture_;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    const double beta = (double)(beta_ / 1000);
    if (use_fused()) {
      PassBArgs b;
      float2* src = d_psi_.p;
      float scale = 1.0f / (float)N;
      if (domain_ == 0) {
        PassAArgs a = passa_args(d_psi_.p, d_t1_.p, 0);
        MS_TRY(pass_a(a, A_FWD, 1));
        ++launches;
        src = d_t1_.p;
      } else {
        scale = (float)nx_ / (float)N;  // FFT_rows(psi) = nx * X
      }
      b = passb_args(src, d_t2_.p, 0);
      b.ctf = CtfParams{(double)wavel, (double)Cs_, (double)df_, (double)A2_, (double)phi2_, 0.0, 0.0, beta,
                        (double)delta_, objap2};
      b.scale = scale;
      MS_TRY(pass_b(b, B_CTF, 1));
      PassAArgs a = passa_args(d_t2_.p, nullptr, 0);
      a.out_f = d_f_.p;
      a.scale = 1.0f;
      MS_TRY(pass_a(a, A_INV | A_INTENSITY, 1));
      launches += 2;
    } else {
      if (int rc = ensure_real()) return rc;
      MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
      MS_TRY(pw_ctf(d_t1_.p, d_kx_.p, d_ky_.p, wavel, Cs_, df_, A2_, phi2_, beta, delta_, objap2, 1.0f / (float)N, g,
                    stream_, &launches));
      MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_INVERSE));
      MS_TRY(pw_abs2(d_t2_.p, d_f_.p, 1.0f, g, stream_, &launches));
    }
    if (det_n_ > 0) {
      if (int rc = detector_chain(dose)) return rc;
    }
    MS_TRY(cudaMemcpyAsync(image_.data(), d_f_.p, sizeof(float) * N, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    float mn = INFINITY, mx = -INFINITY;
    for (float v : image_) {
      mn = std::min(mn, v);
      mx = std::max(mx, v);
    }
    im_min_ = mn;
    im_max_ = mx;
    have_image_ = true;
    return MS_OK;
  }

  // Float32 TIFF of a read-out (the GUI's exports, MainWindow.xaml.cs:684-890):
  // 0 image as GetImValue reads it (readout noise included with a detector
  // model), 1 / 2 exit-wave real / imaginary part (GetEWValueRe/Im, after
  // ms_get_exit_wave), 3 TDS/CBED accumulation (GetTDSVal), 4 exit-wave amplitude.
  int write_tiff(int what, const char* path) {
    if (!path) return fail(MS_ERR_INVALID, "null path");
    const size_t N = (size_t)nx_ * ny_;
    std::vector<float> buf(N);
    if (what == 0) {
      if (!have_image_) return fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
      for (int y = 0; y < ny_; ++y)
        for (int x = 0; x < nx_; ++x)
          if (int rc = im_value(x, y, &buf[(size_t)y * nx_ + x])) return rc;
    } else if (what == 1 || what == 2 || what == 4) {
      if (!have_ew_) return fail(MS_ERR_STATE, "exit wave not read out (ms_get_exit_wave)");
      for (size_t i = 0; i < N; ++i) {
        const float2 v = ew_[i];
        buf[i] = what == 1 ? v.x : what == 2 ? v.y : std::sqrt(v.x * v.x + v.y * v.y);
      }
    } else if (what == 3) {
      if (int rc = tds_host()) return rc;
      std::copy(htds_.begin(), htds_.end(), buf.begin());
    } else {
      return fail(MS_ERR_INVALID, "unknown read-out for TIFF output");
    }
    const int rc = write_tiff_f32(path, buf.data(), nx_, ny_);
    if (rc == 1) return fail(MS_ERR_INVALID, "bad TIFF arguments");
    if (rc != 0) return fail(MS_ERR_IO, std::string("cannot write ") + path);
    return MS_OK;
  }

  // CTF images of the current exit wave at n (defocus, Cs) pairs (the batch
  // Cs/df sweep the reference's GUI leaves as a stub, BP.cs:131-134): the
  // wave is transformed once and re-imaged per pair with SimulateImage's
  // transfer (imagingKernel2, U.cu:1044-1080); Cs = NULL keeps the microscope's.
  int image_series(const float* df, const float* cs, int n, float* images) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!df || !images || n < 1) return fail(MS_ERR_INVALID, "need defoci, an output buffer and n >= 1");
    for (int i = 0; i < n; ++i)
      if (!std::isfinite(df[i]) || (cs && !std::isfinite(cs[i]))) return fail(MS_ERR_INVALID, "non-finite defocus or Cs");
    if (domain_ == 2)
      if (int rc = ensure_real()) return rc;
    const Grid2 g{nx_, ny_};
    const size_t N = (size_t)nx_ * ny_;
    const float wavel = wavel_, objap = aperture_;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    const double beta = (double)(beta_ / 1000);
    MS_TRY(d_img_.resize(N * n));
    if (use_fused()) {
      const float2* src = d_psi_.p;
      float scale = (float)nx_ / (float)N;  // FFT_rows(psi) = nx X
      if (domain_ == 0) {
        MS_TRY(pass_a(passa_args(d_psi_.p, d_t1_.p, 0), A_FWD, 1));
        ++launches;
        src = d_t1_.p;
        scale = 1.0f / (float)N;
      }
      for (int i = 0; i < n; ++i) {
        PassBArgs b = passb_args(src, d_t2_.p, 0);
        b.ctf = CtfParams{(double)wavel, cs ? (double)cs[i] : (double)Cs_, (double)df[i], (double)A2_, (double)phi2_,
                          0.0, 0.0, beta, (double)delta_, objap2};
        b.scale = scale;
        MS_TRY(pass_b(b, B_CTF, 1));
        PassAArgs a = passa_args(d_t2_.p, nullptr, 0);
        a.out_f = d_img_.p + (size_t)i * N;
        MS_TRY(pass_a(a, A_INV | A_INTENSITY, 1));
        launches += 2;
      }
    } else {
      MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
      for (int i = 0; i < n; ++i) {
        MS_TRY(cudaMemcpyAsync(d_t2_.p, d_t1_.p, sizeof(float2) * N, cudaMemcpyDeviceToDevice, stream_));
        MS_TRY(pw_ctf(d_t2_.p, d_kx_.p, d_ky_.p, wavel, cs ? cs[i] : Cs_, df[i], A2_, phi2_, beta, delta_, objap2,
                      1.0f / (float)N, g, stream_, &launches));
        MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t2_.p, CUFFT_INVERSE));
        MS_TRY(pw_abs2(d_t2_.p, d_img_.p + (size_t)i * N, 1.0f, g, stream_, &launches));
      }
    }
    MS_TRY(cudaMemcpyAsync(images, d_img_.p, sizeof(float) * N * n, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return MS_OK;
  }

  int im_value(int x, int y, float* out) {
    if (!have_image_) return fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    if (x < 0 || y < 0 || x >= nx_ || y >= ny_) return fail(MS_ERR_INVALID, "pixel index out of range");
    const size_t p = (size_t)y * nx_ + x;
    if (det_n_ > 0 && image_noisy_) {
      // GetImValue (U.cu:2497-2512): readout noise offset + sigma z on the
      // detector image; z seeded per (pixel, image), so a read repeats
      const uint32_t ctr[4] = {(uint32_t)p, det_serial_ - 1, 0x4EADu, 0u};
      const uint32_t key[2] = {(uint32_t)det_seed_, (uint32_t)(det_seed_ >> 32)};
      uint32_t r[4];
      philox4x32_10(ctr, key, r);
      *out = (float)(det_ro_off_ + clipped_normal(r[0], r[1]) * det_ro_sig_ + image_[p]);
      return MS_OK;
    }
    *out = image_[p];
    return MS_OK;
  }

  // GetDQEImValue (U.cu:2514-2517): the magnitude of the simulated image at a
  // pixel, without the readout noise GetImValue adds.
  int dqe_im_value(int x, int y, float* out) {
    if (!have_image_) return fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    if (x < 0 || y < 0 || x >= nx_ || y >= ny_) return fail(MS_ERR_INVALID, "pixel index out of range");
    *out = std::fabs(image_[(size_t)y * nx_ + x]);
    return MS_OK;
  }

  // Detector model of the noisy image chain: radial DQE and NTF tables
  // (entries per binned frequency pixel), camera counts per electron, readout
  // noise, seed.  n = 0 removes it.
  int set_detector(const float* dqe, const float* ntf, int n, int binning, float conversion, float ro_off, float ro_sig,
                   uint64_t seed) {
    if (n == 0) {
      det_n_ = 0;
      return MS_OK;
    }
    if (n < 1 || n > (1 << 20) || !dqe || !ntf || binning < 1) return fail(MS_ERR_INVALID, "need tables of n >= 1 entries and binning >= 1");
    if (!std::isfinite(conversion) || !std::isfinite(ro_off) || !std::isfinite(ro_sig)) return fail(MS_ERR_INVALID, "non-finite detector constant");
    for (int i = 0; i < n; ++i)
      if (!(dqe[i] >= 0) || !std::isfinite(ntf[i])) return fail(MS_ERR_INVALID, "bad DQE/NTF table entry");
    MS_TRY(d_dqe_.resize(n));
    MS_TRY(d_ntf_.resize(n));
    MS_TRY(copy_sync(d_dqe_.p, dqe, sizeof(float) * n, cudaMemcpyHostToDevice));
    MS_TRY(copy_sync(d_ntf_.p, ntf, sizeof(float) * n, cudaMemcpyHostToDevice));
    det_n_ = n;
    det_bin_ = binning;
    det_conv_ = conversion;
    det_ro_off_ = ro_off;
    det_ro_sig_ = ro_sig;
    det_seed_ = seed;
    det_serial_ = 0;
    return MS_OK;
  }

  // The noisy chain of SimulateImage (U.cu:2345-2437) on the CTF intensity I
  // in d_f_ (FFTs by cuFFT, normalisations folded into the filters):
  //   a = |IFFT(sqrt(DQE) FFT(I)) / N|, counts = round(dose a + sqrt(dose a) z),
  //   image = |IFFT(NTF FFT(counts)) conversion^2 / N|.
  int detector_chain(float dose) {
    const Grid2 g{nx_, ny_};
    const float invN = 1.0f / ((float)nx_ * (float)ny_);
    if (!have_plan_) return fail(MS_ERR_STATE, "FFT plan not created");
    MS_TRY(pw_real_to_complex(d_f_.p, d_t1_.p, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_detector_filter(d_t2_.p, d_dqe_.p, det_n_, det_bin_, true, invN, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t1_.p, CUFFT_INVERSE));
    MS_TRY(pw_shot_noise(d_t1_.p, d_f_.p, dose, det_seed_, det_serial_, g, stream_, &launches));
    MS_TRY(pw_real_to_complex(d_f_.p, d_t1_.p, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_detector_filter(d_t2_.p, d_ntf_.p, det_n_, det_bin_, false, det_conv_ * det_conv_ * invN, g, stream_,
                              &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t2_.p, d_t1_.p, CUFFT_INVERSE));
    MS_TRY(pw_abs(d_t1_.p, d_f_.p, g, stream_, &launches));
    ++det_serial_;
    image_noisy_ = true;
    return MS_OK;
  }

  // RMS contrast over a sub-rectangle (U.cu:2453-2491 computes it over the
  // top-left 512 x 512 with cublasSasum; the rectangle is given here).
  int image_contrast(int t, int l, int b, int r, float* out) {
    if (!have_image_) return fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    if (t < 0 || l < 0 || b > ny_ || r > nx_ || t >= b || l >= r) return fail(MS_ERR_INVALID, "bad rectangle");
    double s = 0, s2 = 0;
    const double n = (double)(b - t) * (r - l);
    for (int y = t; y < b; ++y)
      for (int x = l; x < r; ++x) s += image_[(size_t)y * nx_ + x];
    const double mean = s / n;
    for (int y = t; y < b; ++y)
      for (int x = l; x < r; ++x) {
        const double d = image_[(size_t)y * nx_ + x] - mean;
        s2 += d * d;
      }
    *out = (float)std::sqrt(s2 / n);
    return MS_OK;
  }

  int copy_image(float* dst) {
    if (!have_image_) return fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    if (!dst) return fail(MS_ERR_INVALID, "null destination");
    std::memcpy(dst, image_.data(), sizeof(float) * image_.size());
    return MS_OK;
  }

  int annular(float inner, float outer, double* out) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!(inner >= 0) || !(outer > inner)) return fail(MS_ERR_INVALID, "need 0 <= inner < outer");
    if (int rc = ensure_real()) return rc;
    const Grid2 g{nx_, ny_};
    MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
    const float kin = (inner * 0.001f) / wavel_, kout = (outer * 0.001f) / wavel_;
    MS_TRY(pw_annular(d_t1_.p, d_kx_.p, d_ky_.p, kin * kin, kout * kout, 1.0 / ((double)nx_ * ny_), g, d_partial_.p,
                      d_partial_.p + 1024, stream_, &launches));
    MS_TRY(cudaMemcpyAsync(out, d_partial_.p + 1024, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return MS_OK;
  }

  // ---- STEM raster: probes `batch` at a time through the fused passes ----
  // Per probe: STEMInitialiseWavefunctions (U.cu:2672-2705, L1-normalised),
  // conventional slices 1..S, and the annular detector read from the last
  // column spectrum.  Linear in psi, so probes run unnormalised and each
  // signal is divided by its L1 norm squared at the end.
  int stem_raster(const int* px, const int* py, int n, float inner, float outer, int batch, double* signal) {
    if (!px || !py || !signal) return fail(MS_ERR_INVALID, "null buffer");
    if (!use_fused()) {
      if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
      if (n < 1) return fail(MS_ERR_INVALID, "need at least one probe position");
      if (!(inner >= 0) || !(outer > inner)) return fail(MS_ERR_INVALID, "need 0 <= inner < outer");
      if (batch > 1024) return fail(MS_ERR_INVALID, "batch must be at most 1024 (<= 0: automatic)");
      // plain path: one probe at a time through the reference sequence
      for (int i = 0; i < n; ++i) {
        if (int rc = stem_init_waves(px[i], py[i])) return rc;
        int S = 0;
        if (int rc = get_slices(true, &S)) return rc;
        for (int it = 1; it <= S; ++it)
          if (int rc = step_conventional(it)) return rc;
        if (int rc = annular(inner, outer, signal + i)) return rc;
      }
      return MS_OK;
    }
    if (int rc = raster_prepare(px, py, n, inner, outer, batch)) return rc;
    MS_TRY(cudaEventRecord(ev0_, stream_));
    if (int rc = raster_enqueue(stream_, true)) return rc;
    MS_TRY(cudaEventRecord(ev1_, stream_));
    if (int rc = raster_finish(signal)) return rc;
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    return MS_OK;
  }

  // Probe raster in three phases so that several handles can be captured into
  // one CUDA graph: prepare (stack, tables, tuning, buffers, positions: may
  // allocate and synchronise), enqueue (kernels and async device work only, on
  // `st`), finish (signals to the host).
  // Per probe: STEMInitialiseWavefunctions (U.cu:2672-2705, L1-normalised),
  // conventional slices 1..S, and the annular detector read from the last
  // column spectrum.  Linear in psi, so probes run unnormalised and each
  // signal is divided by its L1 norm squared at the end.
  int raster_prepare(const int* px, const int* py, int n, float inner, float outer, int batch) {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    if (!use_fused()) return fail(MS_ERR_UNSUPPORTED, "the enqueued raster runs on the fused passes");
    if (!px || !py) return fail(MS_ERR_INVALID, "null buffer");
    if (n < 1) return fail(MS_ERR_INVALID, "need at least one probe position");
    if (batch > 1024) return fail(MS_ERR_INVALID, "batch must be at most 1024 (<= 0: automatic)");
    if (!(inner >= 0) || !(outer > inner)) return fail(MS_ERR_INVALID, "need 0 <= inner < outer");
    if (batch <= 0) {
      if (int rc = tune_raster_batch(px[0], py[0], inner, outer, &batch)) return rc;
    }
    if (int rc = build_stack(&rs_S_)) return rc;
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    const long long N = (long long)nx_ * ny_;
    // every probe of a batch meets the same slices: their transmissions are
    // formed once (same sincos as the on-the-fly row pass) and read per probe
    if (!tstack_valid_ || tstack_S_ != rs_S_) {
      MS_TRY(d_tstack_.resize((size_t)rs_S_ * N));
      MS_TRY(pw_transmission_stack(d_stack_.p, sigma2_, d_tstack_.p, (long long)rs_S_ * N, stream_, &launches));
      tstack_valid_ = true;
      tstack_S_ = rs_S_;
    }
    rs_n_ = n;
    rs_B_ = std::min(batch, n);
    plan_for(rs_B_, true);
    MS_TRY(d_bwave_.resize((size_t)rs_B_ * N));
    MS_TRY(d_bpos_.resize(2 * (size_t)n));
    MS_TRY(d_bsig_.resize(2 * (size_t)n));
    MS_TRY(d_bpart_.resize((size_t)rs_B_ * pw_reduce_blocks(N)));
    std::vector<int> pos(2 * (size_t)n);
    std::copy(px, px + n, pos.begin());
    std::copy(py, py + n, pos.begin() + n);
    MS_TRY(copy_sync(d_bpos_.p, pos.data(), sizeof(int) * 2 * n, cudaMemcpyHostToDevice));
    const float kin = (inner * 0.001f) / wavel_, kout = (outer * 0.001f) / wavel_;
    rs_kin2_ = kin * kin;
    rs_kout2_ = kout * kout;
    return MS_OK;
  }

  // Probes per launch of the raster, tuned on the device once per grid: each
  // candidate batch (8 ... 64, at most what a quarter of the free memory
  // holds) runs one batch of probes through every slice, and the fastest per
  // probe is kept.  Batches whose waves fit in L2 (about 12 at 1024^2) keep
  // the passes' wave traffic on chip; larger ones stream it from HBM.
  int tune_raster_batch(int px0, int py0, float inner, float outer, int* out) {
    for (auto& kv : raster_batch_)
      if (kv.first == (long long)nx_ * 100000 + ny_) {
        *out = kv.second & 0xFFFF;
        rs_prefer_loop_ = (kv.second >> 16) != 0;
        return MS_OK;
      }
    size_t free_b = 0, total_b = 0;
    int cap = 64;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      const size_t per = (size_t)nx_ * ny_ * sizeof(float2);
      cap = (int)std::max<size_t>(1, std::min<size_t>(64, free_b / 4 / per));
    }
    const int cands[] = {8, 12, 16, 24, 32, 48, 64};
    int best = std::min(cap, 64);
    bool best_loop = false;
    float best_t = INFINITY;
    for (int B : cands)
      for (int lp = 0; lp < (use_batch_loop() ? 2 : 1); ++lp) {
      if (B > cap) break;
      rs_prefer_loop_ = lp == 1;  // slices in the batched persistent loop, or per pass
      std::vector<int> qx(B, px0), qy(B, py0);
      for (int rep = 0; rep < 2; ++rep) {  // the first run tunes the plans and loads the kernels
        if (int rc = raster_prepare(qx.data(), qy.data(), B, inner, outer, B)) return rc;
        MS_TRY(cudaEventRecord(ev0_, stream_));
        if (int rc = raster_enqueue(stream_, true)) return rc;
        MS_TRY(cudaEventRecord(ev1_, stream_));
        MS_TRY(cudaEventSynchronize(ev1_));
        if (rs_loop_) {
          MS_TRY(copy_sync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost));
          if (*h_loop_err_ != 0) return loop_timeout_fail();
        }
      }
      float ms = 0.0f;
      MS_TRY(cudaEventElapsedTime(&ms, ev0_, ev1_));
      const float per_probe = ms / (float)B;
      if (per_probe < best_t) {
        best_t = per_probe;
        best = B;
        best_loop = rs_prefer_loop_;
      }
      }
    rs_prefer_loop_ = best_loop;
    raster_batch_.push_back({(long long)nx_ * 100000 + ny_, best | (best_loop ? 1 << 16 : 0)});
    *out = best;
    return MS_OK;
  }

  // Probes of raster positions start .. start+nb-1 into the batch buffer (real
  // space, unnormalised) and their L1 norms (STEMInitialiseWavefunctions,
  // U.cu:2672-2705), enqueued on `st`.
  int raster_probes(cudaStream_t st, int start, int nb) {
    const long long N = (long long)nx_ * ny_;
    const int n = rs_n_;
    const Grid2 g{nx_, ny_};
    const float apert = (float)((double)aperture_ * 0.001 / (double)wavel_);
    const PlanChoice pc = plan_for(rs_B_, true);
    const int vr = pc.row, vc = pc.col;
    MS_TRY(pw_probe_batch(d_bwave_.p, N, nb, d_kx_.p, d_ky_.p, d_bpos_.p + start, d_bpos_.p + n + start, apert,
                          ps_, df_, Cs_, wavel_, g, st, &launches));
    PassBArgs bi = passb_args(d_bwave_.p, d_bwave_.p, vc);
    bi.batch_stride_wave = N;
    MS_TRY(launch_pass_b(bi, vc, B_INV_ONLY, nb, st));
    PassAArgs ai = passa_args(d_bwave_.p, d_bwave_.p, vr);
    ai.batch_stride_wave = N;
    MS_TRY(launch_pass_a(ai, vr, A_INV, nb, st));
    launches += 2;
    MS_TRY(pw_sum_abs_batch(d_bwave_.p, N, N, nb, d_bpart_.p, d_bsig_.p + n + start, st, &launches));
    return MS_OK;
  }

  // The batched persistent loop serves this handle's batches (square 256, 512
  // or 1024 grids, no forced plan, MS_OPT_SLICE_LOOP on).
  bool use_batch_loop() const {
    return use_fused() && !loop_off_ && forced_plan_ < 0 && nx_ == ny_ && batch_loop_supported(nx_, 0);
  }
  // One group of the batched loop over the raster batch at `start`: the
  // probes through the transmission stack, the detector on the last slice.
  LoopGroup raster_group(int start, int nb) {
    const long long N = (long long)nx_ * ny_;
    const int v = batch_loop_plan(nx_);
    LoopGroup g{};
    g.n = nx_;
    g.B = nb;
    g.wave = d_bwave_.p;
    g.tstack = d_tstack_.p;
    g.inst_stride = 0;
    g.slice_stride = N;
    g.a = passa_args(d_bwave_.p, d_bwave_.p, v);
    g.b = passb_args(d_bwave_.p, d_bwave_.p, v);
    g.b.kin2 = rs_kin2_;
    g.b.kout2 = rs_kout2_;
    g.b.scale = 1.0f / (float)N;
    g.sig = d_bsig_.p + start;
    return g;
  }
  // Launch of the batched loop over one or two groups (g1 may be null), with
  // this handle's barrier state (the counter cleared first; the error word is
  // cleared by the caller at the start of a sequence).
  int enqueue_batch_loop(cudaStream_t st, const LoopGroup& g0, const LoopGroup* g1, int S) {
    BatchLoopArgs L{};
    L.g[0] = g0;
    if (g1) L.g[1] = *g1;
    L.S = S;
    L.sync.count = d_loop_sync_.p;
    L.sync.error = reinterpret_cast<int*>(d_loop_sync_.p + 1);
    L.sync.limit_ns = loop_limit_ns_;
    L.sync.expect_extra = loop_extra_;
    int grid = 0;
    MS_TRY(batch_loop_prepare(g0.n, g1 ? g1->n : 0, g0.Vstack == nullptr, &grid));
    MS_TRY(cudaMemsetAsync(d_loop_sync_.p, 0, sizeof(unsigned int), st));
    MS_TRY(launch_batch_loop(L, grid, st));
    ++launches;
    return MS_OK;
  }
  int raster_tuning(int* batch, int* persistent) {
    if (!batch || !persistent) return fail(MS_ERR_INVALID, "null output");
    *batch = rs_B_;
    *persistent = rs_loop_ ? 1 : 0;
    return MS_OK;
  }
  int raster_slices() const { return rs_S_; }
  bool raster_prefers_loop() const { return rs_prefer_loop_; }
  int raster_batch() const { return rs_B_; }
  int raster_count() const { return rs_n_; }
  int grid_n() const { return nx_; }
  // Clears the raster's signal sums on `st` (its batches then run through
  // raster_probes and another handle's batched-loop launches).
  int raster_begin(cudaStream_t st) {
    MS_TRY(cudaMemsetAsync(d_bsig_.p, 0, sizeof(double) * 2 * rs_n_, st));
    rs_loop_ = false;
    return MS_OK;
  }
  int loop_begin(cudaStream_t st) {
    *h_loop_err_ = 0;
    MS_TRY(cudaMemsetAsync(d_loop_sync_.p, 0, 2 * sizeof(unsigned int), st));
    return MS_OK;
  }
  int loop_check(cudaStream_t st) {
    MS_TRY(cudaMemcpyAsync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    MS_TRY(cudaStreamSynchronize(st));
    if (*h_loop_err_ != 0) return loop_timeout_fail();
    return MS_OK;
  }

  // `allow_loop`: the slices of each batch run in the batched persistent loop
  // (one launch per batch) where it is provided; otherwise, and always when
  // several handles' rasters run as concurrent graph branches, one launch per
  // pass.
  int raster_enqueue(cudaStream_t st, bool allow_loop = false) {
    const long long N = (long long)nx_ * ny_;
    const int B = rs_B_, n = rs_n_, S = rs_S_;
    const PlanChoice pc = plan_for(B, true);
    const int vr = pc.row, vc = pc.col;
    const bool loop = allow_loop && use_batch_loop() && rs_prefer_loop_;
    MS_TRY(cudaMemsetAsync(d_bsig_.p, 0, sizeof(double) * 2 * n, st));
    if (loop) MS_TRY(cudaMemsetAsync(d_loop_sync_.p, 0, 2 * sizeof(unsigned int), st));
    rs_loop_ = loop;
    for (int start = 0; start < n; start += B) {
      const int nb = std::min(B, n - start);
      if (int rc = raster_probes(st, start, nb)) return rc;
      if (loop) {
        const LoopGroup g = raster_group(start, nb);
        if (int rc = enqueue_batch_loop(st, g, nullptr, S)) return rc;
        continue;
      }
      for (int it = 1; it <= S; ++it) {
        PassAArgs a = passa_args(d_bwave_.p, d_bwave_.p, vr);
        a.batch_stride_wave = N;
        a.batch_stride_V = 0;
        a.tr = d_tstack_.p + (size_t)(it - 1) * N;
        MS_TRY(launch_pass_a(a, vr, it == 1 ? (A_MULT_TC | A_FWD) : (A_INV | A_MULT_TC | A_FWD), nb, st));
        PassBArgs b = passb_args(d_bwave_.p, d_bwave_.p, vc);
        b.batch_stride_wave = N;
        if (it < S) {
          MS_TRY(launch_pass_b(b, vc, B_PROPAGATE, nb, st));
        } else {
          b.sig = d_bsig_.p + start;
          b.kin2 = rs_kin2_;
          b.kout2 = rs_kout2_;
          b.scale = 1.0f / (float)N;
          MS_TRY(launch_pass_b(b, vc, B_DETECT, nb, st));
        }
        launches += 2;
      }
    }
    return MS_OK;
  }

  int raster_finish(double* signal) {
    const int n = rs_n_;
    std::vector<double> host(2 * (size_t)n);
    MS_TRY(copy_sync(host.data(), d_bsig_.p, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
    if (rs_loop_) {
      MS_TRY(copy_sync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost));
      if (*h_loop_err_ != 0) return loop_timeout_fail();
    }
    for (int i = 0; i < n; ++i) {
      const double l1 = host[n + i];
      if (!(l1 > 0)) return fail(MS_ERR_NUMERIC, "probe is empty (aperture smaller than one frequency pixel)");
      signal[i] = host[i] / (l1 * l1);
    }
    return MS_OK;
  }

  cudaStream_t stream() const { return stream_; }
  bool fused() const { return use_fused(); }
  void set_last_device_ms(float ms) { last_device_ms_ = ms; }

  // z-bins of the atom index for the loaded box (U.cu:1409-1411), range-checked.
  int index_zbins(int* nz) {
    const float zext = std::ceil((box_.MaxZ - box_.MinZ) / (float)1);
    if (!std::isfinite(zext) || zext < 0.0f || (double)zext * kBins2 > (double)(INT_MAX - 1))
      return fail(MS_ERR_INVALID, "structure too deep for the atom index: " + std::to_string(zext) + " z-bins");
    *nz = (int)zext;
    *nz += (*nz == 0);
    return MS_OK;
  }

  // Potential stacks of nb frozen-phonon configurations (passes pass0 ..
  // pass0 + nb - 1, displaced as ms_upload_binned_atoms_tds): every
  // configuration binned into its own index (the same bit-exact binning),
  // then per slice one table launch and one separable-potential launch over
  // all nb (instance = blockIdx), into d_fpstack_ [config][slice][ny][nx].
  int tds_potential_batch(uint64_t seed, uint32_t pass0, int nb, float sigma, int S) {
    const int n = (int)hx_.size();
    int nz = 0;
    if (int rc = index_zbins(&nz)) return rc;
    if (nz != nzb_) return fail(MS_ERR_STATE, "atom index out of date");
    const long long nbins = (long long)nz * kBins2;
    const size_t N = (size_t)nx_ * ny_;
    std::vector<float> hx((size_t)nb * n), hy((size_t)nb * n), hz((size_t)nb * n);
    tds_displace(hx_.data(), hy_.data(), hz_.data(), n, seed, pass0, sigma, hx.data(), hy.data(), hz.data(), nb);
    MS_TRY(d_tdsx_.resize((size_t)nb * n));
    MS_TRY(d_tdsy_.resize((size_t)nb * n));
    MS_TRY(d_tdsz_.resize((size_t)nb * n));
    MS_TRY(d_tds_atoms_.resize((size_t)nb * n));
    MS_TRY(d_tds_off_.resize((size_t)nb * (nbins + 1)));
    // (copies from pageable memory return once the data is staged, so the
    // host vectors may go out of scope when this returns)
    MS_TRY(cudaMemcpyAsync(d_tdsx_.p, hx.data(), sizeof(float) * hx.size(), cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemcpyAsync(d_tdsy_.p, hy.data(), sizeof(float) * hy.size(), cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemcpyAsync(d_tdsz_.p, hz.data(), sizeof(float) * hz.size(), cudaMemcpyHostToDevice, stream_));
    BinScratch scr{d_key_.p, d_idx_.p, d_cursor_.p, d_blocksum_.p};
    for (int k = 0; k < nb; ++k) {
      AtomIndex idx{d_tds_atoms_.p + (size_t)k * n, d_tds_off_.p + (size_t)k * (nbins + 1), 0, 0};
      MS_TRY(build_atom_index(d_Zin_.p, d_tdsx_.p + (size_t)k * n, d_tdsy_.p + (size_t)k * n,
                              d_tdsz_.p + (size_t)k * n, n, box_, nz, idx, scr, stream_));
      launches += 8;
    }
    return separable_stack(S, d_fpstack_.p, N, nb, d_tds_atoms_.p, d_tds_off_.p, n, nbins + 1);
  }

  // ---- frozen-phonon series (the GUI's pass loop, MainWindow.xaml.cs:353-402) ----
  // Configurations first_pass .. first_pass + nconf - 1, each displaced as
  // ms_upload_binned_atoms_tds(seed, pass, sigma), through conventional slices
  // 1..S from the initial wave.  diff = sum over configurations of
  // |centre(FFT(psi_exit))| (AddTDSWaves, U.cu:2734-2766), image = mean of the
  // deterministic CTF images (SimulateImage).  Fused path: `batch`
  // configurations share every pass launch (instance = blockIdx.y, each with its
  // own potential stack); plain path: one configuration at a time through the
  // reference's launch sequence.  The handle's atom index is left at the last
  // configuration.
  int frozen_phonon(uint64_t seed, uint32_t first_pass, int nconf, float sigma, int batch, float* diff, float* image) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (stem_) return fail(MS_ERR_UNSUPPORTED, "the frozen-phonon series runs in TEM mode");
    if (nconf < 1 || batch < 1 || batch > 256) return fail(MS_ERR_INVALID, "need nconf >= 1 and batch 1..256");
    if (!(sigma >= 0) || !std::isfinite(sigma)) return fail(MS_ERR_INVALID, "bad thermal displacement sigma");
    if (int rc = require_potential_inputs()) return rc;
    int S = 0;
    if (int rc = get_slices(true, &S)) return rc;
    if (S < 1) return fail(MS_ERR_INVALID, "structure has no slices");
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    const long long N = (long long)nx_ * ny_;
    const Grid2 g{nx_, ny_};
    const float wavel = wavel_, objap = aperture_;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    const CtfParams ctf{(double)wavel, (double)Cs_, (double)df_, (double)A2_, (double)phi2_, 0.0, 0.0,
                        (double)(beta_ / 1000), (double)delta_, objap2};
    const int kind = pot_mode_ == 1 ? POT_PROJECTED : POT_CONVENTIONAL;
    const bool fused = use_fused();
    const int B = fused ? std::min(batch, nconf) : 1;
    MS_TRY(d_fpdiff_.resize(N));
    MS_TRY(d_fpsum_.resize(N));
    MS_TRY(d_fpimg_.resize((size_t)B * N));
    MS_TRY(cudaMemsetAsync(d_fpdiff_.p, 0, sizeof(float) * N, stream_));
    MS_TRY(cudaMemsetAsync(d_fpsum_.p, 0, sizeof(float) * N, stream_));
    if (fused) {
      MS_TRY(d_fpstack_.resize((size_t)B * S * N));
      MS_TRY(d_bwave_.resize((size_t)B * N));
      plan_for(B);
    }
    invalidate_graph();
    bool fp_loop = false;
    // the fused path bins every configuration of a batch into its own index
    // and builds their potentials slice by slice in one launch each
    // (separable kernel); the handle's index is the last configuration's
    // afterwards, as one upload at a time leaves it
    const bool batch_pot = fused && kind == POT_CONVENTIONAL && separable_ok();
    if (batch_pot && pot_tile_ < 0)
      if (int rc = tune_pot_tile()) return rc;
    MS_TRY(cudaEventRecord(ev0_, stream_));
    for (int start = 0; start < nconf; start += B) {
      const int nb = std::min(B, nconf - start);
      if (!fused) {
        if (int rc = upload_binned(true, seed, first_pass + (uint32_t)start, sigma)) return rc;
        for (int it = 1; it <= S; ++it)
          if (int rc = step_conventional(it)) return rc;
        MS_TRY_FFT(cufftExecC2C(plan_, d_psi_.p, d_t1_.p, CUFFT_FORWARD));
        if (diff) MS_TRY(pw_centre_abs_acc(d_t1_.p, d_fpdiff_.p, 1.0f, g, stream_, &launches));
        if (image) {
          MS_TRY(pw_ctf(d_t1_.p, d_kx_.p, d_ky_.p, wavel, Cs_, df_, A2_, phi2_, (double)(beta_ / 1000), delta_,
                        objap2, 1.0f / (float)N, g, stream_, &launches));
          MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_INVERSE));
          MS_TRY(pw_abs2(d_t2_.p, d_fpimg_.p, 1.0f, g, stream_, &launches));
          MS_TRY(pw_add_batch(d_fpimg_.p, N, 1, d_fpsum_.p, 1.0f / (float)nconf, g, stream_, &launches));
        }
        continue;
      }
      // potential stacks of the nb configurations: [config][slice][ny][nx]
      if (batch_pot) {
        if (int rc = tds_potential_batch(seed, first_pass + (uint32_t)start, nb, sigma, S)) return rc;
      } else {
        for (int k = 0; k < nb; ++k) {
          if (int rc = upload_binned(true, seed, first_pass + (uint32_t)(start + k), sigma)) return rc;
          for (int it = 1; it <= S; ++it)
            if (int rc = potential_slice(kind, it, d_fpstack_.p + ((size_t)k * S + (it - 1)) * N)) return rc;
        }
      }
      for (int k = 0; k < nb; ++k)
        MS_TRY(cudaMemcpyAsync(d_bwave_.p + (size_t)k * N, d_psi0_.p, sizeof(float2) * N, cudaMemcpyDeviceToDevice,
                               stream_));
      if (use_batch_loop()) {
        // the nb configurations through every slice in one persistent launch
        const int v = batch_loop_plan(nx_);
        LoopGroup lg{};
        lg.n = nx_;
        lg.B = nb;
        lg.wave = d_bwave_.p;
        lg.Vstack = d_fpstack_.p;
        lg.inst_stride = (long long)S * N;
        lg.slice_stride = N;
        lg.a = passa_args(d_bwave_.p, d_bwave_.p, v);
        lg.b = passb_args(d_bwave_.p, d_bwave_.p, v);
        if (start == 0) MS_TRY(cudaMemsetAsync(d_loop_sync_.p, 0, 2 * sizeof(unsigned int), stream_));
        if (int rc = enqueue_batch_loop(stream_, lg, nullptr, S)) return rc;
        fp_loop = true;
      } else {
        for (int it = 1; it <= S; ++it) {
          PassAArgs a = passa_args(d_bwave_.p, d_bwave_.p, 0);
          a.batch_stride_wave = N;
          a.batch_stride_V = (long long)S * N;
          a.V = d_fpstack_.p + (size_t)(it - 1) * N;
          MS_TRY(pass_a(a, it == 1 ? (A_MULT_T | A_FWD) : (A_INV | A_MULT_T | A_FWD), nb));
          PassBArgs b = passb_args(d_bwave_.p, d_bwave_.p, 0);
          b.batch_stride_wave = N;
          MS_TRY(pass_b(b, B_PROPAGATE, nb));
          launches += 2;
        }
      }
      if (diff) {
        PassBArgs b = passb_args(d_bwave_.p, d_bwave_.p, 0);
        b.batch_stride_wave = N;
        b.acc = d_fpdiff_.p;
        b.scale = (float)nx_;  // FFT2(psi) = nx FFT_col(X)
        MS_TRY(pass_b(b, B_CBED, nb));
        ++launches;
      }
      if (image) {
        PassBArgs b = passb_args(d_bwave_.p, d_bwave_.p, 0);
        b.batch_stride_wave = N;
        b.ctf = ctf;
        b.scale = (float)nx_ / (float)N;
        MS_TRY(pass_b(b, B_CTF, nb));
        PassAArgs a = passa_args(d_bwave_.p, nullptr, 0);
        a.batch_stride_wave = N;
        a.out_f = d_fpimg_.p;
        MS_TRY(pass_a(a, A_INV | A_INTENSITY, nb));
        MS_TRY(pw_add_batch(d_fpimg_.p, N, nb, d_fpsum_.p, 1.0f / (float)nconf, g, stream_, &launches));
        launches += 2;
      }
    }
    MS_TRY(cudaEventRecord(ev1_, stream_));
    if (batch_pot)
      if (int rc = upload_binned(true, seed, first_pass + (uint32_t)(nconf - 1), sigma)) return rc;
    if (diff) MS_TRY(cudaMemcpyAsync(diff, d_fpdiff_.p, sizeof(float) * N, cudaMemcpyDeviceToHost, stream_));
    if (image) MS_TRY(cudaMemcpyAsync(image, d_fpsum_.p, sizeof(float) * N, cudaMemcpyDeviceToHost, stream_));
    if (fp_loop)
      MS_TRY(cudaMemcpyAsync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    if (fp_loop && *h_loop_err_ != 0) return loop_timeout_fail();
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    return MS_OK;
  }

  // ---- whole-run entry points ----
  int build_stack(int* nslices) {
    if (int rc = require_potential_inputs()) return rc;
    int S = 0;
    if (int rc = get_slices(true, &S)) return rc;
    if (S < 1) return fail(MS_ERR_INVALID, "structure has no slices");
    if (!stack_valid_ || nstack_ != S) {
      const size_t N = (size_t)nx_ * ny_;
      MS_TRY(d_stack_.resize(N * S));
      const int kind = pot_mode_ == 1 ? POT_PROJECTED : POT_CONVENTIONAL;
      if (kind == POT_CONVENTIONAL && pot_tile_ < 0 && !capturing_)
        if (int rc = tune_pot_tile()) return rc;
      // device time of the stack (ms_get_last_device_ms)
      MS_TRY(cudaEventRecord(ev0_, stream_));
      if (kind == POT_CONVENTIONAL && separable_ok()) {
        if (int rc = separable_stack(S, d_stack_.p, N, 1)) return rc;
      } else {
        for (int it = 1; it <= S; ++it)
          if (int rc = potential_slice(kind, it, d_stack_.p + (it - 1) * N)) return rc;
      }
      MS_TRY(cudaEventRecord(ev1_, stream_));
      MS_TRY(cudaStreamSynchronize(stream_));
      MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
      nstack_ = S;
      stack_valid_ = true;
      tstack_valid_ = false;
      // the slice-loop graph reads the stack at replay: it stays valid while
      // the stack keeps its allocation (checked in run_conventional)
    }
    if (nslices) *nslices = S;
    return MS_OK;
  }

  // A whole conventional run whose potential stack must first be built:
  // slice i's transmission and propagation (the fused passes, on the pass
  // stream) run while the potentials of the next slices are built (on the
  // handle's stream, tables on the side stream); the stack is kept for later
  // runs, which replay the persistent loop.  Device time of the whole, build
  // included, in last_device_ms_.
  int run_conventional_streamed(int S, int* nslices) {
    if (int rc = require_potential_inputs()) return rc;
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    plan_for(1);  // (tuning synchronises: before the streams fork)
    if (pot_tile_ < 0)
      if (int rc = tune_pot_tile()) return rc;
    const size_t N = (size_t)nx_ * ny_;
    MS_TRY(d_stack_.resize(N * S));
    MS_TRY(cudaEventRecord(ev0_, stream_));
    MS_TRY(cudaEventRecord(ev_fork2_, stream_));
    MS_TRY(cudaStreamWaitEvent(pass_, ev_fork2_, 0));
    int rc = separable_stack(S, d_stack_.p, N, 1, nullptr, nullptr, 0, 0, [&](int it, cudaEvent_t done) -> int {
      MS_TRY(cudaStreamWaitEvent(pass_, done, 0));
      launches += 2;
      return enqueue_fused_step(d_stack_.p + (size_t)(it - 1) * N, it == 1, pass_);
    });
    // join the pass stream (also on failure, so that the handle's stream
    // orders after everything enqueued)
    MS_TRY(cudaEventRecord(ev_join_, pass_));
    MS_TRY(cudaStreamWaitEvent(stream_, ev_join_, 0));
    if (rc != MS_OK) return rc;
    MS_TRY(cudaEventRecord(ev1_, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    if (int rc2 = check_pass_err()) return rc2;
    nstack_ = S;
    stack_valid_ = true;
    tstack_valid_ = false;
    domain_ = 1;
    if (nslices) *nslices = S;
    return MS_OK;
  }

  int run_conventional(int* nslices) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    int S = 0;
    if (use_fused() && pot_mode_ == 0 && overlap_build_ && have_index_ && have_fp_ && have_freq_) {
      if (int rc = get_slices(true, &S)) return rc;
      if (S >= 1 && (!stack_valid_ || nstack_ != S) && separable_ok()) return run_conventional_streamed(S, nslices);
    }
    if (int rc = build_stack(&S)) return rc;
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    const bool loop = use_loop();
    if (use_fused()) {
      if (loop) {
        if (int rc = prepare_loop(S)) return rc;
      } else {
        plan_for(1);  // tune outside the capture (tuning allocates and synchronises)
      }
      if (!graph_exec_ || graph_S_ != S || graph_stack_ != d_stack_.p) {
        invalidate_graph();
        MS_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        int rc = MS_OK;
        if (loop) {
          // the whole slice loop: one cooperative launch, its barrier state
          // cleared before it and its error word read back after it
          rc = enqueue_loop(d_stack_.p, S, true);
          if (rc == MS_OK && cudaMemcpyAsync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int),
                                             cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
            rc = fail(MS_ERR_CUDA, "loop error read-back");
        } else {
          for (int it = 1; it <= S && rc == MS_OK; ++it)
            rc = enqueue_fused_step(d_stack_.p + (size_t)(it - 1) * nx_ * ny_, it == 1);
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream_, &graph);
        if (rc != MS_OK) {
          if (graph) cudaGraphDestroy(graph);
          return rc;
        }
        if (e != cudaSuccess) return fail(MS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&graph_exec_, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          graph_exec_ = nullptr;
          return fail(MS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        graph_S_ = S;
        graph_stack_ = d_stack_.p;
      }
      *h_loop_err_ = 0;
      MS_TRY(cudaEventRecord(ev0_, stream_));
      MS_TRY(cudaGraphLaunch(graph_exec_, stream_));
      launches += loop ? 1 : 2LL * S;
      domain_ = 1;
    } else {
      MS_TRY(cudaEventRecord(ev0_, stream_));
      for (int it = 1; it <= S; ++it)
        if (int rc = transmit_propagate(d_stack_.p + (size_t)(it - 1) * nx_ * ny_, it == 1)) return rc;
    }
    MS_TRY(cudaEventRecord(ev1_, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    if (loop && use_fused() && *h_loop_err_ != 0) return loop_timeout_fail();
    if (!loop && use_fused())
      if (int rc = check_pass_err()) return rc;
    if (nslices) *nslices = S;
    return MS_OK;
  }

  // The persistent slice loop runs the conventional loop where it is provided
  // (square 256, 512, 1024 grids), unless MS_OPT_SLICE_LOOP turns it off or an
  // FFT plan variant is forced (MS_OPT_FFT_PLAN selects per-pass kernels).
  bool use_loop() const {
    return use_fused() && !loop_off_ && forced_plan_ < 0 && slice_loop_supported(nx_, ny_);
  }
  // Chooses the loop kernel variant for this grid (forced by
  // MS_OPT_LOOP_VARIANT, else tuned once: every variant runs a short loop of
  // up to 16 slices over the resident stack, three times after two warm-up
  // launches, and the fastest is kept).  Needs the potential stack; outside
  // stream capture (it synchronises).
  int prepare_loop(int S) {
    if (loop_grid_ > 0 && loop_grid_n_ == nx_ && loop_tuned_for_ == forced_loop_) return MS_OK;
    int best_v = -1, best_grid = 0;
    float best_t = INFINITY;
    const int St = std::min(S, 16);
    for (int v = 0; v < slice_loop_variants(); ++v) {
      if (forced_loop_ >= 0 && v != forced_loop_) continue;
      int grid = 0;
      if (slice_loop_prepare(nx_, v, &grid) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      if (forced_loop_ >= 0) {
        best_v = v;
        best_grid = grid;
        break;
      }
      loop_v_ = v;
      loop_grid_ = grid;
      for (int k = 0; k < 2; ++k)
        if (int rc = enqueue_loop(d_stack_.p, St, k == 0)) return rc;
      MS_TRY(cudaEventRecord(ev0_, stream_));
      for (int k = 0; k < 3; ++k)
        if (int rc = enqueue_loop(d_stack_.p, St, false)) return rc;
      MS_TRY(cudaEventRecord(ev1_, stream_));
      MS_TRY(cudaMemcpyAsync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream_));
      MS_TRY(cudaStreamSynchronize(stream_));
      launches += 5;
      if (*h_loop_err_ != 0) return loop_timeout_fail();
      float ms = 0.0f;
      MS_TRY(cudaEventElapsedTime(&ms, ev0_, ev1_));
      if (ms < best_t) {
        best_t = ms;
        best_v = v;
        best_grid = grid;
      }
    }
    if (best_v < 0) return fail(MS_ERR_CUDA, "no persistent slice-loop variant could be prepared on this device");
    loop_v_ = best_v;
    loop_grid_ = best_grid;
    loop_grid_n_ = nx_;
    loop_tuned_for_ = forced_loop_;
    domain_ = 0;  // tuning left scratch in the wave; every run starts from psi0
    return MS_OK;
  }
  int potential_sum_info(int* last, int* next) {
    if (last) *last = last_pot_sum_;
    if (next) *next = separable_ok() ? 2 : 1;
    return MS_OK;
  }

  int slice_loop_info(int* variant, int* columns, int* grid) {
    if (!variant || !columns || !grid) return fail(MS_ERR_INVALID, "null output");
    if (!use_loop()) {
      *variant = -1;
      *columns = 0;
      *grid = 0;
      return MS_OK;
    }
    int S = 0;
    if (int rc = build_stack(&S)) return rc;
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    if (int rc = prepare_loop(S)) return rc;
    *variant = loop_v_;
    *columns = slice_loop_columns(loop_v_);
    *grid = loop_grid_;
    return MS_OK;
  }
  LoopArgs loop_args(const float* Vstack, int S) {
    const int v = slice_loop_plan(nx_, loop_v_);
    LoopArgs L{};
    L.a = passa_args(d_psi0_.p, d_psi_.p, v);
    L.b = passb_args(d_psi_.p, d_psi_.p, v);
    L.psi0 = d_psi0_.p;
    L.wave = d_psi_.p;
    L.Vstack = Vstack;
    L.vstride = (long long)nx_ * ny_;
    L.S = S;
    L.sync.count = d_loop_sync_.p;
    L.sync.error = reinterpret_cast<int*>(d_loop_sync_.p + 1);
    L.sync.limit_ns = loop_limit_ns_;
    L.sync.expect_extra = loop_extra_;
    return L;
  }
  // Enqueues the slice loop over S slices of Vstack (no host sync, no
  // allocation): the arrival counter is cleared first, and the error word too
  // when `clear_error` (the first launch of a sequence).
  int enqueue_loop(const float* Vstack, int S, bool clear_error) {
    fd_state_ = false;
    MS_TRY(cudaMemsetAsync(d_loop_sync_.p, 0, (clear_error ? 2 : 1) * sizeof(unsigned int), stream_));
    MS_TRY(launch_slice_loop(loop_args(Vstack, S), loop_v_, loop_grid_, stream_));
    domain_ = 1;
    return MS_OK;
  }
  int loop_timeout_fail() {
    domain_ = 0;
    have_waves_ = false;
    return fail(MS_ERR_CUDA,
                "persistent slice loop: a grid-barrier wait ran out (MS_OPT_LOOP_WAIT_US); the wave is undefined, "
                "initialise the wavefunctions again");
  }

  int time_slices(int steps, int reps, float* total_ms, float* row_ms, float* col_ms) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (steps < 1 || reps < 1 || steps > 100000) return fail(MS_ERR_INVALID, "need 1 <= steps <= 100000, reps >= 1");
    int S = 0;
    if (int rc = build_stack(&S)) return rc;
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    const size_t N = (size_t)nx_ * ny_;
    const bool loop = use_loop() && steps <= S;
    if (loop) {
      if (int rc = prepare_loop(S)) return rc;
    }
    MS_TRY(cudaStreamSynchronize(stream_));
    // whole steps, back to back (the persistent loop: one launch per repetition)
    *h_loop_err_ = 0;
    MS_TRY(cudaEventRecord(ev0_, stream_));
    for (int r = 0; r < reps; ++r) {
      if (loop) {
        if (int rc = enqueue_loop(d_stack_.p, steps, r == 0)) return rc;
        ++launches;
      } else {
        for (int k = 0; k < steps; ++k)
          if (int rc = transmit_propagate(d_stack_.p + (size_t)(k % S) * N, k == 0)) return rc;
      }
    }
    MS_TRY(cudaEventRecord(ev1_, stream_));
    if (loop)
      MS_TRY(cudaMemcpyAsync(h_loop_err_, d_loop_sync_.p + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    if (loop && *h_loop_err_ != 0) return loop_timeout_fail();
    if (int rc = check_pass_err()) return rc;
    MS_TRY(cudaEventElapsedTime(total_ms, ev0_, ev1_));
    if (!row_ms || !col_ms) return MS_OK;  // no per-pass breakdown requested
    *row_ms = *col_ms = 0.0f;
    if (loop) return MS_OK;  // one launch per repetition: no per-pass split
    if (use_fused()) {
      // the same sequence with an event between every pass: per-launch averages
      std::vector<cudaEvent_t> ev(2 * steps + 1, nullptr);
      int rc = MS_OK;
      for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = fail(MS_ERR_CUDA, "cudaEventCreate failed");
      if (rc == MS_OK) {
        cudaEventRecord(ev[0], stream_);
        for (int k = 0; k < steps && rc == MS_OK; ++k) {
          PassAArgs a = passa_args(k == 0 ? d_psi0_.p : d_psi_.p, d_psi_.p, 0);
          a.V = d_stack_.p + (size_t)(k % S) * N;
          cudaError_t e1 = pass_a(a, k == 0 ? (A_MULT_T | A_FWD) : (A_INV | A_MULT_T | A_FWD), 1);
          cudaEventRecord(ev[2 * k + 1], stream_);
          cudaError_t e2 = pass_b(passb_args(d_psi_.p, d_psi_.p, 0), B_PROPAGATE, 1);
          cudaEventRecord(ev[2 * k + 2], stream_);
          if (e1 != cudaSuccess || e2 != cudaSuccess) rc = cuda_fail(e1 != cudaSuccess ? e1 : e2, "timed pass launch");
        }
        launches += 2LL * steps;
        domain_ = 1;
        if (cudaEventSynchronize(ev[2 * steps]) != cudaSuccess && rc == MS_OK) rc = fail(MS_ERR_CUDA, "event sync");
        double ta = 0, tb = 0;
        for (int k = 0; k < steps && rc == MS_OK; ++k) {
          float m1 = 0, m2 = 0;
          cudaEventElapsedTime(&m1, ev[2 * k], ev[2 * k + 1]);
          cudaEventElapsedTime(&m2, ev[2 * k + 1], ev[2 * k + 2]);
          ta += m1;
          tb += m2;
        }
        *row_ms = (float)(ta / steps);
        *col_ms = (float)(tb / steps);
      }
      for (auto& e : ev)
        if (e) cudaEventDestroy(e);
      if (rc != MS_OK) return rc;
      if (int rc2 = check_pass_err()) return rc2;
    }
    return MS_OK;
  }

  int fft2_host(const float* in, float* out, int nx, int ny, int sign) {
    if (!fused_supported(nx, ny)) return fail(MS_ERR_UNSUPPORTED, "grid not supported by the fused FFT passes");
    const size_t N = (size_t)nx * ny;
    const int v = forced_plan_ >= 0 ? forced_plan_ : 0;
    DevBuf<float2> buf, tw1, tw2;
    MS_TRY(buf.resize(N));
    std::vector<float2> tw(2 * (size_t)std::max(nx, ny));
    const int sx = make_twiddles(nx, v, tw.data());
    MS_TRY(tw1.resize(std::max(sx, 1)));
    MS_TRY(copy_sync(tw1.p, tw.data(), sizeof(float2) * sx, cudaMemcpyHostToDevice));
    const int sy = make_twiddles(ny, v, tw.data());
    MS_TRY(tw2.resize(std::max(sy, 1)));
    MS_TRY(copy_sync(tw2.p, tw.data(), sizeof(float2) * sy, cudaMemcpyHostToDevice));
    MS_TRY(copy_sync(buf.p, in, sizeof(float2) * N, cudaMemcpyHostToDevice));
    PassAArgs a{};
    a.in = buf.p; a.out = buf.p; a.tw = tw1.p; a.nx = nx; a.ny = ny; a.scale = 1.0f;
    PassBArgs b{};
    b.in = buf.p; b.out = buf.p; b.tw = tw2.p; b.nx = nx; b.ny = ny; b.scale = 1.0f;
    MS_TRY(launch_pass_a(a, v, sign < 0 ? A_FWD : A_INV, 1, stream_));
    MS_TRY(launch_pass_b(b, v, sign < 0 ? B_FWD_ONLY : B_INV_ONLY, 1, stream_));
    launches += 2;
    MS_TRY(cudaMemcpyAsync(out, buf.p, sizeof(float2) * N, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return MS_OK;
  }

  // ---- differentiable focal series (no reference counterpart) ----
  // L = sum_d sum_p (I_d - T_d)^2 with I_d = |B_d psi_S|^2, psi_S the wave
  // after conventional slices 1..S of the potential stack from the initial
  // wave and B_d the coherent transfer of SimulateImage (U.cu:2311-2343) at
  // defocus d.  The adjoint runs the slices backwards with the conjugated
  // propagator and transmission:
  //   g_S = sum_d B_d^H [2 (I_d - T_d) B_d psi_S],   h = A^H g_n,
  //   dL/dV_n = -2 sigma Im(conj(h) t_n psi_{n-1}),  g_{n-1} = conj(t_n) h,
  // and through the potential build to the atoms' x, y.  The waves psi_{n-1}
  // are recomputed segment by segment from checkpoints every K slices
  // (K = ceil(sqrt(S)) unless MS_OPT_CHECKPOINT sets it; K >= S keeps one
  // segment, K = 1 stores every wave in the forward sweep).
  // All waves are held in the fused passes' row-frequency form X with
  // IFFT_row(X) = field; the adjoint state g uses the same form.
  int focal(const float* defoci, int nd, const float* targets, int S, double* loss, float* images, float* dLdV,
            double* dLdxy, bool grad) {
    if (!have_waves_) return fail(MS_ERR_STATE, "wavefunctions not initialised");
    if (!defoci || !targets || !loss || nd < 1) return fail(MS_ERR_INVALID, "need defoci, targets, loss and nd >= 1");
    for (int d = 0; d < nd; ++d)
      if (!std::isfinite(defoci[d])) return fail(MS_ERR_INVALID, "non-finite defocus");
    if (!use_fused()) return fail(MS_ERR_UNSUPPORTED, "the focal series runs on the fused passes (grid 64..4096, powers of two)");
    if (stem_) return fail(MS_ERR_UNSUPPORTED, "the focal series needs TEM calculation variables");
    if (int rc = require_potential_inputs()) return rc;
    int Sall = 0;
    if (int rc = get_slices(true, &Sall)) return rc;
    if (S < 1 || S > Sall) return fail(MS_ERR_INVALID, "slice count must be 1..ms_get_slices(conventional)");
    if (dLdxy && pot_mode_ != 0)
      return fail(MS_ERR_UNSUPPORTED, "atom gradients need the conventional potential (MS_OPT_POTENTIAL 0)");
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    plan_for(1);
    const size_t N = (size_t)nx_ * ny_;
    int K = S;
    if (grad) K = ckpt_ > 0 ? std::min(ckpt_, S) : auto_checkpoint_stride(S, (size_t)nx_ * ny_);
    const int nck = (S + K - 1) / K;
    MS_TRY(d_T_.resize(N * nd));
    MS_TRY(d_Phi_.resize(N));
    MS_TRY(d_loss_.resize(1));
    if (images) MS_TRY(d_img_.resize(N * nd));
    if (grad) {
      MS_TRY(d_G_.resize(N));
      MS_TRY(d_U_.resize(N));
      MS_TRY(d_ck_.resize(N * std::max(nck - 1, 1)));
      MS_TRY(d_seg_.resize(N * K));
      MS_TRY(d_dV_.resize(dLdV ? N * S : 2 * N));
      if (dLdxy) {
        MS_TRY(d_dxy_.resize(2 * (size_t)natoms_));
        if (int rc = zbin_starts()) return rc;
      }
    }
    invalidate_graph();  // the sweep below leaves d_psi_ at psi_S
    MS_TRY(cudaMemcpyAsync(d_T_.p, targets, sizeof(float) * N * nd, cudaMemcpyHostToDevice, stream_));
    MS_TRY(cudaMemsetAsync(d_loss_.p, 0, sizeof(double), stream_));
    // (after any atom-position adjoint still on the second pixel stream, which
    // an earlier call that failed part-way may have left unjoined)
    MS_TRY(cudaEventRecord(ev_join_, pix_[1]));
    MS_TRY(cudaStreamWaitEvent(stream_, ev_join_, 0));
    if (grad && dLdxy) MS_TRY(cudaMemsetAsync(d_dxy_.p, 0, sizeof(double) * 2 * natoms_, stream_));
    // timed from here: the potential stack (when the atoms changed), the sweeps
    MS_TRY(cudaEventRecord(ev0_, stream_));
    if (int rc = build_stack(&Sall)) return rc;
    // forward sweep; checkpoint c (c = 1..nck-1) holds X_{cK}; the waves of
    // the last segment (psi_{clast} .. psi_{S-1}) are kept as they pass
    const int clast = ((S - 1) / K) * K;
    for (int n = 1; n <= S; ++n) {
      if (grad && n > 1 && (n - 1) % K == 0)
        MS_TRY(cudaMemcpyAsync(d_ck_.p + (size_t)((n - 1) / K - 1) * N, d_psi_.p, sizeof(float2) * N,
                               cudaMemcpyDeviceToDevice, stream_));
      if (grad && n - 1 >= clast) {
        PassAArgs a = passa_args(n == 1 ? d_psi0_.p : d_psi_.p, d_psi_.p, 0);
        a.V = d_stack_.p + (size_t)(n - 1) * N;
        a.out2 = d_seg_.p + (size_t)(n - 1 - clast) * N;
        MS_TRY(pass_a(a, n == 1 ? (A_SAVE | A_MULT_T | A_FWD) : (A_INV | A_SAVE | A_MULT_T | A_FWD), 1));
        MS_TRY(pass_b(passb_args(d_psi_.p, d_psi_.p, 0), B_PROPAGATE, 1));
        domain_ = 1;
      } else if (int rc = enqueue_fused_step(d_stack_.p + (size_t)(n - 1) * N, n == 1)) {
        return rc;
      }
      launches += 2;
    }
    // images, loss and the adjoint seed
    const float wavel = wavel_, objap = aperture_;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    for (int d = 0; d < nd; ++d) {
      PassBArgs b = passb_args(d_psi_.p, d_Phi_.p, 0);
      b.ctf = CtfParams{(double)wavel, (double)Cs_, (double)defoci[d], (double)A2_, (double)phi2_, 0.0, 0.0,
                        (double)(beta_ / 1000), (double)delta_, objap2};
      b.scale = (float)nx_ / (float)N;  // FFT_rows(psi) = nx X
      MS_TRY(pass_b(b, B_CTF, 1));
      PassAArgs a = passa_args(d_Phi_.p, grad ? d_U_.p : nullptr, 0);
      a.T = d_T_.p + (size_t)d * N;
      a.loss = d_loss_.p;
      a.out_f = images ? d_img_.p + (size_t)d * N : nullptr;
      MS_TRY(pass_a(a, grad ? (A_INV | A_RESID | A_FWD) : (A_INV | A_RESID), 1));
      launches += 2;
      if (grad) {
        b.in = d_U_.p;
        b.out = d_G_.p;
        b.scale = 1.0f / (float)N;
        b.accumulate = d > 0;
        MS_TRY(pass_b(b, B_CTF_ADJ, 1));
        ++launches;
      }
    }
    if (grad) {
      for (int c = clast; c >= 0; c -= K) {
        const int e = std::min(c + K, S);
        // psi_c .. psi_{e-1} (real space) into segment slots 0 .. e-1-c
        // (the last segment's are there from the forward sweep)
        const float2* src = c == 0 ? d_psi0_.p : d_ck_.p + (size_t)(c / K - 1) * N;
        const float2* cur = src;
        for (int n = c + 1; n <= e - 1 && c != clast; ++n) {
          PassAArgs a = passa_args(cur, d_t1_.p, 0);
          a.V = d_stack_.p + (size_t)(n - 1) * N;
          a.out2 = d_seg_.p + (size_t)(n - 1 - c) * N;
          const bool real_in = (n == 1);
          MS_TRY(pass_a(a, real_in ? (A_SAVE | A_MULT_T | A_FWD) : (A_INV | A_SAVE | A_MULT_T | A_FWD), 1));
          MS_TRY(pass_b(passb_args(d_t1_.p, d_t1_.p, 0), B_PROPAGATE, 1));
          launches += 2;
          cur = d_t1_.p;
        }
        float2* last = d_seg_.p + (size_t)(e - 1 - c) * N;
        if (c == clast) {
          // saved by the forward sweep
        } else if (e - 1 == 0) {
          MS_TRY(cudaMemcpyAsync(last, d_psi0_.p, sizeof(float2) * N, cudaMemcpyDeviceToDevice, stream_));
        } else {
          MS_TRY(pass_a(passa_args(cur, last, 0), A_INV, 1));
          ++launches;
        }
        // adjoint steps e .. c+1
        for (int n = e; n >= c + 1; --n) {
          PassBArgs b = passb_args(d_G_.p, d_G_.p, 0);
          b.scale = (float)nx_;
          MS_TRY(pass_b(b, B_PROPAGATE_ADJ, 1));
          PassAArgs a = passa_args(d_G_.p, d_G_.p, 0);
          a.V = d_stack_.p + (size_t)(n - 1) * N;
          a.in2 = d_seg_.p + (size_t)(n - 1 - c) * N;
          // (without dLdV kept per slice: two buffers, slice n in n & 1, free
          // again once slice n + 2's atom-position adjoint has read it)
          float* dV = dLdV ? d_dV_.p + (size_t)(n - 1) * N : d_dV_.p + (size_t)(n & 1) * N;
          if (!dLdV && dLdxy) MS_TRY(cudaStreamWaitEvent(stream_, ev_adj_[n & 1], 0));
          a.out_f = dV;
          a.scale = 1.0f / (float)nx_;
          MS_TRY(pass_a(a, A_INV | A_ADJ | A_FWD, 1));
          launches += 2;
          if (dLdxy) {
            const PotArgs pa = pot_args(POT_CONVENTIONAL, n, nullptr);
            const int a0 = hzoff_[pa.kt], a1 = hzoff_[pa.kb + 1];
            const bool sep = separable_ok();
            // on a second stream: the next slices' adjoint passes do not wait
            // for it (it reads dV and adds into dL/dxy only)
            MS_TRY(cudaEventRecord(ev_dv_, stream_));
            MS_TRY(cudaStreamWaitEvent(pix_[1], ev_dv_, 0));
            MS_TRY(launch_potential_adjoint(pa, dV, d_idx_.p, a0, a1, d_dxy_.p, pix_[1], sep));
            MS_TRY(cudaEventRecord(ev_adj_[n & 1], pix_[1]));
            launches += sep ? 2 : 1;
          }
        }
      }
      if (dLdxy) {
        MS_TRY(cudaEventRecord(ev_join_, pix_[1]));
        MS_TRY(cudaStreamWaitEvent(stream_, ev_join_, 0));
      }
    }
    MS_TRY(cudaEventRecord(ev1_, stream_));
    MS_TRY(cudaMemcpyAsync(loss, d_loss_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    if (images)
      MS_TRY(cudaMemcpyAsync(images, d_img_.p, sizeof(float) * N * nd, cudaMemcpyDeviceToHost, stream_));
    if (grad && dLdV)
      MS_TRY(cudaMemcpyAsync(dLdV, d_dV_.p, sizeof(float) * N * S, cudaMemcpyDeviceToHost, stream_));
    if (grad && dLdxy)
      MS_TRY(cudaMemcpyAsync(dLdxy, d_dxy_.p, sizeof(double) * 2 * natoms_, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    MS_TRY(cudaEventElapsedTime(&last_device_ms_, ev0_, ev1_));
    domain_ = 1;
    return MS_OK;
  }

  // First sorted atom of every 1-A z-bin (CSR offsets at bin k * 2500), k = 0..nz.
  int zbin_starts() {
    if ((int)hzoff_.size() == nzb_ + 1) return MS_OK;
    hzoff_.assign(nzb_ + 1, 0);
    MS_TRY(cudaMemcpy2DAsync(hzoff_.data(), sizeof(int), d_off_.p, sizeof(int) * kBins2, sizeof(int), nzb_ + 1,
                             cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return MS_OK;
  }

  int last_device_ms(float* out) {
    *out = last_device_ms_;
    return MS_OK;
  }

  // Device time of one fused pass (pass 0: row pass with `op` = PassAFlags;
  // pass 1: column pass with `op` = PassBMode) of plan `variant` over `batch`
  // scratch instances, averaged over `reps` back-to-back launches.
  int time_pass(int pass, int op, int variant, int batch, int reps, float* us) {
    if (!have_freq_ || !use_fused()) return fail(MS_ERR_STATE, "fused grid not set up (ms_precalculate_frequencies)");
    if (pass < 0 || pass > 1 || variant < 0 || variant >= plan_variants() || batch < 1 || batch > 256 || reps < 1)
      return fail(MS_ERR_INVALID, "bad pass, variant, batch or reps");
    if (pass == 0 && (op & (A_FD | A_RESID | A_ADJ | A_SAVE | A_INTENSITY | A_REAL)) != 0)
      return fail(MS_ERR_INVALID, "row-pass timing covers A_INV, A_MULT_T, A_MULT_TC and A_FWD");
    if (pass == 1 && (op == B_CBED || op == B_DETECT || op == B_FD || op == B_CTF_ADJ))
      return fail(MS_ERR_INVALID, "column-pass timing covers the wave-to-wave modes");
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    const long long N = (long long)nx_ * ny_;
    DevBuf<float2> w, T;
    DevBuf<float> V;
    MS_TRY(w.resize((size_t)batch * N));
    MS_TRY(V.resize((size_t)N));
    MS_TRY(T.resize((size_t)N));  // one transmission slice shared by the instances (A_MULT_TC)
    MS_TRY(cudaMemsetAsync(w.p, 0, sizeof(float2) * batch * N, stream_));
    MS_TRY(cudaMemsetAsync(V.p, 0, sizeof(float) * N, stream_));
    MS_TRY(cudaMemsetAsync(T.p, 0, sizeof(float2) * N, stream_));
    PassAArgs a = passa_args(w.p, w.p, variant);
    a.V = V.p;
    a.tr = T.p;
    a.batch_stride_wave = N;
    PassBArgs b = passb_args(w.p, w.p, variant);
    b.batch_stride_wave = N;
    b.ctf = CtfParams{(double)wavel_, (double)Cs_, (double)df_, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1e30f};
    auto launch = [&]() {
      return pass == 0 ? launch_pass_a(a, variant, op, batch, stream_) : launch_pass_b(b, variant, op, batch, stream_);
    };
    for (int k = 0; k < 2; ++k) MS_TRY(launch());
    MS_TRY(cudaEventRecord(ev0_, stream_));
    for (int k = 0; k < reps; ++k) MS_TRY(launch());
    MS_TRY(cudaEventRecord(ev1_, stream_));
    MS_TRY(cudaEventSynchronize(ev1_));
    float ms = 0.0f;
    MS_TRY(cudaEventElapsedTime(&ms, ev0_, ev1_));
    launches += reps + 2;
    *us = 1000.0f * ms / (float)reps;
    return check_pass_err();
  }

  // Checkpoint stride when none is set: every wave stored (no recomputation)
  // when the S waves take at most an eighth of the device's free memory, else
  // ceil(sqrt(S)) (sqrt(S) checkpoints, each segment recomputed once).
  static int auto_checkpoint_stride(int S, size_t N) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = 0;
    }
    if ((size_t)S * N * sizeof(float2) <= free_b / 8) return 1;
    return (int)std::ceil(std::sqrt((double)S));
  }

  // ---- inspection ----
  int fft_plan(int batch, int* row, int* col) {
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    if (!use_fused()) return fail(MS_ERR_UNSUPPORTED, "grid not handled by the fused passes");
    if (batch < 1) return fail(MS_ERR_INVALID, "batch must be >= 1");
    const PlanChoice c = plan_for(batch);
    *row = c.row;
    *col = c.col;
    return MS_OK;
  }

  int binned_counts(int* n, int* nz) {
    if (!have_index_) return fail(MS_ERR_STATE, "atoms not binned");
    *n = natoms_;
    *nz = nzb_;
    return MS_OK;
  }

  int copy_binned(int* off, int* Z, float* x, float* y, float* z) {
    if (!have_index_) return fail(MS_ERR_STATE, "atoms not binned");
    std::vector<float4> at(natoms_);
    MS_TRY(copy_sync(at.data(), d_atoms_.p, sizeof(float4) * natoms_, cudaMemcpyDeviceToHost));
    MS_TRY(copy_sync(off, d_off_.p, sizeof(int) * ((size_t)nzb_ * kBins2 + 1), cudaMemcpyDeviceToHost));
    for (int i = 0; i < natoms_; ++i) {
      x[i] = at[i].x;
      y[i] = at[i].y;
      z[i] = at[i].z;
      int zz;
      std::memcpy(&zz, &at[i].w, sizeof(int));
      Z[i] = zz;
    }
    return MS_OK;
  }

  int copy_potential(int kind, int it, float* dst) {
    if (int rc = require_potential_inputs()) return rc;
    if (it < 1) return fail(MS_ERR_INVALID, "iteration counts from 1");
    if (kind < 0 || kind > 3) return fail(MS_ERR_INVALID, "unknown potential kind");
    if (int rc = potential_slice(kind, it, d_f_.p)) return rc;
    MS_TRY(cudaMemcpyAsync(dst, d_f_.p, sizeof(float) * nx_ * ny_, cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    return MS_OK;
  }

  // ---- simple accessors ----
  int device() const { return device_; }
  const Box& box() const { return box_; }
  bool have_atoms() const { return have_atoms_; }
  float kmax() const { return kmax_; }
  bool have_freq() const { return have_freq_; }
  int nx() const { return nx_; }
  int ny() const { return ny_; }
  float ew_min() const { return ew_min_; }
  float ew_max() const { return ew_max_; }
  bool have_ew() const { return have_ew_; }
  float im_min() const { return im_min_; }
  float im_max() const { return im_max_; }
  bool have_image() const { return have_image_; }

  // Copies through the handle's stream and waits.  A plain cudaMemcpy runs on
  // the legacy default stream, which the handle's non-blocking stream does not
  // wait for, and from pageable memory it may return before the DMA lands.
  cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, stream_);
    return e == cudaSuccess ? cudaStreamSynchronize(stream_) : e;
  }

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }

 private:
  static constexpr float FLT_MAX_ = 3.40282347e+38f;

  int cuda_fail(cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? MS_ERR_NOMEM : MS_ERR_CUDA;
  }

  bool use_fused() const { return fused_ok_ && !force_plain_; }


  // Drops the captured slice-loop graph (it holds the wave buffers, tables and
  // set-up scalars as kernel arguments).
  void drop_conv_graph() {
    if (graph_exec_) {
      cudaGraphExecDestroy(graph_exec_);
      graph_exec_ = nullptr;
    }
    graph_S_ = -1;
  }
  // Every change of the grid, structure, parameters or options drops both
  // captured graphs (conventional loop and FD run).
  void invalidate_graph() {
    drop_conv_graph();
    drop_fd_graph();
  }

  int require_potential_inputs() {
    if (!have_index_) return fail(MS_ERR_STATE, "atoms not binned (ms_upload_binned_atoms)");
    if (!have_fp_) return fail(MS_ERR_STATE, "parameterisation not loaded (ms_get_parameterisation)");
    if (!have_freq_) return fail(MS_ERR_STATE, "frequencies not precalculated");
    for (int z : hZ_)
      if (z > nrows_fp_) return fail(MS_ERR_INVALID, "an atom's Z has no row in the parameterisation table");
    return MS_OK;
  }

  // Common tail of the initialisers: psi- = psi0, and the second level for
  // finite differences psi = IFFT(P(dzFD) FFT(psi0)) / N (U.cu:1984-1993).
  int finish_init() {
    const Grid2 g{nx_, ny_};
    const size_t N = (size_t)nx_ * ny_;
    MS_TRY(cudaMemcpyAsync(d_psim_.p, d_psi0_.p, sizeof(float2) * N, cudaMemcpyDeviceToDevice, stream_));
    const float nf = 1.0f / std::sqrt((float)(nx_ * ny_));
    MS_TRY(pw_props(d_kx_.p, d_ky_.p, dzFD_, wavel_, kmax_, d_t2_.p, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_psi0_.p, d_t1_.p, CUFFT_FORWARD));
    MS_TRY(pw_cmul(d_t1_.p, d_t2_.p, d_t1_.p, nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_psi_.p, CUFFT_INVERSE));
    MS_TRY(pw_scale(d_psi_.p, nf, g, stream_, &launches));
    MS_TRY(cudaStreamSynchronize(stream_));
    domain_ = 0;
    fd_state_ = false;
    have_waves_ = true;
    // (the propagator tables depend on dz, the wavelength and the grid only:
    // they stay valid across re-initialisations, keyed by prop_dz_)
    return MS_OK;
  }

  // Propagator factors for the fused column pass: P(kx,ky) = px[kx] * py[ky]
  // with px = exp(-i pi dz lambda kx^2) / N and py = exp(-i pi dz lambda ky^2),
  // phases in FP64 (CreatePropsKernel U.cu:399-428 uses pi = 3.14159265).
  int ensure_prop_tables(float dz) {
    if (dz == prop_dz_ && d_px_.p) return MS_OK;
    std::vector<float2> px(nx_), py(ny_);
    const double invN = 1.0 / ((double)nx_ * ny_);
    // unit factors nearest modulus 1 (unit_fp32); the 1/N of the fused
    // passes is a power of two, so scaling px by it is exact
    const float fN = (float)invN;
    for (int i = 0; i < nx_; ++i) {
      const double ph = 3.14159265 * (double)dz * (double)wavel_ * (double)hkx_[i] * (double)hkx_[i];
      const float2 u = unit_fp32(std::cos(ph), -std::sin(ph));
      px[i] = make_float2(u.x * fN, u.y * fN);
    }
    for (int j = 0; j < ny_; ++j) {
      const double ph = 3.14159265 * (double)dz * (double)wavel_ * (double)hky_[j] * (double)hky_[j];
      py[j] = unit_fp32(std::cos(ph), -std::sin(ph));
    }
    MS_TRY(d_px_.resize(nx_));
    MS_TRY(d_py_.resize(ny_));
    MS_TRY(copy_sync(d_px_.p, px.data(), sizeof(float2) * nx_, cudaMemcpyHostToDevice));
    MS_TRY(copy_sync(d_py_.p, py.data(), sizeof(float2) * ny_, cudaMemcpyHostToDevice));
    prop_dz_ = dz;
    // plain path: full propagator array, as CreatePropsKernel
    MS_TRY(d_P_.resize((size_t)nx_ * ny_));
    MS_TRY(pw_props(d_kx_.p, d_ky_.p, dz, wavel_, kmax_, d_P_.p, Grid2{nx_, ny_}, stream_, &launches));
    return MS_OK;
  }

  // FFT plan variants of the row and column passes for a batch size: forced
  // by MS_OPT_FFT_PLAN, else the autotuned choice (timed once per batch size).
  struct PlanChoice {
    int row = 0, col = 0;
  };
  // `tc`: the row pass multiplies by a precomputed transmission (A_MULT_TC,
  // the batched raster) rather than forming exp(i sigma V) itself; the two
  // load different operands and are tuned apart.
  PlanChoice plan_for(int batch, bool tc = false) {
    if (forced_plan_ >= 0) return PlanChoice{forced_plan_, forced_plan_};
    const int bucket = batch <= 1 ? 1 : batch < 8 ? 4 : batch < 32 ? 16 : 64;
    const int key = bucket + (tc ? 1000 : 0);
    for (auto& kv : tuned_)
      if (kv.first == key) return kv.second;
    PlanChoice c = autotune(bucket, tc);
    tuned_.push_back({key, c});
    return c;
  }

  // Times every plan variant of the steady-state row pass and the propagating
  // column pass on scratch waves (batch instances), on this device, then the
  // three fastest of each in pairs, alternating, and keeps the fastest pair.
  // Scratch is zero-filled so the transmission's sincos stays on its fast
  // path.  On any launch failure the variant is skipped.
  PlanChoice autotune(int batch, bool tc) {
    PlanChoice best;
    const long long N = (long long)nx_ * ny_;
    DevBuf<float2> w, T;
    DevBuf<float> V;
    if (w.resize((size_t)batch * N) != cudaSuccess || V.resize((size_t)N) != cudaSuccess) return best;
    if (tc && T.resize((size_t)N) != cudaSuccess) return best;
    cudaMemsetAsync(w.p, 0, sizeof(float2) * batch * N, stream_);
    cudaMemsetAsync(V.p, 0, sizeof(float) * N, stream_);
    if (tc) cudaMemsetAsync(T.p, 0, sizeof(float2) * N, stream_);
    const int row_op = tc ? (A_INV | A_MULT_TC | A_FWD) : (A_INV | A_MULT_T | A_FWD);
    if (ensure_prop_tables(convdz_) != MS_OK) return best;
    const int reps = 8, nv = plan_variants();
    auto row_args = [&](int v) {
      PassAArgs a = passa_args(w.p, w.p, v);
      a.V = V.p;
      a.tr = T.p;
      a.batch_stride_wave = N;
      a.batch_stride_V = 0;
      return a;
    };
    auto col_args = [&](int v) {
      PassBArgs b = passb_args(w.p, w.p, v);
      b.batch_stride_wave = N;
      return b;
    };
    auto elapsed = [&](auto&& body) {
      float ms = INFINITY;
      cudaEventRecord(ev0_, stream_);
      body();
      cudaEventRecord(ev1_, stream_);
      if (cudaEventSynchronize(ev1_) != cudaSuccess || cudaEventElapsedTime(&ms, ev0_, ev1_) != cudaSuccess) {
        cudaGetLastError();
        return INFINITY;
      }
      return ms;
    };
    // each variant of each pass alone
    std::vector<float> ta(nv, INFINITY), tb(nv, INFINITY);
    for (int v = 0; v < nv; ++v) {
      const PassAArgs a = row_args(v);
      const PassBArgs b = col_args(v);
      bool ok = true;
      for (int k = 0; k < 2 && ok; ++k)  // first launches load the kernels
        ok = launch_pass_a(a, v, row_op, batch, stream_) == cudaSuccess &&
             launch_pass_b(b, v, B_PROPAGATE, batch, stream_) == cudaSuccess;
      if (!ok || cudaStreamSynchronize(stream_) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      ta[v] = elapsed([&] { for (int k = 0; k < reps; ++k) launch_pass_a(a, v, row_op, batch, stream_); });
      tb[v] = elapsed([&] { for (int k = 0; k < reps; ++k) launch_pass_b(b, v, B_PROPAGATE, batch, stream_); });
      launches += 2LL * (reps + 2);
    }
    // the three fastest of each, paired and timed alternating as the slice
    // loop runs them (a pass's speed depends on its neighbour: programmatic
    // dependent launch lets the next pass's CTAs in while this one drains)
    auto top3 = [&](const std::vector<float>& t) {
      std::vector<int> idx(nv);
      for (int v = 0; v < nv; ++v) idx[v] = v;
      std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return t[x] < t[y]; });
      idx.resize(std::min(nv, 3));
      return idx;
    };
    float best_t = INFINITY;
    for (int r : top3(ta)) {
      if (!(ta[r] < INFINITY)) continue;
      for (int c : top3(tb)) {
        if (!(tb[c] < INFINITY)) continue;
        const PassAArgs a = row_args(r);
        const PassBArgs b = col_args(c);
        const float t = elapsed([&] {
          for (int k = 0; k < reps; ++k) {
            launch_pass_a(a, r, row_op, batch, stream_);
            launch_pass_b(b, c, B_PROPAGATE, batch, stream_);
          }
        });
        launches += 2LL * reps;
        if (t < best_t) {
          best_t = t;
          best.row = r;
          best.col = c;
        }
      }
    }
    cudaStreamSynchronize(stream_);
    return best;
  }

  PassAArgs passa_args(const float2* in, float2* out, int variant) {
    PassAArgs a{};
    a.in = in; a.out = out; a.tw = d_twx_[variant].p; a.nx = nx_; a.ny = ny_;
    a.sigma = sigma2_; a.scale = 1.0f;
    return a;
  }
  PassBArgs passb_args(const float2* in, float2* out, int variant) {
    PassBArgs b{};
    b.in = in; b.out = out; b.tw = d_twy_[variant].p; b.px = d_px_.p; b.py = d_py_.p;
    b.kx = d_kx_.p; b.ky = d_ky_.p; b.kmax = kmax_; b.nx = nx_; b.ny = ny_; b.scale = 1.0f;
    band_limit_thresholds(kmax_, &b.k2_lt, &b.k2_le);
    b.err = d_pass_err_.p;  // (long propagation columns: tensor-copy staging, see check_pass_err)
    return b;
  }
  // The column pass's tensor-copy waits are bounded: one that ran out set the
  // error word (its columns were left as they were).  Checked where the
  // handle synchronises after such passes (whole runs, timing, read-outs).
  int check_pass_err() {
    int h = 0;
    MS_TRY(cudaMemcpyAsync(&h, d_pass_err_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    MS_TRY(cudaStreamSynchronize(stream_));
    if (h == 0) return MS_OK;
    MS_TRY(cudaMemsetAsync(d_pass_err_.p, 0, sizeof(int), stream_));
    return fail(MS_ERR_CUDA, "a column pass's tensor-copy wait ran out (bounded at one second)");
  }
  // Row / column pass launchers with the plan tuned for `batch` instances.
  cudaError_t pass_a(PassAArgs a, int flags, int batch = 1, cudaStream_t s = nullptr) {
    const int v = plan_for(batch).row;
    a.tw = d_twx_[v].p;
    return launch_pass_a(a, v, flags, batch, s ? s : stream_);
  }
  cudaError_t pass_b(PassBArgs b, int mode, int batch = 1, cudaStream_t s = nullptr) {
    const int v = plan_for(batch).col;
    b.tw = d_twy_[v].p;
    return launch_pass_b(b, v, mode, batch, s ? s : stream_);
  }

  // Enqueue one fused conventional step on the stream (no host sync, no
  // allocation or copy: safe inside stream capture once the propagator
  // tables exist).
  int enqueue_fused_step(const float* V, bool first, cudaStream_t s = nullptr) {
    fd_state_ = false;
    // iteration 1 starts from the initial wave (real space); later ones from
    // the current wave in whichever domain it is held
    PassAArgs a = passa_args(first ? d_psi0_.p : d_psi_.p, d_psi_.p, 0);
    a.V = V;
    const int fl = (first || domain_ == 0) ? (A_MULT_T | A_FWD) : (A_INV | A_MULT_T | A_FWD);
    MS_TRY(pass_a(a, fl, 1, s));
    MS_TRY(pass_b(passb_args(d_psi_.p, d_psi_.p, 0), B_PROPAGATE, 1, s));
    domain_ = 1;
    return MS_OK;
  }

  // transmission + propagation of one conventional slice with potential V.
  int transmit_propagate(const float* V, bool first) {
    if (int rc = ensure_prop_tables(convdz_)) return rc;
    if (domain_ == 2)
      if (int rc = ensure_real()) return rc;
    if (use_fused()) {
      if (int rc = enqueue_fused_step(V, first)) return rc;
      launches += 2;
      return MS_OK;
    }
    // plain path: the reference's launch sequence (U.cu:2101-2122)
    if (int rc = ensure_real()) return rc;
    fd_state_ = false;
    const Grid2 g{nx_, ny_};
    const float nf = 1.0f / std::sqrt((float)(nx_ * ny_));
    MS_TRY(pw_transmission(V, sigma2_, d_t2_.p, g, stream_, &launches));
    MS_TRY(pw_cmul(d_t2_.p, first ? d_psi0_.p : d_psi_.p, d_t1_.p, 1.0f, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_t2_.p, CUFFT_FORWARD));
    MS_TRY(pw_cmul(d_t2_.p, d_P_.p, d_t1_.p, nf, g, stream_, &launches));
    MS_TRY_FFT(cufftExecC2C(plan_, d_t1_.p, d_psi_.p, CUFFT_INVERSE));
    MS_TRY(pw_scale(d_psi_.p, nf, g, stream_, &launches));
    domain_ = 0;
    return MS_OK;
  }

  int ensure_real() {
    if (domain_ == 0) return MS_OK;
    if (domain_ == 2) {
      // fused finite differences: psi_n = IFFT_row(X), the FD state stays valid
      MS_TRY(pass_a(passa_args(d_fdX_.p, d_psi_.p, 0), A_INV, 1));
      ++launches;
      domain_ = 0;
      return MS_OK;
    }
    PassAArgs a = passa_args(d_psi_.p, d_psi_.p, 0);
    MS_TRY(pass_a(a, A_INV, 1));
    ++launches;
    domain_ = 0;
    return MS_OK;
  }

  // Separable potentials of slices 1..S into out + (it - 1) * N (and, for a
  // batch of nb indices set up as in tds_potential_batch, instance k at
  // out + k * S * N), npix table buffers deep: the tables of the next slices
  // are built on the side stream while earlier slices' potentials run.  Slice
  // it's potential runs on pixel stream it % npix (stream 0 is the handle's):
  // consecutive slices are independent, and on several streams the last CTAs
  // of one launch overlap the first of the next.  The tables' side stream has
  // the higher priority, so the next slices' tables are not queued behind
  // potential CTAs.  Event order: tables(it) after
  // potential(it - npix), which read the same buffer; potential(it) after
  // tables(it).  The side stream joins the handle's stream through the last
  // potentials' dependence on their tables.
  int separable_stack(int S, float* out, size_t N, int nb, const float4* atoms = nullptr, const int* off = nullptr,
                      long long b_atoms = 0, long long b_off = 0,
                      const std::function<int(int, cudaEvent_t)>& after_slice = nullptr, int npix = kPixStreams) {
    npix = std::min(std::max(npix, 1), kPixStreams);
    if (pot_tile_ < 0 && !capturing_)
      if (int rc = tune_pot_tile()) return rc;
    const int tile = std::min(std::max(pot_tile_, 0), potential_tiles_separable() - 1);
    const size_t per = (size_t)nb * natoms_ * kTabStride;  // one buffer
    if (d_tab_.n < npix * per) MS_TRY(d_tab_.resize(npix * per));
    MS_TRY(cudaEventRecord(ev_fork_, stream_));
    MS_TRY(cudaStreamWaitEvent(side_, ev_fork_, 0));
    for (int k = 1; k < npix; ++k) MS_TRY(cudaStreamWaitEvent(pix_[k], ev_fork_, 0));
    int rc = MS_OK;
    for (int it = 1; it <= S && rc == MS_OK; ++it)
      rc = separable_slice(it, out, N, nb, per, tile, atoms, off, b_atoms, b_off, S, after_slice, npix);
    // join the other pixel streams (also on failure, so that the handle's
    // stream orders after everything enqueued)
    for (int k = 1; k < npix; ++k) {
      MS_TRY(cudaEventRecord(ev_pjoin_[k], pix_[k]));
      MS_TRY(cudaStreamWaitEvent(stream_, ev_pjoin_[k], 0));
    }
    if (rc != MS_OK) return rc;
    last_pot_sum_ = 2;
    return MS_OK;
  }
  // One slice of separable_stack: its atom tables on the side stream (into
  // table buffer it % npix, once the potential of slice it - npix, which read
  // that buffer, is done), then its potential on pixel stream it % npix.
  int separable_slice(int it, float* out, size_t N, int nb, size_t per, int tile, const float4* atoms,
                      const int* off, long long b_atoms, long long b_off, int S,
                      const std::function<int(int, cudaEvent_t)>& after_slice, int npix) {
    const int buf = it % npix;
    cudaStream_t ps = pix_[buf];
    PotArgs a = pot_args(POT_CONVENTIONAL, it, out + (size_t)(it - 1) * N);
    a.tab = d_tab_.p + buf * per;
    if (atoms) {
      a.atoms = atoms;
      a.off = off;
      a.b_atoms = b_atoms;
      a.b_off = b_off;
      a.b_tab = (long long)natoms_ * kTabStride;
      a.b_V = (long long)S * N;
    }
    if (it > npix) MS_TRY(cudaStreamWaitEvent(side_, ev_pix_[buf], 0));
    MS_TRY(launch_atom_tables(a, side_, nb));
    MS_TRY(cudaEventRecord(ev_tab_[buf], side_));
    MS_TRY(cudaStreamWaitEvent(ps, ev_tab_[buf], 0));
    MS_TRY(launch_potential_from_tables(a, ps, tile, nb));
    MS_TRY(cudaEventRecord(ev_pix_[buf], ps));
    launches += 2;
    if (after_slice)
      if (int rc = after_slice(it, ev_pix_[buf])) return rc;
    return MS_OK;
  }

  // Whether element row r's Gaussian expansion holds for the loaded table:
  // checked once per row in FP64, with the kernel's FP32-rounded exponents and
  // weights, against vatom (U.cu:160-193) on 0.25 <= r <= 2.2365 A.
  bool gauss_row_ok(int r) {
    if (r < 0 || r >= 103 || r >= nrows_fp_) return false;
    if (gauss_row_ok_[r] >= 0) return gauss_row_ok_[r] == 1;
    bool ok = (int)kGaussFit[r][0] == kGaussJ;
    const double pi = 3.141592654;
    const double* f = &hfp_[r * 12];
    const float* al = &hgauss_[(r * 2) * kGaussJ];
    const float* w = &hgauss_[(r * 2 + 1) * kGaussJ];
    for (int i = 0; ok && i < 1000; ++i) {
      const double rad = 0.25 * std::pow(2.2365 / 0.25, i / 999.0), r2 = rad * rad;
      double L = 0.0, G = 0.0;
      for (int k = 0; k < 3; ++k) {
        L += f[2 * k] * std::exp(-2.0 * pi * rad * std::sqrt(f[2 * k + 1]));
        G += f[6 + 2 * k] * std::exp(-(pi * rad) * (pi * rad) / f[7 + 2 * k]) * std::pow(f[7 + 2 * k], -1.5);
      }
      const double v = 150.4121417 * L / rad + 266.5157269 * G;
      double e = 0.0;
      for (int j = 0; j < kGaussJ; ++j) e += (double)w[j] * std::exp2(-(double)al[j] * r2);
      ok = v > 0.0 && std::fabs(e - v) <= kGaussTol * v;
    }
    gauss_row_ok_[r] = ok ? 1 : 0;
    return ok;
  }
  // The separable conventional kernel applies when every element of the
  // specimen has a valid expansion (MS_OPT_POTENTIAL_SUM 0 or 2).
  bool separable_ok() {
    if (pot_sum_ == 1 || !have_fp_) return false;
    for (int z = 1; z <= 103; ++z)
      if (z < (int)zpresent_.size() && zpresent_[z] && !gauss_row_ok(z - 1)) return false;
    return true;
  }

  // Potential of one slice into out (ny x nx floats).
  int potential_slice(int kind, int it, float* out) {
    const bool sep = kind == POT_CONVENTIONAL && separable_ok();
    if (kind == POT_CONVENTIONAL && pot_sum_ == 2 && !sep)
      return fail(MS_ERR_UNSUPPORTED, "an element of the specimen has no valid Gaussian expansion");
    if (kind == POT_CONVENTIONAL && pot_tile_ < 0 && !capturing_)
      if (int rc = tune_pot_tile()) return rc;
    const PotArgs a = pot_args(kind, it, out);
    const int ntile = sep ? potential_tiles_separable() : potential_tiles();
    MS_TRY(launch_potential(a, kind, stream_, kind == POT_CONVENTIONAL ? std::min(std::max(pot_tile_, 0), ntile - 1) : 0,
                            sep));
    launches += sep ? 2 : 1;
    last_pot_sum_ = kind == POT_CONVENTIONAL ? (sep ? 2 : 1) : last_pot_sum_;
    return MS_OK;
  }

  // Tile shape of the conventional potential kernel for this grid, tuned on
  // the device the first time it is needed: each shape builds the mid-slab
  // slice (one warm-up launch, then three timed) and the fastest is kept.
  int tune_pot_tile() {
    int S = 0;
    if (int rc = get_slices(true, &S)) return rc;
    const int it = std::max(1, S / 2);
    const size_t N = (size_t)nx_ * ny_;
    MS_TRY(d_V_.resize(N));
    float best_t = INFINITY;
    int best = 0;
    const bool sep = separable_ok();
    for (int t = 0; t < (sep ? potential_tiles_separable() : potential_tiles()); ++t) {
      const PotArgs a = pot_args(POT_CONVENTIONAL, it, d_V_.p);
      MS_TRY(launch_potential(a, POT_CONVENTIONAL, stream_, t, sep));
      MS_TRY(cudaEventRecord(ev0_, stream_));
      for (int k = 0; k < 3; ++k) MS_TRY(launch_potential(a, POT_CONVENTIONAL, stream_, t, sep));
      MS_TRY(cudaEventRecord(ev1_, stream_));
      MS_TRY(cudaEventSynchronize(ev1_));
      float ms = 0.0f;
      MS_TRY(cudaEventElapsedTime(&ms, ev0_, ev1_));
      launches += sep ? 8 : 4;
      if (ms < best_t) {
        best_t = ms;
        best = t;
      }
    }
    pot_tile_ = best;
    return MS_OK;
  }

  PotArgs pot_args(int kind, int it, float* out) {
    PotArgs a{};
    a.atoms = d_atoms_.p;
    a.off = d_off_.p;
    a.coef = d_coef_.p;
    a.tab = d_tab_.p;
    a.gauss = d_gauss_.p;
    a.V = out;
    a.nx = nx_;
    a.ny = ny_;
    a.nz = nzb_;
    a.ps = ps_;
    a.bw_x = (box_.MaxX - box_.MinX) / kBins;
    a.bw_y = (box_.MaxY - box_.MinY) / kBins;
    const float top = box_.MaxZ - box_.MinZ;
    if (kind == POT_CONVENTIONAL) {
      // binnedAtomPKernel3 U.cu:582-653 launched at U.cu:2101 with z = top - convdz*it
      const float z = box_.MaxZ - box_.MinZ - convdz_ * it;
      const int K = (int)std::floor((box_.MaxZ - box_.MinZ - z) / (float)1);
      a.kt = std::max(K - lbz_, 0);
      a.kb = std::min(K + lbz_, nzb_ - 1);
      a.xoff = xoff_;
      a.yoff = yoff_;
      a.nsub = 20;
      for (int m = 1; m <= 20; ++m) {
        a.zsub[m - 1] = z - m * convdz_ / 20.0f;
        a.zsub_lo[m - 1] = (float)(((double)z - m * (double)convdz_ / 20.0) - (double)a.zsub[m - 1]);
      }
      a.wsub = convdz_ / 20.0f;
    } else if (kind == POT_RS) {
      // binnedAtomPKernelRS U.cu:655-727 at z = top - dz*it, dz = 1 (int) (U.cu:2129-2137)
      const float z = box_.MaxZ - box_.MinZ - (float)(1 * it);
      const int K = (int)std::floor((box_.MaxZ - box_.MinZ - z) / (float)1);
      a.kt = std::max(K - lbz_, 0);
      a.kb = std::min(K + lbz_, nzb_ - 1);
      a.xoff = xoff_;
      a.yoff = yoff_;
      a.nsub = 10;
      for (int m = 1; m <= 10; ++m) {
        a.zsub[m - 1] = z - (float)(m * 1) / 10.0f;
        a.zsub_lo[m - 1] = (float)(((double)z - m / 10.0) - (double)a.zsub[m - 1]);
      }
      a.wsub = 1 / 10.0f;
    } else if (kind == POT_FD) {
      // binnedAtomPKernelFD U.cu:883-946 at z = top - dzFD*it, no offsets
      const float z = box_.MaxZ - box_.MinZ - dzFD_ * it;
      const int K = (int)std::floor((box_.MaxZ - box_.MinZ - z) / (float)1);
      a.kt = std::max(K - lbz_, 0);
      a.kb = std::min(K + lbz_, nzb_ - 1);
      a.xoff = 0.0f;
      a.yoff = 0.0f;
      a.nsub = 1;
      a.zsub[0] = z;
      a.wsub = 1.0f;
    } else {
      // projected slab it: depth in [(it-1) dz, it dz)
      a.xoff = xoff_;
      a.yoff = yoff_;
      a.top = top;
      a.slab_dz = convdz_;
      a.slab = it - 1;
      a.kt = std::max((int)std::floor((it - 1) * convdz_) - 1, 0);
      a.kb = std::min((int)std::floor(it * convdz_) + 1, nzb_ - 1);
    }
    return a;
  }

  // Thermal displacements of atoms [a0, a1) for one pass: counter-based
  // (Philox keyed by the seed, counter = atom, pass), so any split of the
  // atoms over threads gives the same positions.
  static void tds_displace_range(const float* x, const float* y, const float* z, int a0, int a1, uint64_t seed,
                                 uint32_t pass, float sigma, float* xo, float* yo, float* zo) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const double twopi = 6.283185307179586;
    for (int a = a0; a < a1; ++a) {
      uint32_t ctr[4] = {(uint32_t)a, pass, 0x5EEDu, 0u}, r[4];
      philox4x32_10(ctr, key, r);
      double u[4];
      for (int j = 0; j < 4; ++j) u[j] = ((double)r[j] + 0.5) * 2.3283064365386963e-10;
      const double m0 = std::sqrt(-2.0 * std::log(u[0])), m1 = std::sqrt(-2.0 * std::log(u[2]));
      xo[a] = (float)((double)x[a] + (double)sigma * m0 * std::cos(twopi * u[1]));
      yo[a] = (float)((double)y[a] + (double)sigma * m0 * std::sin(twopi * u[1]));
      zo[a] = (float)((double)z[a] + (double)sigma * m1 * std::cos(twopi * u[3]));
    }
  }
  // Displacements of nb passes pass0 .. pass0 + nb - 1 into xo + k * n etc.,
  // split over the host's threads (about 140 ns per atom and pass on one).
  static void tds_displace(const float* x, const float* y, const float* z, int n, uint64_t seed, uint32_t pass0,
                           float sigma, float* xo, float* yo, float* zo, int nb = 1) {
    const long long total = (long long)n * nb;
    const int hw = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const int nt = (int)std::max<long long>(1, std::min<long long>(hw, total / 4096));
    auto work = [&](int t) {
      const long long q0 = total * t / nt, q1 = total * (t + 1) / nt;
      for (long long q = q0; q < q1;) {
        const int k = (int)(q / n), a0 = (int)(q % n);
        const int a1 = (int)std::min<long long>(n, a0 + (q1 - q));
        const size_t o = (size_t)k * n;
        tds_displace_range(x, y, z, a0, a1, seed, pass0 + (uint32_t)k, sigma, xo + o, yo + o, zo + o);
        q += a1 - a0;
      }
    };
    if (nt == 1) {
      work(0);
      return;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& h : th) h.join();
  }

  // state
  int device_;
  cudaStream_t stream_ = nullptr;
  cudaStream_t side_ = nullptr;
  // pixel streams of a separable stack (0: the handle's stream)
  static constexpr int kPixStreams = 3;
  cudaStream_t pix_[kPixStreams] = {};
  cudaStream_t pass_ = nullptr;  // slice passes overlapping the stack build (run_conventional_streamed)
  cudaEvent_t ev_tab_[kPixStreams] = {}, ev_pix_[kPixStreams] = {}, ev_pjoin_[kPixStreams] = {};
  cudaEvent_t ev_fork_ = nullptr, ev_fork2_ = nullptr, ev_join_ = nullptr;
  cudaEvent_t ev_dv_ = nullptr, ev_adj_[2] = {};  // focal-series gradient: dV ready, dV buffer read
  bool overlap_build_ = true;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  bool force_plain_ = false, full_table_ = false;
  int pot_mode_ = 0;
  // structure
  std::vector<int> hZ_;
  std::vector<float> hx_, hy_, hz_;
  Box box_{};
  bool have_atoms_ = false, have_index_ = false;
  int natoms_ = 0, nzb_ = 0;
  DevBuf<int> d_Zin_, d_off_, d_key_, d_idx_, d_cursor_, d_blocksum_;
  DevBuf<float> d_xin_, d_yin_, d_zin_;
  DevBuf<float4> d_atoms_;
  // table
  DevBuf<float> d_coef_;
  int nrows_fp_ = 0;
  bool have_fp_ = false;
  // separable potential: expansions [103][2][kGaussJ], per-atom tables of the
  // current slice, the loaded rows (FP64), per-row check (-1 not yet checked)
  static constexpr double kGaussTol = 2e-7;
  DevBuf<float> d_gauss_, d_tab_;
  DevBuf<float> d_tdsx_, d_tdsy_, d_tdsz_;  // displaced positions of a frozen-phonon batch
  DevBuf<float4> d_tds_atoms_;              // their atom indices [config][n], [config][nbins + 1]
  DevBuf<int> d_tds_off_;
  std::vector<double> hfp_;
  std::vector<float> hgauss_;
  std::vector<int> gauss_row_ok_;
  std::vector<char> zpresent_;
  int pot_sum_ = 0, last_pot_sum_ = 0;
  // microscope
  float kV_ = 0, df_ = 0, A2_ = 0, phi2_ = 0, Cs_ = 0, beta_ = 0, delta_ = 0, aperture_ = 0;
  bool have_micro_ = false;
  // calculation
  int nx_ = 0, ny_ = 0, nFD_ = 0, lbz_ = 3;
  float ps_ = 0, xoff_ = 0, yoff_ = 0, wavel_ = 0, sigma2_ = 0, dzFD_ = 0, kmax_ = 0, convdz_ = 1.0f;
  bool stem_ = false, have_calc_ = false, have_freq_ = false, fd_stable_ = false, fused_ok_ = false;
  std::vector<float> hkx_, hky_;
  DevBuf<float> d_kx_, d_ky_;
  DevBuf<float2> d_twx_[6], d_twy_[6], d_px_, d_py_, d_P_;
  int forced_plan_ = -1, ckpt_ = 0;
  float last_device_ms_ = 0.0f;
  // detector model of the noisy image chain
  DevBuf<float> d_dqe_, d_ntf_;
  int det_n_ = 0, det_bin_ = 4;
  float det_conv_ = 8.0f, det_ro_off_ = 4.0f, det_ro_sig_ = 1.33f;
  uint64_t det_seed_ = 0;
  uint32_t det_serial_ = 0;
  bool image_noisy_ = false;
  int pot_tile_ = -1;                    // tuned tile shape of the conventional potential (-1: not yet)
  bool pot_tile_forced_ = false;
  int rs_n_ = 0, rs_B_ = 1, rs_S_ = 0;  // prepared probe raster
  bool rs_loop_ = false;                 // its slices ran in the batched persistent loop
  bool rs_prefer_loop_ = true;           // tuned: batched loop (or per pass) for this grid's rasters
  float rs_kin2_ = 0, rs_kout2_ = 0;
  std::vector<int> hzoff_;  // first sorted atom per z-bin (focal-series atom gradient)
  DevBuf<float2> d_ck_, d_seg_, d_G_, d_U_, d_Phi_;
  DevBuf<float> d_T_, d_dV_, d_img_, d_fpstack_, d_fpdiff_, d_fpsum_, d_fpimg_;
  DevBuf<double> d_loss_, d_dxy_;
  std::vector<std::pair<int, PlanChoice>> tuned_;
  std::vector<std::pair<long long, int>> raster_batch_;  // tuned probes per launch by grid
  float prop_dz_ = -1.0f;
  cufftHandle plan_ = 0;
  bool have_plan_ = false;
  // waves
  DevBuf<float2> d_psi0_, d_psi_, d_psim_, d_t1_, d_t2_, d_grad_, d_fdX_, d_fdQ_, d_fdS_;
  bool fd_state_ = false;
  DevBuf<float> d_V_, d_f_, d_tds_, d_stack_;
  DevBuf<float2> d_tstack_;  // transmissions of the stack (probe rasters)
  bool tstack_valid_ = false;
  int tstack_S_ = 0;
  DevBuf<double> d_partial_, d_bsig_, d_bpart_;
  DevBuf<float2> d_bwave_;
  DevBuf<int> d_bpos_;
  int domain_ = 0;  // 0 real space, 1 row-frequency state of the fused passes,
                    // 2 fused finite differences (d_psi_ stale, X in d_fdX_)
  bool have_waves_ = false, stack_valid_ = false, have_tds_ = false, tds_host_valid_ = false;
  int nstack_ = 0;
  cudaGraphExec_t graph_exec_ = nullptr;
  // whole FD runs: resident band-limited planes and the captured step graph
  DevBuf<float> d_fdstack_;
  DevBuf<float2> d_fdstack_c_;
  bool fd_stack_valid_ = false, fd_stack_fused_ = false, capturing_ = false;
  int fd_nstack_ = 0;
  float fd_stack_dz_ = -1.0f;
  cudaGraphExec_t fd_graph_ = nullptr;
  int fd_graph_S_ = -1;
  const float* fd_graph_stack_ = nullptr;
  float2 *fd_graph_psi_ = nullptr, *fd_graph_psim_ = nullptr, *fd_graph_psi_end_ = nullptr,
         *fd_graph_psim_end_ = nullptr;
  // persistent slice loop: barrier state [count, error], pinned error copy
  DevBuf<unsigned int> d_loop_sync_;
  DevBuf<int> d_pass_err_;  // error word of the column pass's tensor-copy waits
  unsigned int* h_loop_err_ = nullptr;
  int loop_grid_ = 0, loop_grid_n_ = 0, loop_v_ = 0, forced_loop_ = -1, loop_tuned_for_ = -2;
  bool loop_off_ = false;
  unsigned int loop_extra_ = 0;
  unsigned long long loop_limit_ns_ = 1000000000ull;
  int graph_S_ = -1;
  const float* graph_stack_ = nullptr;  // stack allocation the graph was captured on
  // host read-out
  std::vector<float2> ew_;
  float ew_min_ = 0, ew_max_ = 0;
  bool have_ew_ = false;
  std::vector<float> image_, htds_;
  float im_min_ = 0, im_max_ = 0;
  bool have_image_ = false, have_image_buf_ = false;
};

}  // namespace ms

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct ms_sim {
  ms::Engine* e;
};

namespace {
thread_local std::string g_create_error;
}  // namespace

namespace ms {
// Failures of calls made without a handle (ms_create, the no-allocation
// index build) are reported by ms_last_error(NULL) on the calling thread.
void set_handle_free_error(const std::string& m) { g_create_error = m; }
}  // namespace ms

namespace {

template <class F>
ms_status guarded(ms_sim* s, F&& f) {
  if (!s || !s->e) return MS_ERR_INVALID;
  try {
    if (cudaSetDevice(s->e->device()) != cudaSuccess) return s->e->fail(MS_ERR_CUDA, "cudaSetDevice failed");
    return f(*s->e);
  } catch (const std::bad_alloc&) {
    return s->e->fail(MS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception& ex) {
    return s->e->fail(MS_ERR_INVALID, ex.what());
  }
}

ms_status out_check(ms_sim* s, const void* p) {
  if (!p) return s && s->e ? s->e->fail(MS_ERR_INVALID, "null output pointer") : MS_ERR_INVALID;
  return MS_OK;
}
}  // namespace

extern "C" {

const char* ms_version(void) { return "cudamultislice_b200 0.1 (sm_100a)"; }

ms_status ms_create(int device, ms_sim** out) {
  if (!out) return MS_ERR_INVALID;
  *out = nullptr;
  ms_sim* s = nullptr;
  try {
    s = new ms_sim{new ms::Engine(device)};
  } catch (const std::bad_alloc&) {
    g_create_error = "host allocation failed";
    return MS_ERR_NOMEM;
  }
  const int rc = s->e->init();
  if (rc != MS_OK) {
    g_create_error = s->e->err;
    delete s->e;
    delete s;
    return rc;
  }
  *out = s;
  return MS_OK;
}

ms_status ms_destroy(ms_sim* s) {
  if (!s) return MS_ERR_INVALID;
  delete s->e;
  delete s;
  return MS_OK;
}

const char* ms_last_error(const ms_sim* s) {
  if (!s || !s->e) return g_create_error.c_str();
  return s->e->err.c_str();
}

ms_status ms_set_option(ms_sim* s, int option, int value) {
  return guarded(s, [&](ms::Engine& e) { return e.set_option(option, value); });
}
ms_status ms_import_atoms(ms_sim* s, const char* path) {
  return guarded(s, [&](ms::Engine& e) { return e.import_atoms(path); });
}
ms_status ms_set_atoms(ms_sim* s, const int* Z, const float* x, const float* y, const float* z, int n) {
  return guarded(s, [&](ms::Engine& e) { return e.set_atoms(Z, x, y, z, n); });
}
ms_status ms_upload_binned_atoms(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.upload_binned(false, 0, 0, 0.0f); });
}
ms_status ms_upload_binned_atoms_tds(ms_sim* s, uint64_t seed, uint32_t pass, float sigma) {
  return guarded(s, [&](ms::Engine& e) { return e.upload_binned(true, seed, pass, sigma); });
}
ms_status ms_get_parameterisation(ms_sim* s, const char* path) {
  return guarded(s, [&](ms::Engine& e) { return e.get_parameterisation(path); });
}
ms_status ms_apply_microscope_parameters(ms_sim* s, float kV, float df, float A2, float phi2, float Cs, float beta,
                                         float delta, float aperture) {
  return guarded(s, [&](ms::Engine& e) { return e.apply_microscope(kV, df, A2, phi2, Cs, beta, delta, aperture); });
}
ms_status ms_set_calculation_variables(ms_sim* s, float ps, float df, int nx, int ny, float sx, float sy, float sz,
                                       float xoff, float yoff) {
  (void)sx;
  (void)sy;
  return guarded(s, [&](ms::Engine& e) { return e.set_calc(ps, df, nx, ny, sz, xoff, yoff, false); });
}
ms_status ms_stem_set_calculation_variables(ms_sim* s, float ps, float df, int nx, int ny, float sx, float sy,
                                            float sz) {
  (void)sx;
  (void)sy;
  return guarded(s, [&](ms::Engine& e) { return e.set_calc(ps, df, nx, ny, sz, 0.0f, 0.0f, true); });
}
ms_status ms_precalculate_frequencies(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.precalc(); });
}
ms_status ms_initialise_wavefunctions(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.init_waves(-1.0f); });
}
ms_status ms_initialise_wavefunctions_dz(ms_sim* s, float dz) {
  return guarded(s, [&](ms::Engine& e) {
    if (!(dz > 0)) return e.fail(MS_ERR_INVALID, "slice thickness must be positive");
    return e.init_waves(dz);
  });
}
ms_status ms_stem_initialise_wavefunctions(ms_sim* s, int px, int py) {
  return guarded(s, [&](ms::Engine& e) { return e.stem_init_waves(px, py); });
}
ms_status ms_set_fd_dz(ms_sim* s, float dz) {
  return guarded(s, [&](ms::Engine& e) { return e.set_fd_dz(dz); });
}
ms_status ms_multislice_step_fd(ms_sim* s, int it) {
  return guarded(s, [&](ms::Engine& e) { return e.step_fd(it); });
}
ms_status ms_multislice_step_rs(ms_sim* s, int it) {
  return guarded(s, [&](ms::Engine& e) { return e.step_rs(it); });
}
ms_status ms_multislice_step_conventional(ms_sim* s, int it) {
  return guarded(s, [&](ms::Engine& e) { return e.step_conventional(it); });
}
ms_status ms_get_size_x(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_atoms()) return e.fail(MS_ERR_STATE, "no atoms");
    *out = e.box().MaxX - e.box().MinX;
    return (int)MS_OK;
  });
}
ms_status ms_get_size_y(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_atoms()) return e.fail(MS_ERR_STATE, "no atoms");
    *out = e.box().MaxY - e.box().MinY;
    return (int)MS_OK;
  });
}
ms_status ms_get_size_z(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_atoms()) return e.fail(MS_ERR_STATE, "no atoms");
    *out = e.box().MaxZ - e.box().MinZ;
    return (int)MS_OK;
  });
}
ms_status ms_get_slices(ms_sim* s, int conventional, int* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.get_slices(conventional != 0, out); });
}
ms_status ms_get_kmax(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_freq()) return e.fail(MS_ERR_STATE, "frequencies not precalculated");
    *out = e.kmax();
    return (int)MS_OK;
  });
}
ms_status ms_get_exit_wave(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.get_exit_wave(false); });
}
ms_status ms_get_stem_exit_wave(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.get_exit_wave(true); });
}
ms_status ms_free_exit_wave(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.free_exit_wave(); });
}
ms_status ms_get_ew_value_abs(ms_sim* s, int x, int y, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.ew_value(x, y, 0, out); });
}
ms_status ms_get_ew_value_re(ms_sim* s, int x, int y, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.ew_value(x, y, 1, out); });
}
ms_status ms_get_ew_value_im(ms_sim* s, int x, int y, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.ew_value(x, y, 2, out); });
}
ms_status ms_get_ew_min(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_ew()) return e.fail(MS_ERR_STATE, "exit wave not fetched (ms_get_exit_wave)");
    *out = e.ew_min();
    return (int)MS_OK;
  });
}
ms_status ms_get_ew_max(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_ew()) return e.fail(MS_ERR_STATE, "exit wave not fetched (ms_get_exit_wave)");
    *out = e.ew_max();
    return (int)MS_OK;
  });
}
ms_status ms_alloc_tds(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.alloc_tds(); });
}
ms_status ms_add_tds_waves(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.add_tds(); });
}
ms_status ms_get_tds_min(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.tds_query(0, 0, 0, out); });
}
ms_status ms_get_tds_max(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.tds_query(1, 0, 0, out); });
}
ms_status ms_get_tds_val(ms_sim* s, int x, int y, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.tds_query(2, x, y, out); });
}
ms_status ms_alloc_host_image(ms_sim* s) {
  return guarded(s, [&](ms::Engine& e) { return e.alloc_host_image(); });
}
ms_status ms_simulate_image(ms_sim* s, float dose) {
  (void)dose;
  return guarded(s, [&](ms::Engine& e) { return e.simulate_image(dose); });
}
ms_status ms_get_im_value(ms_sim* s, int x, int y, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.im_value(x, y, out); });
}
ms_status ms_get_dqe_im_value(ms_sim* s, int x, int y, float* out) {
  if (ms_status rc = out_check(s, out)) return rc;
  return guarded(s, [&](ms::Engine& e) { return e.dqe_im_value(x, y, out); });
}
ms_status ms_get_im_min(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_image()) return e.fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    *out = e.im_min();
    return (int)MS_OK;
  });
}
ms_status ms_get_im_max(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_image()) return e.fail(MS_ERR_STATE, "image not simulated (ms_simulate_image)");
    *out = e.im_max();
    return (int)MS_OK;
  });
}
ms_status ms_get_image_contrast(ms_sim* s, int t, int l, int b, int r, float* out) {
  if (ms_status rr = out_check(s, out)) return rr;
  return guarded(s, [&](ms::Engine& e) { return e.image_contrast(t, l, b, r, out); });
}
ms_status ms_copy_exit_wave(ms_sim* s, float* dst) {
  return guarded(s, [&](ms::Engine& e) { return e.copy_exit_wave(dst); });
}
ms_status ms_copy_image(ms_sim* s, float* dst) {
  return guarded(s, [&](ms::Engine& e) { return e.copy_image(dst); });
}
ms_status ms_copy_tds(ms_sim* s, float* dst) {
  return guarded(s, [&](ms::Engine& e) { return e.copy_tds(dst); });
}
ms_status ms_get_grid(ms_sim* s, int* nx, int* ny) {
  if (ms_status r = out_check(s, nx)) return r;
  if (ms_status r = out_check(s, ny)) return r;
  return guarded(s, [&](ms::Engine& e) {
    if (!e.have_freq()) return e.fail(MS_ERR_STATE, "frequencies not precalculated");
    *nx = e.nx();
    *ny = e.ny();
    return (int)MS_OK;
  });
}
ms_status ms_build_potential_stack(ms_sim* s, int* nslices) {
  return guarded(s, [&](ms::Engine& e) { return e.build_stack(nslices); });
}
ms_status ms_run_conventional(ms_sim* s, int* nslices) {
  return guarded(s, [&](ms::Engine& e) { return e.run_conventional(nslices); });
}
ms_status ms_get_raster_tuning(ms_sim* s, int* batch, int* persistent) {
  return guarded(s, [&](ms::Engine& e) { return e.raster_tuning(batch, persistent); });
}
ms_status ms_get_potential_sum(ms_sim* s, int* last, int* next) {
  return guarded(s, [&](ms::Engine& e) { return e.potential_sum_info(last, next); });
}
ms_status ms_get_slice_loop(ms_sim* s, int* variant, int* columns, int* grid) {
  return guarded(s, [&](ms::Engine& e) { return e.slice_loop_info(variant, columns, grid); });
}
ms_status ms_run_fd(ms_sim* s, int nsteps, int* nsteps_out) {
  return guarded(s, [&](ms::Engine& e) { return e.run_fd(nsteps, nsteps_out); });
}
ms_status ms_annular_detector(ms_sim* s, float inner, float outer, double* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.annular(inner, outer, out); });
}
ms_status ms_stem_raster(ms_sim* s, const int* px, const int* py, int n, float inner, float outer, int batch,
                         double* signal) {
  return guarded(s, [&](ms::Engine& e) { return e.stem_raster(px, py, n, inner, outer, batch, signal); });
}
ms_status ms_get_binned_counts(ms_sim* s, int* n, int* nz) {
  if (ms_status r = out_check(s, n)) return r;
  if (ms_status r = out_check(s, nz)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.binned_counts(n, nz); });
}
ms_status ms_copy_binned(ms_sim* s, int* off, int* Z, float* x, float* y, float* z) {
  if (!off || !Z || !x || !y || !z) return s && s->e ? s->e->fail(MS_ERR_INVALID, "null destination") : MS_ERR_INVALID;
  return guarded(s, [&](ms::Engine& e) { return e.copy_binned(off, Z, x, y, z); });
}
ms_status ms_copy_potential_slice(ms_sim* s, int kind, int it, float* dst) {
  if (ms_status r = out_check(s, dst)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.copy_potential(kind, it, dst); });
}
ms_status ms_fft2(ms_sim* s, const float* in, float* out, int nx, int ny, int sign) {
  if (!in || !out) return s && s->e ? s->e->fail(MS_ERR_INVALID, "null buffer") : MS_ERR_INVALID;
  return guarded(s, [&](ms::Engine& e) { return e.fft2_host(in, out, nx, ny, sign); });
}
ms_status ms_time_slices(ms_sim* s, int steps, int reps, float* total, float* row, float* col) {
  if (!total) return s && s->e ? s->e->fail(MS_ERR_INVALID, "null output") : MS_ERR_INVALID;
  return guarded(s, [&](ms::Engine& e) { return e.time_slices(steps, reps, total, row, col); });
}
ms_status ms_get_fft_plan(ms_sim* s, int batch, int* row, int* col) {
  if (!row || !col) return s && s->e ? s->e->fail(MS_ERR_INVALID, "null output") : MS_ERR_INVALID;
  return guarded(s, [&](ms::Engine& e) { return e.fft_plan(batch, row, col); });
}
ms_status ms_focal_series(ms_sim* s, const float* defoci, int nd, const float* targets, int nslices, double* loss,
                          float* images) {
  return guarded(s, [&](ms::Engine& e) {
    return e.focal(defoci, nd, targets, nslices, loss, images, nullptr, nullptr, false);
  });
}
ms_status ms_focal_series_grad(ms_sim* s, const float* defoci, int nd, const float* targets, int nslices,
                               double* loss, float* dLdV, double* dLdxy) {
  return guarded(s, [&](ms::Engine& e) {
    return e.focal(defoci, nd, targets, nslices, loss, nullptr, dLdV, dLdxy, true);
  });
}
ms_status ms_time_pass(ms_sim* s, int pass, int op, int variant, int batch, int reps, float* us) {
  if (ms_status r = out_check(s, us)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.time_pass(pass, op, variant, batch, reps, us); });
}
ms_status ms_write_tiff(ms_sim* s, int what, const char* path) {
  return guarded(s, [&](ms::Engine& e) { return e.write_tiff(what, path); });
}
ms_status ms_write_tiff_f32(const char* path, const float* data, int nx, int ny) {
  const int rc = ms::write_tiff_f32(path, data, nx, ny);
  if (rc == 1) {
    ms::set_handle_free_error("ms_write_tiff_f32: bad arguments");
    return MS_ERR_INVALID;
  }
  if (rc != 0) {
    ms::set_handle_free_error(std::string("ms_write_tiff_f32: cannot write ") + path);
    return MS_ERR_IO;
  }
  return MS_OK;
}
ms_status ms_set_detector(ms_sim* s, const float* dqe, const float* ntf, int n, int binning, float conversion,
                          float readout_offset, float readout_sigma, uint64_t seed) {
  return guarded(s, [&](ms::Engine& e) {
    return e.set_detector(dqe, ntf, n, binning, conversion, readout_offset, readout_sigma, seed);
  });
}
ms_status ms_simulate_image_series(ms_sim* s, const float* defoci, const float* cs, int n, float* images) {
  return guarded(s, [&](ms::Engine& e) { return e.image_series(defoci, cs, n, images); });
}
ms_status ms_frozen_phonon(ms_sim* s, uint64_t seed, uint32_t first_pass, int nconfigs, float sigma, int batch,
                           float* diffraction, float* image) {
  return guarded(s, [&](ms::Engine& e) {
    return e.frozen_phonon(seed, first_pass, nconfigs, sigma, batch, diffraction, image);
  });
}
ms_status ms_get_last_device_ms(ms_sim* s, float* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) { return e.last_device_ms(out); });
}
// Several handles' probe rasters (different specimens and grid sizes, one
// device) captured into one CUDA graph: one branch per handle on its own
// stream, forked from and joined into the first handle's stream, launched once.
ms_status ms_stem_raster_concurrent(ms_sim* const* sims, int nsims, const int* const* px, const int* const* py,
                                    const int* n, float inner_mrad, float outer_mrad, int batch,
                                    double* const* signal) {
  if (!sims || nsims < 1 || !px || !py || !n || !signal) return MS_ERR_INVALID;
  for (int k = 0; k < nsims; ++k)
    if (!sims[k] || !sims[k]->e) return MS_ERR_INVALID;
  return guarded(sims[0], [&](ms::Engine& e0) -> int {
    for (int k = 0; k < nsims; ++k) {
      ms::Engine& e = *sims[k]->e;
      if (e.device() != e0.device()) return e0.fail(MS_ERR_INVALID, "all handles must use the same device");
      if (!e.fused()) return e0.fail(MS_ERR_UNSUPPORTED, "every handle must run the fused passes");
      if (!signal[k]) return e0.fail(MS_ERR_INVALID, "null signal buffer");
      if (int rc = e.raster_prepare(px[k], py[k], n[k], inner_mrad, outer_mrad, batch))
        return e0.fail(rc, "handle " + std::to_string(k) + ": " + e.err);
    }
    cudaStream_t st0 = e0.stream();
    // Two handles whose grids the batched persistent loop serves, with equal
    // slice counts: each round takes the next batch of both rasters through
    // every slice in ONE cooperative launch (group 0 the larger grid), on the
    // first handle's stream.
    if (nsims == 2 && sims[0]->e->use_batch_loop() && sims[1]->e->use_batch_loop() &&
        sims[0]->e->raster_prefers_loop() && sims[1]->e->raster_prefers_loop() &&
        sims[0]->e->raster_slices() == sims[1]->e->raster_slices()) {
      const int big = sims[0]->e->grid_n() >= sims[1]->e->grid_n() ? 0 : 1;
      ms::Engine& ea = *sims[big]->e;
      ms::Engine& eb = *sims[1 - big]->e;
      if (ms::batch_loop_supported(ea.grid_n(), eb.grid_n())) {
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) {
          if (t0) cudaEventDestroy(t0);
          return e0.fail(MS_ERR_CUDA, "cudaEventCreate failed");
        }
        int rc = MS_OK;
        cudaError_t ce = cudaEventRecord(t0, st0);
        if (ce == cudaSuccess) rc = ea.raster_begin(st0);
        if (rc == MS_OK) rc = eb.raster_begin(st0);
        if (rc == MS_OK) rc = e0.loop_begin(st0);
        const int na = ea.raster_count(), nb = eb.raster_count(), Ba = ea.raster_batch(), Bb = eb.raster_batch();
        for (int r = 0; ce == cudaSuccess && rc == MS_OK; ++r) {
          const int sa = r * Ba, sb = r * Bb;
          const int ka = std::max(0, std::min(Ba, na - sa)), kb = std::max(0, std::min(Bb, nb - sb));
          if (ka == 0 && kb == 0) break;
          if (ka > 0) rc = ea.raster_probes(st0, sa, ka);
          if (rc == MS_OK && kb > 0) rc = eb.raster_probes(st0, sb, kb);
          if (rc != MS_OK) break;
          if (ka > 0 && kb > 0) {
            const ms::LoopGroup g0 = ea.raster_group(sa, ka), g1 = eb.raster_group(sb, kb);
            rc = e0.enqueue_batch_loop(st0, g0, &g1, ea.raster_slices());
          } else {
            const ms::LoopGroup g0 = ka > 0 ? ea.raster_group(sa, ka) : eb.raster_group(sb, kb);
            rc = e0.enqueue_batch_loop(st0, g0, nullptr, ea.raster_slices());
          }
        }
        if (ce == cudaSuccess && rc == MS_OK) ce = cudaEventRecord(t1, st0);
        if (ce == cudaSuccess && rc == MS_OK) rc = e0.loop_check(st0);
        float ms = 0.0f;
        if (ce == cudaSuccess && rc == MS_OK && cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess)
          e0.set_last_device_ms(ms);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (rc != MS_OK) return rc;
        if (ce != cudaSuccess) return e0.fail(MS_ERR_CUDA, std::string("mixed raster: ") + cudaGetErrorString(ce));
        for (int k = 0; k < nsims; ++k) {
          ms::Engine& e = *sims[k]->e;
          if (int r2 = e.raster_finish(signal[k])) return e0.fail(r2, "handle " + std::to_string(k) + ": " + e.err);
        }
        return (int)MS_OK;
      }
    }
    std::vector<cudaEvent_t> ev(nsims + 2, nullptr);
    for (auto& x : ev)
      if (cudaEventCreate(&x) != cudaSuccess) {
        for (auto& y : ev)
          if (y) cudaEventDestroy(y);
        return e0.fail(MS_ERR_CUDA, "cudaEventCreate failed");
      }
    auto cleanup = [&]() {
      for (auto& y : ev) cudaEventDestroy(y);
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(st0, cudaStreamCaptureModeThreadLocal);
    int rc = MS_OK;
    if (ce == cudaSuccess) {
      ce = cudaEventRecord(ev[0], st0);
      for (int k = 1; k < nsims && ce == cudaSuccess; ++k) ce = cudaStreamWaitEvent(sims[k]->e->stream(), ev[0], 0);
      for (int k = 0; k < nsims && ce == cudaSuccess && rc == MS_OK; ++k) {
        ms::Engine& e = *sims[k]->e;
        rc = e.raster_enqueue(e.stream());
        if (rc != MS_OK) rc = e0.fail(rc, "handle " + std::to_string(k) + ": " + e.err);
      }
      for (int k = 1; k < nsims && ce == cudaSuccess; ++k) {
        ce = cudaEventRecord(ev[k], sims[k]->e->stream());
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st0, ev[k], 0);
      }
      const cudaError_t ee = cudaStreamEndCapture(st0, &graph);
      if (ce == cudaSuccess) ce = ee;
    }
    if (ce == cudaSuccess && rc == MS_OK) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    // ev[0]: fork, ev[1..nsims-1]: joins, ev[nsims], ev[nsims+1]: timing
    if (ce == cudaSuccess && rc == MS_OK) {
      ce = cudaEventRecord(ev[nsims], st0);
      if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, st0);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev[nsims + 1], st0);
    }
    if (exec) {
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st0);
      cudaGraphExecDestroy(exec);
    }
    if (ce == cudaSuccess && rc == MS_OK) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, ev[nsims], ev[nsims + 1]) == cudaSuccess) e0.set_last_device_ms(ms);
    }
    cleanup();
    if (rc != MS_OK) return rc;
    if (ce != cudaSuccess) return e0.fail(MS_ERR_CUDA, std::string("concurrent raster graph: ") + cudaGetErrorString(ce));
    for (int k = 0; k < nsims; ++k) {
      ms::Engine& e = *sims[k]->e;
      if (int r2 = e.raster_finish(signal[k])) return e0.fail(r2, "handle " + std::to_string(k) + ": " + e.err);
    }
    return (int)MS_OK;
  });
}

ms_status ms_get_launch_count(ms_sim* s, long long* out) {
  if (ms_status r = out_check(s, out)) return r;
  return guarded(s, [&](ms::Engine& e) {
    *out = e.launches;
    return (int)MS_OK;
  });
}

}  // extern "C"
