/*
 * ms_oracle.h -- C interface of the FP64 CPU oracle for the multislice hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA engine
 * (cudamultislice_b200) is compared against.  Only tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py may load it; the product never does.
 *
 * It restates the reference engine GUI Simulation/UnmanagedGUISimulation.cu
 * (class UnmanagedMultisliceSimulation, unmanagedGUISimulation.cuh:62-200) on the
 * CPU.  Rules of the restatement:
 *   - every VALUE (potentials, FFTs, propagation, imaging) is computed in FP64;
 *   - every DISCRETE DECISION the reference takes in FP32 (atom bins, z-bin
 *     windows, r^2 < 5 cutoffs, apertures, band limits) and every set-up scalar
 *     the reference computes on the host in FP32 (wavelength, interaction
 *     constant, finite-difference dz, frequencies, kmax, slice planes) is
 *     evaluated with the same FP32 operations in the same order, without FMA
 *     contraction, so that the oracle and the engine agree on the problem and
 *     differ only in arithmetic precision.
 * Parity of this oracle is pinned by known-answer tests (tests/test_oracle.py)
 * and by golden vectors generated from the reference itself (tests/golden/).
 */
#ifndef MS_ORACLE_H
#define MS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_sim or_sim;

/* ---- scalar building blocks (U.cu:41-193) ---- */
double or_bessi0(double x);
double or_bessk0(double x);
/* fparams: 103x12 table, row Z-1 */
double or_vzatom2(const double* fparams, int Z, double r2);
double or_vatom(const double* fparams, int Z, double r2);
int or_parse_fparams(const char* path, double* out /* 103*12 */, int* nrows);

/* ---- FFT (FP64, any size; sign -1 = forward as cuFFT FORWARD) ---- */
int or_fft1d(double* data /* 2n interleaved */, int n, int sign);
int or_fft2d(double* data /* 2*nx*ny */, int nx, int ny, int sign);

/* ---- Philox4x32-10 (Salmon et al., SC'11) and thermal displacements ---- */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void or_tds_displace(const float* x, const float* y, const float* z, int n,
                     uint64_t seed, uint32_t pass, float sigma,
                     float* xo, float* yo, float* zo);

/* ---- element table (U.cu:1188-1243 or full periodic table) ---- */
int or_znum(const char* symbol, int full_table);

/* ---- simulation object mirroring UnmanagedMultisliceSimulation ---- */
or_sim* or_create(void);
void or_destroy(or_sim*);
const char* or_last_error(or_sim*);
int or_set_threads(int n);

int or_import_atoms(or_sim*, const char* path, int full_table);      /* U.cu:1293-1356 */
int or_set_atoms(or_sim*, const int* Z, const float* x, const float* y,
                 const float* z, int n);                             /* box as U.cu:1333-1355 */
int or_get_box(or_sim*, float out[6]);  /* MaxX MinX MaxY MinY MaxZ MinZ */
int or_load_fparams(or_sim*, const char* path);                      /* U.cu:1718-1747 */
int or_bin_atoms(or_sim*);                                           /* U.cu:1358-1536 */
int or_bin_atoms_tds(or_sim*, uint64_t seed, uint32_t pass, float sigma);  /* U.cu:1538-1716 */
int or_get_binned_counts(or_sim*, int* n_atoms, int* n_zbins);
int or_get_binned(or_sim*, int* offsets, int* Z, float* x, float* y, float* z);

int or_apply_microscope(or_sim*, float kV, float df, float A2, float phi2,
                        float Cs, float beta, float delta, float aperture);  /* U.cu:1749-1761 */
int or_set_calc(or_sim*, float ps, float df, int nx, int ny, float sx, float sy,
                float sz, float xoff, float yoff, int stem);         /* U.cu:1763-1875 / 2567-2670 */
int or_precalc(or_sim*);                                             /* U.cu:1877-1964 */
/* scalars: [0] wavel [1] sigma2 [2] dzFD [3] nFD [4] kmax [5] ke2
            [6] conventional dz [7] n conventional slices [8] loadblocksx [9] loadblocksy */
int or_get_scalars(or_sim*, double out[10]);
int or_get_frequencies(or_sim*, float* kx, float* ky);

int or_init_waves(or_sim*, float conv_dz);    /* conv_dz <= 0: U.cu:1966 (dz=1), else U.cu:2003 */
int or_stem_init_waves(or_sim*, int px, int py);                     /* U.cu:2672-2724 */
int or_set_fd_dz(or_sim*, float dz);          /* override the automatic stable FD step */

/* potentials for one slice: out = N doubles (pre-exponential V) */
int or_potential_conventional(or_sim*, int iteration, double* out);  /* binnedAtomPKernel3 U.cu:582-653 */
int or_potential_fd(or_sim*, int iteration, double* out);            /* binnedAtomPKernelFD U.cu:883-946 */
int or_potential_projected(or_sim*, int iteration, float dz, double* out); /* vzatom2 slab mode */
int or_potential_rs(or_sim*, int iteration, double* out);            /* binnedAtomPKernelRS U.cu:655-727 */

int or_step_conventional(or_sim*, int iteration);                    /* U.cu:2085-2124 */
int or_cache_potentials(or_sim*, int on); /* reuse conventional V across probes (test speed only) */
int or_step_given_potential(or_sim*, int iteration, const double* V); /* the step without the potential build */
int or_step_projected(or_sim*, int iteration);                       /* same step, projected V */
int or_step_fd(or_sim*, int iteration);                              /* U.cu:2040-2083 */
int or_step_rs(or_sim*, int iteration);                              /* U.cu:2126-2178, as written */
int or_get_wave(or_sim*, double* out /* 2N */);
int or_set_wave(or_sim*, const double* in /* 2N */);

int or_simulate_image(or_sim*, double* out /* N intensity */);       /* U.cu:2311-2343 */
int or_alloc_tds(or_sim*);                                           /* U.cu:2726-2732 */
int or_add_tds(or_sim*);                                             /* U.cu:2734-2766 */
int or_get_tds(or_sim*, double* out /* N */);
/* annular detector: sum over inner<=theta<outer (mrad) of |FFT(psi)/sqrt(N)|^2 */
int or_annular_detector(or_sim*, float inner_mrad, float outer_mrad, double* out);
/* diffraction intensity |FFT(psi)/sqrt(N)|^2 (unshifted) */
int or_diffraction(or_sim*, double* out);

/* Differentiable focal series (no reference counterpart): loss
 * sum_d sum_px (|B_d psi_S|^2 - T_d)^2 over conventional slices 1..S from the
 * initial wave.  Vstack (S*N) replaces the computed potentials when not NULL. */
int or_focal_forward(or_sim*, const float* defoci, int nd, const double* targets, const double* Vstack,
                     int S, double* loss, double* images);
/* FP64 adjoint: dLdV (S*N) and dLdxy (2 per atom, input order, box fixed). */
int or_focal_grad(or_sim*, const float* defoci, int nd, const double* targets, int S, double* loss,
                  double* dLdV, double* dLdxy);
/* Detector chain of SimulateImage (U.cu:2345-2437) on an FP64 CTF intensity I. */
int or_detector_chain(or_sim*, const double* I, float dose, uint32_t serial, const float* dqe, const float* ntf,
                      int n, int binning, float conversion, uint64_t seed, double* out);
/* The clipped standard normal of the noise (Box-Muller as U.cu:2389-2397). */
double or_clipped_normal(uint32_t r1, uint32_t r2);
/* Test hook: value-only position offset of atom i (decisions unchanged). */
int or_set_value_offset(or_sim*, int i, double dx, double dy);

#ifdef __cplusplus
}
#endif
#endif
