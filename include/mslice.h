/*
 * mslice.h -- C ABI of the B200 multislice engine (libmslice_b200.so).
 *
 * This is the drop-in boundary for the reference's simulation class
 * UnmanagedMultisliceSimulation (GUI Simulation/unmanagedGUISimulation.cuh:62-200,
 * implemented in GUI Simulation/UnmanagedGUISimulation.cu, "U.cu" below), which
 * the reference exposes to .NET through ManagedMultisliceSimulation
 * (GUI Simulation/GUI Simulation.h:17-59, GUI Simulation/ManagedMultislice.cpp).
 * Each reference method has one entry point here, with the same argument
 * meaning and units, in the same call order:
 *
 *   import/set atoms -> upload binned atoms -> get parameterisation ->
 *   apply microscope parameters -> set calculation variables ->
 *   precalculate frequencies -> initialise wavefunctions ->
 *   step x S -> get exit wave -> (simulate image / add TDS waves)
 *
 * Conventions (differences from the reference are deliberate and listed):
 *  - Every function returns ms_status; MS_OK is 0.  The message of the last
 *    failure is ms_last_error().  (The reference reports no errors and calls
 *    exit(1) on a missing fparams.dat, U.cu:1730.)
 *  - Getters that return a float or int in the reference write through an
 *    out-pointer instead.
 *  - Buffers passed in are owned by the caller; the handle owns everything it
 *    allocates.  A handle is driven by one thread at a time and runs all its
 *    GPU work on its own non-default stream.
 *  - Plain pointers and sizes only; no CUDA or PyTorch types cross the ABI.
 */
#ifndef MSLICE_H
#define MSLICE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ms_sim ms_sim;
typedef int ms_status;

enum {
  MS_OK = 0,
  MS_ERR_INVALID = 1,     /* bad argument (size, index, NaN parameter) */
  MS_ERR_STATE = 2,       /* call order violated (e.g. stepping before initialising) */
  MS_ERR_CUDA = 3,        /* CUDA runtime / cuFFT failure */
  MS_ERR_IO = 4,          /* file missing or unreadable */
  MS_ERR_NOMEM = 5,       /* device or host allocation failed */
  MS_ERR_UNSUPPORTED = 6, /* combination not provided (e.g. fused path at this size) */
  MS_ERR_NUMERIC = 7      /* no stable finite-difference step (U.cu:1823-1830) */
};

/* Options (ms_set_option). */
enum {
  MS_OPT_SLICE_PATH = 0,    /* 0 = fused hand-written FFT passes (default where the
                               grid is a power of two 64..4096), 1 = plain path:
                               cuFFT + one kernel per operation, the reference's
                               launch sequence (U.cu:2101-2122) */
  MS_OPT_ELEMENT_TABLE = 1, /* 0 = reference symbol table, unknown -> Z=1 (U.cu:1188-1243);
                               1 = full periodic table Z = 1..103 */
  MS_OPT_POTENTIAL = 2,     /* 0 = conventional 3D-integrated potential, the live
                               reference kernel binnedAtomPKernel3 (U.cu:582-653);
                               1 = projected potential vzatom2 per slab (U.cu:119-152,
                               xy scan of binnedAtomPKernel2 U.cu:513-578) */
  MS_OPT_FFT_PLAN = 3,      /* -1 = autotuned (default): every FFT plan variant of the
                               fused passes is timed on the device once per grid and
                               batch size and the fastest kept; 0..5 = force a variant
                               (0: most points per thread ... 2: most threads per line;
                               3..5: 0..2 with butterflies on the packed FP32x2 pipe).
                               Variants agree to FP32 rounding, not bit for bit. */
  MS_OPT_CHECKPOINT = 4,    /* focal-series gradient: slices between stored waves;
                               0 = automatic (default): every wave when the S waves
                               fit in an eighth of the free device memory, else
                               ceil(sqrt(S)); 1 = store every wave; >= S = one
                               segment recomputed from the initial wave */
  MS_OPT_SLICE_LOOP = 5,    /* fused conventional slice loop (ms_run_conventional,
                               ms_time_slices) on square 256, 512 and 1024 grids:
                               0 = one persistent cooperative launch for all slices,
                               the phases separated by grid barriers (default);
                               1 = one launch per row and per column pass */
  MS_OPT_LOOP_WAIT_US = 6,  /* bound on each grid-barrier wait of the persistent slice
                               loop, microseconds (default 1,000,000); a wait that runs
                               out ends the launch and the call fails with MS_ERR_CUDA */
  MS_OPT_LOOP_WAIT_TEST = 7, /* test hook: > 0 makes every grid barrier wait for that many
                               arrivals more than the grid has, so the wait bound runs out
                               (0 = off, the default) */
  MS_OPT_LOOP_VARIANT = 8,  /* persistent slice loop kernel variant: -1 = tuned on the
                               device once per grid (default); 0..9 = force one: 0-4 run
                               lines of one warp in 256-thread CTAs (column units of 4, 8,
                               4, 8, 2 columns; barrier sleep-poll for 0-1, release
                               reduction with tight poll for 2-4); 5-7 lines of two warps
                               in 512-thread CTAs (units of 4, 2, 8 columns, tight poll);
                               8-9 as 3 and 2 with the ordering carried by the release
                               reduction and the acquire poll alone (no full fences) */
  MS_OPT_POTENTIAL_TILE = 9, /* conventional potential kernel tile: -1 = tuned on the device
                               per grid (default); per-sub-plane kernel 0, 1, 2 = 32 x 8,
                               16 x 16, 64 x 4 pixels; separable kernel 0..3 = 16 x 32,
                               32 x 16 (two pixels per thread), 16 x 64, 32 x 32 (four) */
  MS_OPT_POTENTIAL_SUM = 10, /* how the conventional potential sums an atom's 20 sub-planes
                               (binnedAtomPKernel3, U.cu:582-653): 0 = separable where it
                               applies (default), else per sub-plane; 1 = per (pixel, atom,
                               sub-plane), vatom evaluated term by term; 2 = separable, or
                               MS_ERR_UNSUPPORTED.  Separable: each element's vatom as 12
                               Gaussians in r^2 (checked against the loaded parameterisation
                               to 2e-7 of v on 0.25..2.2365 A), so that an atom's sub-plane
                               sum costs 12 exponentials per pixel; the same sub-planes pass
                               the reference's FP32 cut-off test as term by term. */
  MS_OPT_BUILD_OVERLAP = 11 /* ms_run_conventional when the potential stack must be built:
                               1 = run each slice's fused passes on a second stream while the
                               next slices' potentials are built (default; separable
                               potential, fused path); 0 = build the stack, then run the
                               slices.  Runs over a resident stack replay the persistent
                               loop either way. */
};

/* ---- lifecycle ---- */
/* Constructor U.cu:2551-2556 (creates the cuBLAS handle there; here a stream). */
ms_status ms_create(int device, ms_sim** out);
/* Destructor U.cu:2558-2561. */
ms_status ms_destroy(ms_sim* sim);
/* Message of the handle's last failure; with NULL, of the last failed call made
 * without a handle (ms_create, ms_build_atom_index_noalloc) on this thread. */
const char* ms_last_error(const ms_sim* sim);
const char* ms_version(void);
ms_status ms_set_option(ms_sim* sim, int option, int value);

/* ---- structure ---- */
/* LoadAtomFile U.cu:1293-1356 (.xyz: count, comment, "symbol x y z" rows; the
 * bounding box is padded by 2 A on every side). */
ms_status ms_import_atoms(ms_sim* sim, const char* path);
/* New: atoms by atomic number (the reference's symbol table lacks Ti, Ga, ...). */
ms_status ms_set_atoms(ms_sim* sim, const int* Z, const float* x, const float* y,
                       const float* z, int n);
/* UploadBinnedAtoms U.cu:1358-1536: bins of 50 x 50 in xy and 1 A in z, built
 * on the device, bit-identical to the reference's CSR. */
ms_status ms_upload_binned_atoms(ms_sim* sim);
/* UploadBinnedAtomsTDS U.cu:1538-1716: positions displaced by N(0, sigma^2)
 * per axis from a seeded counter-based generator (Philox4x32-10, counter =
 * (atom, pass)) instead of the unseeded rand() of TDSRand U.cu:29-37. */
ms_status ms_upload_binned_atoms_tds(ms_sim* sim, uint64_t seed, uint32_t pass, float sigma);
/* GetParameterisation U.cu:1718-1747, with the table path given explicitly
 * (the reference reads "fparams.dat" from the working directory). */
ms_status ms_get_parameterisation(ms_sim* sim, const char* path);

/* ---- microscope and set-up ---- */
/* ApplyMicroscopeParameters U.cu:1749-1761: kV, defocus (A), two-fold
 * astigmatism magnitude (A) and angle (rad), Cs (A), beta (mrad), delta (A),
 * objective aperture (mrad). */
ms_status ms_apply_microscope_parameters(ms_sim* sim, float kV, float df, float A2, float phi2,
                                         float Cs, float beta, float delta, float aperture);
/* SetCalculationVariables U.cu:1763-1875: pixel size (A), defocus, grid, the
 * structure size, and the offset (A) of pixel (0,0) from the box corner. */
ms_status ms_set_calculation_variables(ms_sim* sim, float ps, float df, int nx, int ny,
                                       float sx, float sy, float sz, float xoff, float yoff);
/* STEMSetCalculationVariables U.cu:2567-2670 (no offsets; FD step <= 0.06 A). */
ms_status ms_stem_set_calculation_variables(ms_sim* sim, float ps, float df, int nx, int ny,
                                            float sx, float sy, float sz);
/* PreCalculateFrequencies U.cu:1877-1964. */
ms_status ms_precalculate_frequencies(ms_sim* sim);

/* ---- wavefunction initialisation ---- */
/* InitialiseWavefunctions() U.cu:1966-2001 (conventional dz = 1 A). */
ms_status ms_initialise_wavefunctions(ms_sim* sim);
/* InitialiseWavefunctions(float dz) U.cu:2003-2038. */
ms_status ms_initialise_wavefunctions_dz(ms_sim* sim, float dz);
/* STEMInitialiseWavefunctions U.cu:2672-2724: probe at pixel (px, py). */
ms_status ms_stem_initialise_wavefunctions(ms_sim* sim, int px, int py);
/* New: override the automatic stable finite-difference step (U.cu:1815-1846). */
ms_status ms_set_fd_dz(ms_sim* sim, float dz);

/* ---- slice steps (iteration counts from 1, as the reference) ---- */
/* MultisliceStep U.cu:2040-2083 (finite differences). */
ms_status ms_multislice_step_fd(ms_sim* sim, int iteration);
/* MultisliceStepConv U.cu:2085-2124. */
ms_status ms_multislice_step_conventional(ms_sim* sim, int iteration);
/* MultisliceStepRS (U.cu:2126-2178; not exposed by the reference's managed
 * wrapper), as written: the real-space series of ten terms over the
 * un-exponentiated RS potential (binnedAtomPKernelRS U.cu:655-727, dz = 1,
 * ten sub-planes), with the reference's 5-point stencil (centre coefficient 1,
 * edge neighbours read at index 0), restarting from 1 every step; afterwards
 * the wave is the series result and, from the second iteration on, the
 * previous-level wave is that result times the previous wave. */
ms_status ms_multislice_step_rs(ms_sim* sim, int iteration);

/* ---- queries (ManagedMultislice.cpp:89-117) ---- */
ms_status ms_get_size_x(ms_sim* sim, float* out);
ms_status ms_get_size_y(ms_sim* sim, float* out);
ms_status ms_get_size_z(ms_sim* sim, float* out);
/* GetSlices(bool conventional), ManagedMultislice.cpp:105-111. */
ms_status ms_get_slices(ms_sim* sim, int conventional, int* out);
ms_status ms_get_kmax(ms_sim* sim, float* out);

/* ---- read-out ---- */
/* GetExitWave U.cu:2231-2284: exit wave to the handle's host buffer, with the
 * min/max |psi| (the reference finds them with cublasIsamin/Isamax). */
ms_status ms_get_exit_wave(ms_sim* sim);
/* GetSTEMExitWave U.cu:2180-2229: centred |FFT(psi)| kept as the exit wave. */
ms_status ms_get_stem_exit_wave(ms_sim* sim);
/* FreeExitWave U.cu:2286-2289. */
ms_status ms_free_exit_wave(ms_sim* sim);
/* GetEWValueAbs/Re/Im U.cu:2291-2304 and GetEWMin/Max ManagedMultislice.cpp:195-206. */
ms_status ms_get_ew_value_abs(ms_sim* sim, int x, int y, float* out);
ms_status ms_get_ew_value_re(ms_sim* sim, int x, int y, float* out);
ms_status ms_get_ew_value_im(ms_sim* sim, int x, int y, float* out);
ms_status ms_get_ew_min(ms_sim* sim, float* out);
ms_status ms_get_ew_max(ms_sim* sim, float* out);

/* AllocTDS U.cu:2726-2732 / AddTDSWaves U.cu:2734-2766 / GetTDSMin/Max/Val
 * U.cu:2768-2791: accumulated centred |FFT(psi_exit)| (kept on the device). */
ms_status ms_alloc_tds(ms_sim* sim);
ms_status ms_add_tds_waves(ms_sim* sim);
ms_status ms_get_tds_min(ms_sim* sim, float* out);
ms_status ms_get_tds_max(ms_sim* sim, float* out);
ms_status ms_get_tds_val(ms_sim* sim, int x, int y, float* out);

/* AllocHostImage U.cu:2306-2309 / SimulateImage U.cu:2311-2343: the CTF image
 * |IFFT(CTF * FFT(psi))|^2 (imagingKernel2 U.cu:1044-1080).  Without a detector
 * model (the default) that deterministic image is the result and `dose` is
 * unused.  With one (ms_set_detector) the detector chain of U.cu:2345-2437
 * follows: the DQE transfer (sqrt(DQE) on the image spectrum), |.|, shot noise
 * counts = round(dose a + sqrt(dose a) z) with `dose` electrons per pixel, the
 * NTF transfer times conversion^2, |.|; GetImValue (U.cu:2497-2512) then adds
 * readout noise offset + sigma z.  The reference draws z from unseeded rand();
 * here z is seeded Philox4x32-10 (per pixel and per simulated image), clipped
 * to +-3 as the reference does. */
ms_status ms_alloc_host_image(ms_sim* sim);
ms_status ms_simulate_image(ms_sim* sim, float dose);
ms_status ms_get_im_value(ms_sim* sim, int x, int y, float* out);
/* GetDQEImValue U.cu:2514-2517 (declared unmanagedGUISimulation.cuh:191): the
 * simulated image's magnitude at pixel (x, y), without GetImValue's readout
 * noise. */
ms_status ms_get_dqe_im_value(ms_sim* sim, int x, int y, float* out);
/* Detector model for ms_simulate_image (new; the reference compiles fixed K2
 * camera tables in, MTF.h): dqe[n], ntf[n] radial tables indexed by
 * floor(|frequency-pixel distance to the nearest corner| / binning), 0.0001
 * beyond the table (DQEFunc U.cu:1120-1132; the reference uses n = 725,
 * binning 4, conversion 8 counts per electron, readout noise 4 + 1.33 z);
 * seed for the shot and readout noise.  n = 0 removes the model. */
ms_status ms_set_detector(ms_sim* sim, const float* dqe, const float* ntf, int n, int binning, float conversion,
                          float readout_offset, float readout_sigma, uint64_t seed);
ms_status ms_get_im_min(ms_sim* sim, float* out);
ms_status ms_get_im_max(ms_sim* sim, float* out);
/* GetImageContrast (ManagedMultislice.cpp:207-210; computed at U.cu:2453-2491):
 * RMS contrast over rows [t, b) and columns [l, r) of the image. */
ms_status ms_get_image_contrast(ms_sim* sim, int t, int l, int b, int r, float* out);

/* ---- bulk read-out (new; replaces one managed call per pixel, MW.cs:314-321) ---- */
ms_status ms_copy_exit_wave(ms_sim* sim, float* dst /* 2*nx*ny, interleaved re/im */);
ms_status ms_copy_image(ms_sim* sim, float* dst /* nx*ny */);
ms_status ms_copy_tds(ms_sim* sim, float* dst /* nx*ny */);
ms_status ms_get_grid(ms_sim* sim, int* nx, int* ny);

/* ---- whole-run entry points (new) ---- */
/* Builds the potentials of slices 1..S into a device-resident stack (device
 * time of a build that ran in ms_get_last_device_ms).  The separable
 * potential's slices run on three streams of the handle (atom tables on a
 * fourth, at the highest stream priority); the call returns once the stack
 * is complete, and the result does not depend on the stream order. */
ms_status ms_build_potential_stack(ms_sim* sim, int* nslices);
/* Runs conventional slices 1..S from the initial wave (replayed as one
 * captured CUDA graph: on square 256, 512 and 1024 grids a single persistent
 * cooperative launch for all slices, MS_OPT_SLICE_LOOP); equivalent to
 * ms_multislice_step_conventional(i) for i = 1..S, the GUI's step loop
 * (CUDA Simulation GUI/MainWindow.xaml.cs:258-283). */
ms_status ms_run_conventional(ms_sim* sim, int* nslices);
/* Runs finite-difference steps 1..nsteps (nsteps <= 0: ms_get_slices(sim, 0,
 * ...)) from the initial waves: MultisliceStep (U.cu:2040-2083) as the GUI
 * loops over it (MainWindow.xaml.cs:258-283), equivalent to
 * ms_multislice_step_fd(i) for i = 1..nsteps.  The band-limited potential
 * planes are built once into a device-resident stack (rebuilt when the
 * structure, grid or FD step changes); the fused path then replays one
 * captured CUDA graph of two passes per step.  *nsteps_out (may be NULL)
 * receives the step count; device time in ms_get_last_device_ms. */
ms_status ms_run_fd(ms_sim* sim, int nsteps, int* nsteps_out);
/* Annular detector (no reference counterpart; the HAADF/ADF STEM signal):
 * sum over inner <= theta < outer (mrad) of |FFT(psi)|^2 / N. */
ms_status ms_annular_detector(ms_sim* sim, float inner_mrad, float outer_mrad, double* out);

/* STEM raster (new; the reference runs a single probe at the centre, with a
 * "TODO: loop over all stem positions" at CUDA Simulation GUI/MainWindow.xaml.cs:366):
 * for each probe position (px[i], py[i]) in pixels, the probe of
 * STEMInitialiseWavefunctions (U.cu:2672-2705), conventional slices 1..S over
 * the potential stack, and the annular-detector signal of ms_annular_detector,
 * written to signal[i].  Probes run `batch` at a time in one set of launches
 * (batch <= 0: automatic, tuned on the device once per grid size among 8 ... 64
 * probes per launch, at most what a quarter of the free memory holds). */
ms_status ms_stem_raster(ms_sim* sim, const int* px, const int* py, int n, float inner_mrad,
                         float outer_mrad, int batch, double* signal);

/* Float32 TIFF output (new; replaces the GUI's LibTiff.NET export,
 * CUDA Simulation GUI/MainWindow.xaml.cs:684-890, with the same fields: one
 * uncompressed strip of 32-bit IEEE floats, MinIsBlack, top-left, little-endian).
 * what: 0 the simulated image as ms_get_im_value reads it, 1 / 2 the exit wave's
 * real / imaginary part and 4 its amplitude (after ms_get_exit_wave), 3 the TDS /
 * CBED accumulation (ms_add_tds_waves). */
ms_status ms_write_tiff(ms_sim* sim, int what, const char* path);
/* The same TIFF of any nx * ny float array (row 0 at the top); errors are
 * reported by ms_last_error(NULL). */
ms_status ms_write_tiff_f32(const char* path, const float* data, int nx, int ny);

/* Batch Cs/defocus sweep of the current exit wave (new; the reference's GUI
 * leaves it as a stub, CUDA Simulation GUI/BatchProcessing.xaml.cs:131-134): image i
 * of images (n * nx * ny floats) is the ms_simulate_image CTF image at defocus
 * defoci[i] (A) and spherical aberration cs[i] (A; cs = NULL keeps the value
 * of ms_apply_microscope_parameters).  The slices are not re-run. */
ms_status ms_simulate_image_series(ms_sim* sim, const float* defoci, const float* cs, int n, float* images);

/* Frozen-phonon series (new; the reference's GUI loops UploadBinnedAtomsTDS,
 * the slices and AddTDSWaves over passes, CUDA Simulation GUI/MainWindow.xaml.cs:353-402):
 * configurations pass = first_pass .. first_pass + nconfigs - 1, each displaced as
 * ms_upload_binned_atoms_tds(seed, pass, sigma), run through conventional slices
 * 1..S from the initial wave (ms_initialise_wavefunctions_dz), `batch`
 * configurations at a time sharing every launch of the fused passes.
 * diffraction (nx*ny floats, may be NULL) = sum over configurations of
 * |centre(FFT(psi_exit))| as AddTDSWaves (U.cu:2734-2766); image (nx*ny floats,
 * may be NULL) = mean over configurations of the ms_simulate_image CTF image.
 * The handle's atom index is left at the last configuration. */
ms_status ms_frozen_phonon(ms_sim* sim, uint64_t seed, uint32_t first_pass, int nconfigs, float sigma, int batch,
                           float* diffraction, float* image);

/* ---- differentiable focal series (new; no reference counterpart) ----
 * Loss L = sum_d sum_px (I_d(px) - T_d(px))^2, with I_d the CTF image of
 * ms_simulate_image (imagingKernel2, U.cu:1044-1080, at the microscope
 * parameters of ms_apply_microscope_parameters except the defocus, which is
 * defoci[d] in A) of the exit wave after conventional slices 1..nslices from
 * the initial wave (ms_initialise_wavefunctions_dz).  targets: nd*nx*ny floats,
 * image d at offset d*nx*ny, row-major [y][x].  The wave is left at slice
 * nslices in the handle.  images (nd*nx*ny floats) may be NULL. */
ms_status ms_focal_series(ms_sim* sim, const float* defoci, int nd, const float* targets, int nslices,
                          double* loss, float* images);
/* Forward and adjoint of the same loss: dLdV = dL/dV for slices 1..nslices
 * (nslices*nx*ny floats, slice n-1 at offset (n-1)*nx*ny; V in the units of
 * ms_copy_potential_slice), dLdxy = dL/dx, dL/dy per atom in the order given to
 * ms_set_atoms / ms_import_atoms (2 doubles per atom, A^-1; the bounding box is
 * held fixed; needs the conventional potential).  Either may be NULL.  Waves
 * are recomputed from checkpoints every MS_OPT_CHECKPOINT slices. */
ms_status ms_focal_series_grad(ms_sim* sim, const float* defoci, int nd, const float* targets, int nslices,
                               double* loss, float* dLdV, double* dLdxy);

/* Several specimens' probe rasters in one CUDA-graph launch (batching of
 * mixed grid sizes; no reference counterpart): handle k (its own
 * specimen, grid and potentials; all handles on one device, fused path) runs
 * the raster of ms_stem_raster over its n[k] positions px[k], py[k] into
 * signal[k].  The handles' work is captured as concurrent branches of one graph
 * (one stream each, forked from and joined into sims[0]'s stream) and launched
 * once; ms_get_last_device_ms(sims[0]) then gives its device time.  Errors are
 * reported on sims[0]. */
ms_status ms_stem_raster_concurrent(ms_sim* const* sims, int nsims, const int* const* px, const int* const* py,
                                    const int* n, float inner_mrad, float outer_mrad, int batch,
                                    double* const* signal);

/* ---- inspection (parity tests and measurement) ---- */
/* Microseconds per launch of one fused pass on scratch waves (CUDA events,
 * `reps` back-to-back launches after two warm-up launches): pass 0 = row pass
 * with op = a combination of 1 (inverse row FFT), 2 (x exp(i sigma V)),
 * 512 (x a precomputed transmission, as the batched raster), 4 (forward row
 * FFT); pass 1 = column pass with op = 0 (forward column FFT),
 * 1 (inverse), 2 (propagate), 3 (CTF), 6 (band limit), 8 (adjoint propagate);
 * FFT plan `variant`, `batch` instances. */
ms_status ms_time_pass(ms_sim* sim, int pass, int op, int variant, int batch, int reps, float* us);
/* Device milliseconds (CUDA events on the handle's stream) of the last
 * focal-series call (from after the target upload to before the read-back),
 * frozen-phonon series, concurrent raster, ms_run_conventional (the slice
 * loop: one graph launch on the fused path) or potential-stack build. */
ms_status ms_get_last_device_ms(ms_sim* sim, float* out);
ms_status ms_get_binned_counts(ms_sim* sim, int* n_atoms, int* n_zbins);
ms_status ms_copy_binned(ms_sim* sim, int* offsets, int* Z, float* x, float* y, float* z);
/* kind: 0 conventional slice, 1 finite-difference plane, 2 projected slab (current
 * conventional dz), 3 RS plane (ms_multislice_step_rs) */
ms_status ms_copy_potential_slice(ms_sim* sim, int kind, int iteration, float* dst /* nx*ny */);
/* 2D FFT of a host array through the engine's own FFT passes (sign -1
 * forward, +1 inverse, unnormalised); grid must be fused-supported. */
ms_status ms_fft2(ms_sim* sim, const float* in, float* out, int nx, int ny, int sign);
/* Times `steps` fused (or plain) conventional steps over the resident
 * potential stack with CUDA events on the handle's stream, repeated `reps`
 * times; writes the total milliseconds and, when ms_row_pass and ms_col_pass
 * are not NULL, the per-launch averages of the two fused passes measured in a
 * second run of `steps` steps with an event between every pass. */
ms_status ms_time_slices(ms_sim* sim, int steps, int reps, float* ms_total, float* ms_row_pass,
                         float* ms_col_pass);
/* FFT plan variants (row pass, column pass) used for `batch` instances, tuning
 * them first if needed (MS_OPT_FFT_PLAN). */
ms_status ms_get_fft_plan(ms_sim* sim, int batch, int* row_variant, int* col_variant);
/* The last raster's probes per launch and whether its slices ran in the
 * batched persistent loop (1) or per pass (0); with batch <= 0 both are the
 * device-tuned choice. */
ms_status ms_get_raster_tuning(ms_sim* sim, int* batch, int* persistent);
/* The persistent slice loop this grid runs: kernel variant (-1 when the loop
 * does not run here), columns per column unit, CTAs (one per SM); tunes the
 * variant first if needed (MS_OPT_LOOP_VARIANT). */
ms_status ms_get_slice_loop(ms_sim* sim, int* variant, int* columns, int* grid);
/* Number of this library's kernels launched by the handle so far. */
ms_status ms_get_launch_count(ms_sim* sim, long long* out);
/* How the last conventional potential was summed (1 = per sub-plane,
 * 2 = separable, 0 = none built yet) and how the next one would be
 * (MS_OPT_POTENTIAL_SUM and the specimen's elements). */
ms_status ms_get_potential_sum(ms_sim* sim, int* last, int* next);

/* ---- atom index without device allocation (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc: an application whose memory manager
 * owns every device allocation, or a loop that cannot take cudaMalloc's
 * implicit device synchronisation.  Builds
 * the same bit-exact atom index as ms_upload_binned_atoms from atoms already on
 * the device (d_Z, d_x, d_y, d_z: n entries each) into caller-owned device
 * buffers: d_atoms (4*n floats, 16-byte aligned: x, y, z shifted by the box
 * minimum, then Z as int bits, sorted z-bin -> y-bin -> x-bin, input order within
 * a bin) and d_offsets (nz*2500 + 1 ints, offsets_capacity of them available).
 * `box` is a host array {MaxX, MinX, MaxY, MinY, MaxZ, MinZ} (LoadAtomFile's
 * padded box); nz = ceil(MaxZ - MinZ) one-angstrom z-bins is returned in *nz_out.
 * Work is enqueued on `stream` (a cudaStream_t, NULL for the default stream) and
 * the call returns without waiting.  Scratch is one fixed device array of about
 * 3.1 MB inside the library, held by every GPU that loads it until exit; limits:
 * n <= 131072 atoms and nz <= 209 z-bins, larger requests (and boxes with
 * non-finite entries) fail with MS_ERR_INVALID before any GPU work.  All calls share that array: calls whose GPU work overlaps
 * race and corrupt each other's result.  The first call on a device looks up the
 * array's device address, so make it before any stream capture.  Errors are
 * reported by ms_last_error(NULL). */
ms_status ms_build_atom_index_noalloc(const int* d_Z, const float* d_x, const float* d_y, const float* d_z,
                                      int n, const float* box, float* d_atoms, int* d_offsets,
                                      int offsets_capacity, int* nz_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MSLICE_H */
