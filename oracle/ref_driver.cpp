// ref_driver.cpp -- C entry points around the reference engine class, for the
// oracle-pinning build only (oracle/ref_build.sh -> oracle/_ref/libmsref.so).
//
// TEST INFRASTRUCTURE ONLY.  It drives the reference's own
// UnmanagedMultisliceSimulation (GUI Simulation/unmanagedGUISimulation.cuh,
// compiled unchanged from the reference tree) through the same call sequence
// as its GUI (CUDA Simulation GUI/MainWindow.xaml.cs:244-306, 353-402), and
// copies results out so tests/golden/make_golden_ref.py can store them as
// golden vectors.  Private members are opened only to read the atom index
// and the per-slice transmission the class keeps on the device.
//
// The reference source file is compiled inside this translation unit (it is
// included, not copied), so that the driver can also launch two of its
// kernels that no public method exposes on their own:
//  - imagingKernel2 (U.cu:1044-1080), the deterministic CTF transfer that
//    SimulateImage applies before its detector-noise chain (U.cu:2323-2333);
//  - binnedAtomPKernel2 (U.cu:513-578), the projected-potential kernel (vzatom2
//    over one one-angstrom z-bin), which no method of the class launches.
#include <cuComplex.h>
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include "UnmanagedGUISimulation.cu"
#undef private

extern "C" {

void* ref_create() { return new UnmanagedMultisliceSimulation(); }

void ref_import_atoms(void* h, const char* path) { ((UnmanagedMultisliceSimulation*)h)->LoadAtomFile(path); }

void ref_upload_binned(void* h) { ((UnmanagedMultisliceSimulation*)h)->UploadBinnedAtoms(); }

// Reads ./fparams.dat as the reference does (U.cu:1720).
void ref_get_parameterisation(void* h) { ((UnmanagedMultisliceSimulation*)h)->GetParameterisation(); }

void ref_apply(void* h, float kV, float df, float A2, float phi2, float Cs, float beta, float delta, float ap) {
  ((UnmanagedMultisliceSimulation*)h)->ApplyMicroscopeParameters(kV, df, A2, phi2, Cs, beta, delta, ap);
}

void ref_box(void* h, float* out6) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  out6[0] = s->MaximumX; out6[1] = s->MinimumX; out6[2] = s->MaximumY;
  out6[3] = s->MinimumY; out6[4] = s->MaximumZ; out6[5] = s->MinimumZ;
}

void ref_set_calc(void* h, float ps, float df, int nx, int ny, float xoff, float yoff, int stem) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  const float sx = s->MaximumX - s->MinimumX, sy = s->MaximumY - s->MinimumY, sz = s->MaximumZ - s->MinimumZ;
  if (stem) {
    s->STEMSetCalculationVariables(ps, df, nx, ny, sx, sy, sz);
    // STEMSetCalculationVariables leaves the block offsets unset (the
    // constructor never initialises them); the STEM path uses none.
    s->blockxoffset = 0.0f;
    s->blockyoffset = 0.0f;
  } else {
    s->SetCalculationVariables(ps, df, nx, ny, sx, sy, sz, xoff, yoff);
  }
}

void ref_precalc(void* h) { ((UnmanagedMultisliceSimulation*)h)->PreCalculateFrequencies(); }

void ref_init(void* h, float dz) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  if (dz > 0) s->InitialiseWavefunctions(dz); else s->InitialiseWavefunctions();
}

void ref_stem_init(void* h, int px, int py) { ((UnmanagedMultisliceSimulation*)h)->STEMInitialiseWavefunctions(px, py); }

int ref_slices(void* h, int conventional) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  if (conventional) return (int)std::ceil((s->MaximumZ - s->MinimumZ) / s->conventionaldz);  // ManagedMultislice.cpp:108
  return s->numberOfSlices;
}

void ref_scalars(void* h, float* out) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  out[0] = s->wavel; out[1] = s->sigma2; out[2] = s->dzFiniteDifference; out[3] = (float)s->numberOfSlices;
  out[4] = s->kmax; out[5] = s->conventionaldz;
}

void ref_step_conv(void* h, int i) { ((UnmanagedMultisliceSimulation*)h)->MultisliceStepConv(i); }
void ref_step_fd(void* h, int i) { ((UnmanagedMultisliceSimulation*)h)->MultisliceStep(i); }
// MultisliceStepRS (U.cu:2126-2178), a public method the managed wrapper does
// not expose; afterwards devV holds the RS potential {sumz, 0} of that step.
void ref_step_rs(void* h, int i) { ((UnmanagedMultisliceSimulation*)h)->MultisliceStepRS(i); }

// binnedAtomPKernel2 (U.cu:513-578) over one-angstrom z-bin `bin`: the kernel
// scans z-bin floor((MaxZ-MinZ-z)/dz) with an int dz, launched here with
// dz = 1 and z = (MaxZ-MinZ) - bin - 0.5, on the 32 x 8 blocks of every
// launch of the class.  Writes exp(i sigma2 V) as {cos, sin} to out (2n floats).
void ref_projected(void* h, int bin, float* out, int n) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  dim3 dimBlock(32, 8, 1);
  dim3 dimGrid((s->resolutionX + dimBlock.x - 1) / dimBlock.x, (s->resolutionY + dimBlock.y - 1) / dimBlock.y, 1);
  const float top = s->MaximumZ - s->MinimumZ;
  const float z = top - (float)bin - 0.5f;
  binnedAtomPKernel2<<<dimGrid, dimBlock>>>(s->devV, s->PixelScale, s->atomMemories.fparamsdev,
                                            s->atomMemories.devAtomZPos, s->atomMemories.devAtomXPos,
                                            s->atomMemories.devAtomYPos, s->atomMemories.devAtomZNum,
                                            s->atomMemories.devBlockStartPositions, 1, z, (int)std::ceil(top / 1.0f),
                                            s->sigma2, s->blockxoffset, s->blockyoffset);
  cudaMemcpy(out, s->devV, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost);
}

// The deterministic part of SimulateImage (U.cu:2323-2333): FFT(Psi),
// normalisingKernel, imagingKernel2 (objective aperture, CTF with Cs, df,
// two- and three-fold astigmatism, spatial and temporal coherence envelopes),
// inverse FFT, normalisingKernel.  Writes that complex image (2n floats); its
// squared modulus is the image before the detector chain.  Psi is unchanged.
void ref_ctf_image(void* h, float* out, int n) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  dim3 dimBlock(32, 8, 1);
  dim3 dimGrid((s->resolutionX + dimBlock.x - 1) / dimBlock.x, (s->resolutionY + dimBlock.y - 1) / dimBlock.y, 1);
  cuComplex *img = nullptr, *img2 = nullptr;
  cudaMalloc(&img, sizeof(cuComplex) * n);
  cudaMalloc(&img2, sizeof(cuComplex) * n);
  cufftExecC2C(s->plan, s->Psi, s->PsiPlus, CUFFT_FORWARD);
  normalisingKernel<<<dimGrid, dimBlock>>>(s->PsiPlus, s->normalisingfactor);
  imagingKernel2<<<dimGrid, dimBlock>>>(s->PsiPlus, s->resolutionX, s->resolutionY, s->Cs, s->df, s->Mod2fold,
                                        s->Arg2fold, s->Mod3fold, s->Arg3fold, s->objectiveAperture, s->wavel, img2,
                                        s->xFrequencies, s->yFrequencies, s->beta / 1000, s->delta);
  cufftExecC2C(s->plan, img2, img, CUFFT_INVERSE);
  normalisingKernel<<<dimGrid, dimBlock>>>(img, s->normalisingfactor);
  cudaMemcpy(out, img, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost);
  cudaFree(img);
  cudaFree(img2);
}

// The transmission function the last conventional step used (devV, U.cu:2101).
void ref_transmission(void* h, float* out, int n) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  cudaMemcpy(out, s->devV, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost);
}

// The current wave Psi without freeing anything (GetExitWave frees the scratch).
void ref_wave(void* h, float* out, int n) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  cudaMemcpy(out, s->Psi, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost);
}

// GetExitWave (U.cu:2231-2284): EW and the min/max |psi|.
void ref_exit_wave(void* h, float* out, int n, float* minmax) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  s->GetExitWave();
  std::memcpy(out, s->EW, sizeof(float) * 2 * n);
  minmax[0] = s->minposEW;
  minmax[1] = s->maxposEW;
  s->FreeExitWave();
}

void ref_alloc_tds(void* h) { ((UnmanagedMultisliceSimulation*)h)->AllocTDS(); }
void ref_add_tds(void* h) { ((UnmanagedMultisliceSimulation*)h)->AddTDSWaves(); }
void ref_tds(void* h, float* out, int n) {
  std::memcpy(out, ((UnmanagedMultisliceSimulation*)h)->TDS, sizeof(float) * n);
}

// The atom index built by UploadBinnedAtoms (U.cu:1520-1525).
void ref_binned(void* h, int n, int nbins, int* off, int* Z, float* x, float* y, float* z) {
  auto* s = (UnmanagedMultisliceSimulation*)h;
  cudaMemcpy(off, s->atomMemories.devBlockStartPositions, sizeof(int) * (nbins + 1), cudaMemcpyDeviceToHost);
  cudaMemcpy(Z, s->atomMemories.devAtomZNum, sizeof(int) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(x, s->atomMemories.devAtomXPos, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(y, s->atomMemories.devAtomYPos, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(z, s->atomMemories.devAtomZPos, sizeof(float) * n, cudaMemcpyDeviceToHost);
}

int ref_sync() { return (int)cudaDeviceSynchronize(); }
const char* ref_last_cuda_error() { return cudaGetErrorString(cudaGetLastError()); }

}  // extern "C"
