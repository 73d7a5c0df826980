// ms_noalloc.cu -- an atom-index build that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application whose memory
// manager owns every device allocation (a pooled allocator that forbids
// foreign cudaMalloc/cudaFree), or a latency-critical loop that cannot afford
// the implicit device-wide synchronisation of cudaMalloc/cudaFree.  For them this file provides
// ms_build_atom_index_noalloc: the bit-exact atom binning of
// ms_upload_binned_atoms, reading the atoms from and writing the index to
// device buffers the caller already owns.  Its scratch (bin keys, the
// permutation, per-bin cursors and scan partials) lives in one fixed
// file-scope device array, so nothing is allocated per call.
//
// Costs and limits of that choice:
//  - the array (kScratchInts ints, about 3.1 MB) is part of the module image:
//    every GPU that loads libmslice_b200.so holds it until the process exits;
//  - at most kMaxAtoms atoms and kMaxBins bins (z-bins x 2500) per call;
//  - every call uses the same array and leaves the last call's contents in
//    it.  The per-bin counters, which must start at zero, are cleared by each
//    call; calls whose GPU work overlaps (two streams, or two threads without
//    ordering) race on the array and corrupt each other's index;
//  - host code may not hand the array's name to a kernel (the name is only a
//    host-side stand-in); the device address is looked up once per device with
//    cudaGetSymbolAddress.  That look-up happens on the first call on each
//    device, so the first call on a device should come before any stream
//    capture.
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/mslice.h"
#include "ms_atoms.cuh"

namespace ms {
// Message store read by ms_last_error(NULL) (ms_engine.cu).
void set_handle_free_error(const std::string& m);

namespace {

constexpr int kMaxAtoms = 131072;
constexpr int kMaxBins = 524288;  // up to 209 one-angstrom z-bins of 50 x 50
constexpr int kMaxTileSums = (kMaxBins + 4095) / 4096 + 1;
constexpr size_t kScratchInts = 2 * (size_t)kMaxAtoms + kMaxBins + kMaxTileSums;

static __device__ __align__(256) int g_index_scratch[kScratchInts];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
int* g_addr[kMaxDevices] = {};

ms_status noalloc_fail(int code, const std::string& m) {
  set_handle_free_error(m);
  return code;
}

// Device address of g_index_scratch on the current device (looked up once).
int scratch_address(int** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(MS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(MS_ERR_UNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_index_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(MS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_addr[dev] = static_cast<int*>(p);
  }
  *out = g_addr[dev];
  return MS_OK;
}

}  // namespace
}  // namespace ms

extern "C" ms_status ms_build_atom_index_noalloc(const int* d_Z, const float* d_x, const float* d_y, const float* d_z,
                                                 int n, const float* box, float* d_atoms, int* d_offsets,
                                                 int offsets_capacity, int* nz_out, void* stream) {
  using namespace ms;
  if (!d_Z || !d_x || !d_y || !d_z || !box || !d_atoms || !d_offsets || !nz_out)
    return noalloc_fail(MS_ERR_INVALID, "null pointer argument");
  if (n < 1) return noalloc_fail(MS_ERR_INVALID, "need at least one atom");
  if (n > kMaxAtoms)
    return noalloc_fail(MS_ERR_INVALID, "ms_build_atom_index_noalloc: " + std::to_string(n) +
                                            " atoms exceed the fixed scratch limit of " + std::to_string(kMaxAtoms) +
                                            "; use ms_upload_binned_atoms");
  if (reinterpret_cast<uintptr_t>(d_atoms) % 16 != 0)
    return noalloc_fail(MS_ERR_INVALID, "d_atoms must be 16-byte aligned (float4 records)");
  Box b{box[0], box[1], box[2], box[3], box[4], box[5]};
  for (int i = 0; i < 6; ++i)
    if (!std::isfinite(box[i])) return noalloc_fail(MS_ERR_INVALID, "box entries must be finite");
  if (!(b.MaxX > b.MinX) || !(b.MaxY > b.MinY) || !(b.MaxZ >= b.MinZ))
    return noalloc_fail(MS_ERR_INVALID, "box must satisfy Max > Min in x and y, Max >= Min in z");
  // nSlices = ceil((MaximumZ-MinimumZ)/dz), dz = 1 (U.cu:1409-1411); the
  // z-bin count is checked against the scratch limit while still a float, so
  // the conversion to int below is always in range
  const float zext = std::ceil((b.MaxZ - b.MinZ) / (float)1);
  if (!(zext <= (float)(kMaxBins / kBins2)))
    return noalloc_fail(MS_ERR_INVALID, "ms_build_atom_index_noalloc: " + std::to_string(zext) +
                                            " z-bins exceed the fixed scratch limit of " +
                                            std::to_string(kMaxBins / kBins2) + "; use ms_upload_binned_atoms");
  int nz = (int)zext;
  nz += (nz == 0);
  const long long nbins = (long long)nz * kBins2;
  if ((long long)offsets_capacity < nbins + 1)
    return noalloc_fail(MS_ERR_INVALID, "d_offsets holds " + std::to_string(offsets_capacity) + " ints, need " +
                                            std::to_string(nbins + 1));
  int* scratch = nullptr;
  if (int rc = scratch_address(&scratch)) return rc;
  BinScratch scr{scratch, scratch + kMaxAtoms, scratch + 2 * kMaxAtoms, scratch + 2 * kMaxAtoms + kMaxBins};
  AtomIndex idx{reinterpret_cast<float4*>(d_atoms), d_offsets, 0, 0};
  cudaError_t e = build_atom_index(d_Z, d_x, d_y, d_z, n, b, nz, idx, scr, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return noalloc_fail(MS_ERR_CUDA, std::string("atom index launch: ") + cudaGetErrorString(e));
  *nz_out = nz;
  return MS_OK;
}
