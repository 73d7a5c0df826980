// ref_symbol_fix.h -- force-included when compiling the reference engine
// (GUI Simulation/UnmanagedGUISimulation.cu) for the oracle-pinning build.
//
// The reference uploads its __constant__ parameters with the CUDA <= 4 form
// cudaMemcpyToSymbol("name", ...) (U.cu:1868-1873, 2663-2668).  Current CUDA
// resolves symbols only by address, so those calls fail silently and every
// kernel then sees zero-sized grids.  This header routes the string form to
// the symbol of that name; the reference source itself is compiled unchanged.
#pragma once
#include <cuda_runtime.h>
#include <cstring>

template <class A, class B, class C, class D, class E, class F>
static cudaError_t ms_ref_copy_to_symbol(const char* name, const void* src, size_t count, size_t offset, A& consts_,
                                         B& res_, C& maxs_, D& blocks_, E& grids_, F& bins_) {
  if (!std::strcmp(name, "consts")) return cudaMemcpyToSymbol(consts_, src, count, offset);
  if (!std::strcmp(name, "res")) return cudaMemcpyToSymbol(res_, src, count, offset);
  if (!std::strcmp(name, "maxs")) return cudaMemcpyToSymbol(maxs_, src, count, offset);
  if (!std::strcmp(name, "blocks")) return cudaMemcpyToSymbol(blocks_, src, count, offset);
  if (!std::strcmp(name, "grids")) return cudaMemcpyToSymbol(grids_, src, count, offset);
  if (!std::strcmp(name, "bins")) return cudaMemcpyToSymbol(bins_, src, count, offset);
  return cudaErrorInvalidSymbol;
}

#define cudaMemcpyToSymbol(sym, src, count, off) \
  ms_ref_copy_to_symbol(sym, src, count, off, consts, res, maxs, blocks, grids, bins)
