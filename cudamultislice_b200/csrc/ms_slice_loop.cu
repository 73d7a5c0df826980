// ms_slice_loop.cu -- launch of the persistent slice-loop kernel
// (ms_slice_loop.cuh) for square grids of 256, 512 and 1024 points.
#include "ms_slice_loop.cuh"

namespace ms {

namespace {

template <int N>
using LoopPL = typename PlanSel<N, LoopPlan<N>::V>::T;

template <int N>
cudaError_t loop_prepare(int* grid) {
  using PL = LoopPL<N>;
  using SH = LoopShape<PL, kLoopCW>;
  static_assert(PL::P == 32, "loop plan must run one warp per line");
  auto kernel = k_slice_loop<PL, kLoopCW>;
  static unsigned long long done = 0;
  if (cudaError_t e = set_smem_once(done, kernel, SH::SMEM)) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return e;
  if (cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return e;
  if (cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SH::NT, SH::SMEM)) return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  *grid = sms;  // one CTA per SM: every line of a phase has its own warp
  return cudaSuccess;
}

template <int N>
cudaError_t loop_launch(const LoopArgs& L, int grid, cudaStream_t s) {
  using PL = LoopPL<N>;
  using SH = LoopShape<PL, kLoopCW>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(SH::NT);
  cfg.dynamicSmemBytes = SH::SMEM;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_slice_loop<PL, kLoopCW>, L);
}

}  // namespace

int slice_loop_variant(int nx, int ny) {
  if (nx != ny) return -1;
  switch (nx) {
    case 256: return LoopPlan<256>::V;
    case 512: return LoopPlan<512>::V;
    case 1024: return LoopPlan<1024>::V;
    default: return -1;
  }
}

cudaError_t slice_loop_prepare(int n, int* grid) {
  switch (n) {
    case 256: return loop_prepare<256>(grid);
    case 512: return loop_prepare<512>(grid);
    case 1024: return loop_prepare<1024>(grid);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_slice_loop(const LoopArgs& L, int grid, cudaStream_t s) {
  if (L.a.nx != L.a.ny || L.b.nx != L.a.nx || L.b.ny != L.a.ny || L.S < 1 || grid < 1)
    return cudaErrorInvalidValue;
  switch (L.a.nx) {
    case 256: return loop_launch<256>(L, grid, s);
    case 512: return loop_launch<512>(L, grid, s);
    case 1024: return loop_launch<1024>(L, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ms
