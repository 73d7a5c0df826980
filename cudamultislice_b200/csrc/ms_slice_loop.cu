// ms_slice_loop.cu -- launch of the persistent slice-loop kernel
// (ms_slice_loop.cuh) for square grids of 256, 512 and 1024 points.
#include "ms_slice_loop.cuh"

namespace ms {

namespace {

template <int N>
using LoopPL = typename PlanSel<N, LoopPlan<N>::V>::T;

template <int N, int V>
cudaError_t loop_prepare(int* grid) {
  using PL = LoopPL<N>;
  using LV = LoopVariant<V>;
  using SH = LoopShape<PL, LV::CW>;
  static_assert(PL::P == 32, "loop plan must run one warp per line");
  auto kernel = k_slice_loop<PL, LV::CW, LV::TIGHT>;
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

template <int N, int V>
cudaError_t loop_launch(const LoopArgs& L, int grid, cudaStream_t s) {
  using PL = LoopPL<N>;
  using LV = LoopVariant<V>;
  using SH = LoopShape<PL, LV::CW>;
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
  return cudaLaunchKernelEx(&cfg, k_slice_loop<PL, LV::CW, LV::TIGHT>, L);
}

template <int V>
cudaError_t prepare_v(int n, int* grid) {
  switch (n) {
    case 256: return loop_prepare<256, V>(grid);
    case 512: return loop_prepare<512, V>(grid);
    case 1024: return loop_prepare<1024, V>(grid);
    default: return cudaErrorInvalidValue;
  }
}
template <int V>
cudaError_t launch_v(const LoopArgs& L, int grid, cudaStream_t s) {
  switch (L.a.nx) {
    case 256: return loop_launch<256, V>(L, grid, s);
    case 512: return loop_launch<512, V>(L, grid, s);
    case 1024: return loop_launch<1024, V>(L, grid, s);
    default: return cudaErrorInvalidValue;
  }
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

int slice_loop_variants() { return kLoopVariants; }

int slice_loop_columns(int variant) {
  switch (variant) {
    case 0: return LoopVariant<0>::CW;
    case 1: return LoopVariant<1>::CW;
    case 2: return LoopVariant<2>::CW;
    case 3: return LoopVariant<3>::CW;
    case 4: return LoopVariant<4>::CW;
    default: return 0;
  }
}

cudaError_t slice_loop_prepare(int n, int variant, int* grid) {
  switch (variant) {
    case 0: return prepare_v<0>(n, grid);
    case 1: return prepare_v<1>(n, grid);
    case 2: return prepare_v<2>(n, grid);
    case 3: return prepare_v<3>(n, grid);
    case 4: return prepare_v<4>(n, grid);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_slice_loop(const LoopArgs& L, int variant, int grid, cudaStream_t s) {
  if (L.a.nx != L.a.ny || L.b.nx != L.a.nx || L.b.ny != L.a.ny || L.S < 1 || grid < 1)
    return cudaErrorInvalidValue;
  switch (variant) {
    case 0: return launch_v<0>(L, grid, s);
    case 1: return launch_v<1>(L, grid, s);
    case 2: return launch_v<2>(L, grid, s);
    case 3: return launch_v<3>(L, grid, s);
    case 4: return launch_v<4>(L, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ms
