// ms_slice_loop.cu -- launch of the persistent slice-loop kernel
// (ms_slice_loop.cuh) for square grids of 256, 512 and 1024 points.
#include "ms_slice_loop.cuh"

namespace ms {

namespace {

template <int N, int V>
using LoopPL = typename PlanSel<N, LoopPlan<N, (LoopVariant<V>::NT > 256)>::V>::T;


template <int N, int V>
cudaError_t loop_prepare(int* grid) {
  using PL = LoopPL<N, V>;
  using LV = LoopVariant<V>;
  using SH = LoopShape<PL, LV::CW, LV::NT>;
  static_assert(PL::P * LV::NT == 32 * 256 || PL::P * LV::NT == 64 * 512, "plan and CTA size must match");
  auto kernel = k_slice_loop<PL, LV::CW, LV::TIGHT, LV::NT, LV::FENCED>;
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
  using PL = LoopPL<N, V>;
  using LV = LoopVariant<V>;
  using SH = LoopShape<PL, LV::CW, LV::NT>;
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
  return cudaLaunchKernelEx(&cfg, k_slice_loop<PL, LV::CW, LV::TIGHT, LV::NT, LV::FENCED>, L);
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

bool slice_loop_supported(int nx, int ny) { return nx == ny && (nx == 256 || nx == 512 || nx == 1024); }

int slice_loop_plan(int n, int variant) {
  const bool wide = variant >= 5 && variant <= 7;
  switch (n) {
    case 256: return wide ? LoopPlan<256, true>::V : LoopPlan<256, false>::V;
    case 512: return wide ? LoopPlan<512, true>::V : LoopPlan<512, false>::V;
    case 1024: return wide ? LoopPlan<1024, true>::V : LoopPlan<1024, false>::V;
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
    case 5: return LoopVariant<5>::CW;
    case 6: return LoopVariant<6>::CW;
    case 7: return LoopVariant<7>::CW;
    case 8: return LoopVariant<8>::CW;
    case 9: return LoopVariant<9>::CW;
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
    case 5: return prepare_v<5>(n, grid);
    case 6: return prepare_v<6>(n, grid);
    case 7: return prepare_v<7>(n, grid);
    case 8: return prepare_v<8>(n, grid);
    case 9: return prepare_v<9>(n, grid);
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
    case 5: return launch_v<5>(L, grid, s);
    case 6: return launch_v<6>(L, grid, s);
    case 7: return launch_v<7>(L, grid, s);
    case 8: return launch_v<8>(L, grid, s);
    case 9: return launch_v<9>(L, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---- batched loop ----
namespace {
template <int N>
using NarrowPL = typename PlanSel<N, LoopPlan<N, false>::V>::T;
constexpr int kBatchCW = 4;

template <int N0, int N1, bool TC>
cudaError_t batch_prepare_t(int* grid) {
  using PL0 = NarrowPL<N0>;
  using PL1 = NarrowPL<N1>;
  using SH = BatchShape<PL0, PL1, kBatchCW>;
  auto kernel = k_batch_loop<PL0, PL1, kBatchCW, TC>;
  static unsigned long long done = 0;
  if (cudaError_t e = set_smem_once(done, kernel, SH::SMEM)) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return e;
  if (cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return e;
  if (cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SH::NT, SH::SMEM)) return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  *grid = sms;
  return cudaSuccess;
}

template <int N0, int N1, bool TC>
cudaError_t batch_launch_t(const BatchLoopArgs& L, int grid, cudaStream_t s) {
  using PL0 = NarrowPL<N0>;
  using PL1 = NarrowPL<N1>;
  using SH = BatchShape<PL0, PL1, kBatchCW>;
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
  return cudaLaunchKernelEx(&cfg, k_batch_loop<PL0, PL1, kBatchCW, TC>, L);
}

// (n0, n1) -> instantiation; n1 = 0: one group (the second plan repeats the first)
template <class F>
cudaError_t by_pair(int n0, int n1, F&& f) {
  if (n1 == 0 || n1 == n0) {  // one grid size (one or two groups of it)
    if (n0 == 1024) return f(std::integral_constant<int, 1024>(), std::integral_constant<int, 1024>());
    if (n0 == 512) return f(std::integral_constant<int, 512>(), std::integral_constant<int, 512>());
    if (n0 == 256) return f(std::integral_constant<int, 256>(), std::integral_constant<int, 256>());
  } else {
    if (n0 == 1024 && n1 == 512) return f(std::integral_constant<int, 1024>(), std::integral_constant<int, 512>());
    if (n0 == 1024 && n1 == 256) return f(std::integral_constant<int, 1024>(), std::integral_constant<int, 256>());
    if (n0 == 512 && n1 == 256) return f(std::integral_constant<int, 512>(), std::integral_constant<int, 256>());
  }
  return cudaErrorInvalidValue;
}
}  // namespace

bool batch_loop_supported(int n0, int n1) {
  return ((n1 == 0 || n1 == n0) && (n0 == 256 || n0 == 512 || n0 == 1024)) ||
         (n0 == 1024 && (n1 == 512 || n1 == 256)) || (n0 == 512 && n1 == 256);
}

int batch_loop_plan(int n) {
  switch (n) {
    case 256: return LoopPlan<256, false>::V;
    case 512: return LoopPlan<512, false>::V;
    case 1024: return LoopPlan<1024, false>::V;
    default: return -1;
  }
}

cudaError_t batch_loop_prepare(int n0, int n1, bool tc, int* grid) {
  return by_pair(n0, n1, [&](auto a, auto b) {
    return tc ? batch_prepare_t<decltype(a)::value, decltype(b)::value, true>(grid)
              : batch_prepare_t<decltype(a)::value, decltype(b)::value, false>(grid);
  });
}

cudaError_t launch_batch_loop(const BatchLoopArgs& L, int grid, cudaStream_t s) {
  const int n0 = L.g[0].n, n1 = (L.g[1].n > 0 && L.g[1].B > 0) ? L.g[1].n : 0;
  if (L.S < 1 || grid < 1 || L.g[0].B < 1 || !batch_loop_supported(n0, n1)) return cudaErrorInvalidValue;
  const bool tc = L.g[0].Vstack == nullptr;
  for (int k = 0; k < (n1 ? 2 : 1); ++k) {
    const LoopGroup& g = L.g[k];
    // every group of a launch takes the same potential source
    if (!g.wave || (tc ? !g.tstack : !g.Vstack) || (tc && g.Vstack) || g.a.nx != g.n || g.a.ny != g.n ||
        g.b.nx != g.n || g.b.ny != g.n)
      return cudaErrorInvalidValue;
  }
  return by_pair(n0, n1, [&](auto a, auto b) {
    return tc ? batch_launch_t<decltype(a)::value, decltype(b)::value, true>(L, grid, s)
              : batch_launch_t<decltype(a)::value, decltype(b)::value, false>(L, grid, s);
  });
}

}  // namespace ms
