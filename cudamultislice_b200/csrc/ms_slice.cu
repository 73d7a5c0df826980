// ms_slice.cu -- routing of the fused slice passes by line length and plan
// variant (kernels in ms_slice_impl.cuh, one translation unit per length).
#include "ms_slice_impl.cuh"

namespace ms {

namespace {
template <class F>
cudaError_t by_length(int n, F&& f) {
  switch (n) {
    case 64: return f(std::integral_constant<int, 64>());
    case 128: return f(std::integral_constant<int, 128>());
    case 256: return f(std::integral_constant<int, 256>());
    case 512: return f(std::integral_constant<int, 512>());
    case 1024: return f(std::integral_constant<int, 1024>());
    case 2048: return f(std::integral_constant<int, 2048>());
    case 4096: return f(std::integral_constant<int, 4096>());
    default: return cudaErrorInvalidValue;
  }
}
bool supported_length(int n) { return n >= 64 && n <= 4096 && (n & (n - 1)) == 0; }
}  // namespace

bool fused_supported(int nx, int ny) { return supported_length(nx) && supported_length(ny); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to
// the driver library), looked up once.
bool wave_tensor_map(CUtensorMap* m, const float2* base, int nx, int ny, int cb) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = []() -> Encode {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<Encode>(fn);
  }();
  if (!encode || ((uintptr_t)base & 15) || nx <= 0 || ny <= 0 || ((size_t)nx * sizeof(float2)) % 16 ||
      (2 * cb * (int)sizeof(float)) % 16 || ny % kTmaRows)
    return false;
  // the wave as floats: 2 nx per row, ny rows; boxes of 2 cb floats x 256 rows
  const cuuint64_t dims[2] = {(cuuint64_t)2 * nx, (cuuint64_t)ny};
  const cuuint64_t strides[1] = {(cuuint64_t)nx * sizeof(float2)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * cb), (cuuint32_t)kTmaRows};
  const cuuint32_t elem[2] = {1, 1};
  return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void band_limit_thresholds(float kmax, float* k2_lt, float* k2_le) {
  auto first = [](float m, bool strict) {
    // smallest x >= 0 with sqrtf(x) >= m (strict: > m); sqrtf is monotone
    auto pass = [&](float x) { return strict ? std::sqrt(x) > m : std::sqrt(x) >= m; };
    float x = (float)((double)m * (double)m);
    while (x > 0.0f && pass(std::nextafter(x, 0.0f))) x = std::nextafter(x, 0.0f);
    while (!pass(x)) x = std::nextafter(x, INFINITY);
    return x;
  };
  *k2_lt = first(kmax, false);
  *k2_le = first(kmax, true);
}

float2 unit_fp32(double c, double s) {
  const float c0 = (float)c, s0 = (float)s;
  float bc = c0, bs = s0;
  double bn = INFINITY, ba = INFINITY;
  const double ang = std::atan2(s, c);
  for (int dc = -1; dc <= 1; ++dc)
    for (int ds = -1; ds <= 1; ++ds) {
      const float cc = dc == 0 ? c0 : std::nextafter(c0, dc > 0 ? INFINITY : -INFINITY);
      const float ss = ds == 0 ? s0 : std::nextafter(s0, ds > 0 ? INFINITY : -INFINITY);
      const double n = std::fabs((double)cc * cc + (double)ss * ss - 1.0);
      const double a = std::fabs(std::atan2((double)ss, (double)cc) - ang);
      if (n < bn || (n == bn && a < ba)) {
        bn = n;
        ba = a;
        bc = cc;
        bs = ss;
      }
    }
  return make_float2(bc, bs);
}

int plan_variants() { return kPlanVariants; }

int make_twiddles(int n, int variant, float2* host_out) {
  int size = 0;
  by_length(n, [&](auto c) {
    size = twiddles_n<decltype(c)::value>(variant, host_out);
    return cudaSuccess;
  });
  return size;
}

cudaError_t launch_pass_a(const PassAArgs& a, int variant, int flags, int batch, cudaStream_t s) {
  return by_length(a.nx, [&](auto c) { return dispatch_a_n<decltype(c)::value>(a, variant, flags, batch, s); });
}

cudaError_t launch_pass_b(const PassBArgs& a, int variant, int mode, int batch, cudaStream_t s) {
  return by_length(a.ny, [&](auto c) { return dispatch_b_n<decltype(c)::value>(a, variant, mode, batch, s); });
}

}  // namespace ms
