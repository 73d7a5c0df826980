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
