// ms_slice_n64.cu -- fused slice passes for lines of 64 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(64)
}  // namespace ms
