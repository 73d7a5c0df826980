// ms_slice_n128.cu -- fused slice passes for lines of 128 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(128)
}  // namespace ms
