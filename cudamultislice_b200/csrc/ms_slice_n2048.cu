// ms_slice_n2048.cu -- fused slice passes for lines of 2048 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(2048)
}  // namespace ms
