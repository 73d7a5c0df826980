// ms_slice_n4096.cu -- fused slice passes for lines of 4096 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(4096)
}  // namespace ms
