// ms_slice_n1024.cu -- fused slice passes for lines of 1024 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(1024)
}  // namespace ms
