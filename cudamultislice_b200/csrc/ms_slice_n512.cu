// ms_slice_n512.cu -- fused slice passes for lines of 512 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(512)
}  // namespace ms
