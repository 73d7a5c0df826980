// ms_slice_n256.cu -- fused slice passes for lines of 256 points (all plan variants).
#include "ms_slice_impl.cuh"

namespace ms {
MS_SLICE_INSTANTIATE(256)
}  // namespace ms
