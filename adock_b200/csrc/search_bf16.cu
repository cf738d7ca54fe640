// Search kernels instantiated for __nv_bfloat16 grid storage (FP32 interpolation and accumulation).
#include "search_impl.cuh"

namespace adock {
ADOCK_SEARCH_INSTANTIATE(__nv_bfloat16)
}  // namespace adock
