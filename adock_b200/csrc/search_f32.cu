// Search kernels instantiated for float grid storage (FP32 interpolation and accumulation).
#include "search_impl.cuh"

namespace adock {
ADOCK_SEARCH_INSTANTIATE(float)
}  // namespace adock
