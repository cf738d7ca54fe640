// Search kernels instantiated for __half grid storage (FP32 interpolation and accumulation).
#include "search_impl.cuh"

namespace adock {
ADOCK_SEARCH_INSTANTIATE(__half)
}  // namespace adock
