// Error reporting, version and device queries of the adock_b200 C-ABI.
#include "common.cuh"
#include <stdarg.h>
#include <stdio.h>

namespace adock {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
    set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), where);
    return ADOCK_E_CUDA;
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
    return n;
}

}  // namespace adock

extern "C" int adock_version(void) { return ADOCK_ABI_VERSION; }
extern "C" const char* adock_last_error(void) { return adock::g_err; }
