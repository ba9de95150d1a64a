// Library-level entry points: version, status strings, CUDA error capture.
#include <cstdio>
#include "common.cuh"

namespace amlp {

static thread_local char g_cuda_err[256] = "";

void set_cuda_error(cudaError_t e) {
    std::snprintf(g_cuda_err, sizeof(g_cuda_err), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
}

amlp_status check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return AMLP_ERR_CUDA;
    }
    return AMLP_OK;
}

}  // namespace amlp

extern "C" int amlp_version(void) { return 1; }

extern "C" const char *amlp_status_string(amlp_status s) {
    switch (s) {
        case AMLP_OK: return "ok";
        case AMLP_ERR_INVALID_ARG: return "invalid argument";
        case AMLP_ERR_UNSUPPORTED: return "unsupported parameters (no compiled kernel for them)";
        case AMLP_ERR_WORKSPACE: return "workspace missing or too small";
        case AMLP_ERR_CUDA: return "CUDA error";
        case AMLP_ERR_CAPACITY: return "output capacity too small";
        case AMLP_ERR_TOO_LARGE: return "size beyond the fixed scratch of the allocation-free entry point";
        default: return "unknown status";
    }
}

extern "C" const char *amlp_last_cuda_error(void) { return amlp::g_cuda_err; }
