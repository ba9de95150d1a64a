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

// FP32 FMA throughput probe: 8 independent multiply-add chains per thread.
constexpr int kProbeChains = 8;
__global__ void __launch_bounds__(512) k_fma_probe(float *out, int iters, float mul, float add) {
    float v[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) v[c] = (float)(threadIdx.x + c) * 1e-3f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) v[c] = fmaf(v[c], mul, add);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) s += v[c];
    if (s == 12345.678f) out[0] = s;  // never true for these inputs; keeps the chains alive
}

}  // namespace amlp

extern "C" amlp_status amlp_fp32_fma_probe(float *d_out, int iters, double *flops, void *stream) {
    if (!d_out || iters <= 0 || !flops) return AMLP_ERR_INVALID_ARG;
    const int blocks = 4 * amlp::kNumSM, threads = 512;
    amlp::k_fma_probe<<<blocks, threads, 0, amlp::as_stream(stream)>>>(d_out, iters, 0.9999999f, 1e-7f);
    *flops = 2.0 * amlp::kProbeChains * (double)iters * blocks * threads;
    return amlp::check_launch();
}

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
        case AMLP_ERR_DEVICE_WAIT: return "a bounded device-side wait gave up (see amlp_device_error)";
        default: return "unknown status";
    }
}

extern "C" const char *amlp_last_cuda_error(void) { return amlp::g_cuda_err; }
