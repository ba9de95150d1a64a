// Shared helpers of libamlp: status handling, launch geometry, exact-rounding
// float helpers and the quaternion rotation of the reference kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/amlp.h"

namespace amlp {

constexpr int kNumSM = 148;  // B200; grids are sized in multiples of it

void set_cuda_error(cudaError_t e);
amlp_status check_launch();
amlp_status device_wait_status();  // AMLP_ERR_DEVICE_WAIT if a bounded device wait gave up

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

__host__ __device__ inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Carves a caller workspace into aligned slices.
struct Carver {
    char *base;
    size_t used = 0, cap;
    Carver(void *p, size_t c) : base(static_cast<char *>(p)), cap(c) {}
    template <class T> T *take(size_t count) {
        size_t off = align_up(used);
        used = off + count * sizeof(T);
        return reinterpret_cast<T *>(base + off);
    }
    bool ok() const { return used <= cap; }
};

// Quaternion rotation of a body point written with the operation order of the
// reference kernels (PosToPtsKernels.py:54-71) and no FMA contraction, so that
// the rotated points round exactly as the FP32 oracle's do.
__device__ __forceinline__ float3 rotate_ref(float4 q, float3 p) {
    float qw = q.x, qx = q.y, qy = q.z, qz = q.w;
    float a = __fsub_rn(__fmul_rn(qw, qw), __fadd_rn(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qy, qy)), __fmul_rn(qz, qz)));
    float dot = __fadd_rn(__fadd_rn(__fmul_rn(qx, p.x), __fmul_rn(qy, p.y)), __fmul_rn(qz, p.z));
    float cx = __fsub_rn(__fmul_rn(qy, p.z), __fmul_rn(qz, p.y));
    float cy = __fsub_rn(__fmul_rn(qz, p.x), __fmul_rn(qx, p.z));
    float cz = __fsub_rn(__fmul_rn(qx, p.y), __fmul_rn(qy, p.x));
    float3 o;
    o.x = __fadd_rn(__fmul_rn(a, p.x), __fmul_rn(2.0f, __fadd_rn(__fmul_rn(qw, cx), __fmul_rn(dot, qx))));
    o.y = __fadd_rn(__fmul_rn(a, p.y), __fmul_rn(2.0f, __fadd_rn(__fmul_rn(qw, cy), __fmul_rn(dot, qy))));
    o.z = __fadd_rn(__fmul_rn(a, p.z), __fmul_rn(2.0f, __fadd_rn(__fmul_rn(qw, cz), __fmul_rn(dot, qz))));
    return o;
}

// Minimum-image translation pos[j] - pos[i] and its length, in the reference's
// FP32 operation order (DescriptorGenerator.py:168-171).
__device__ __forceinline__ float3 min_image(const float *pos, int i, int j, float L, float *dist) {
    float half = __fmul_rn(0.5f, L);
    float t[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float d = __fsub_rn(pos[3 * j + k], pos[3 * i + k]);
        d = d > half ? __fsub_rn(d, L) : d;
        d = d < -half ? __fadd_rn(L, d) : d;
        t[k] = d;
    }
    *dist = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(t[0], t[0]), __fmul_rn(t[1], t[1])), __fmul_rn(t[2], t[2])));
    return make_float3(t[0], t[1], t[2]);
}

__device__ __forceinline__ float4 load_quat(const float *q, int i) {
    return reinterpret_cast<const float4 *>(q)[i];
}

__device__ __forceinline__ float act_f(int act, float z) {
    if (act == AMLP_ACT_RELU) return fmaxf(z, 0.0f);
    if (act == AMLP_ACT_TANH) return tanhf(z);
    return z / (1.0f + __expf(-z));
}

// Derivative of the activation as a function of the pre-activation z.
__device__ __forceinline__ float act_df(int act, float z) {
    if (act == AMLP_ACT_RELU) return z > 0.0f ? 1.0f : 0.0f;
    if (act == AMLP_ACT_TANH) { float t = tanhf(z); return 1.0f - t * t; }
    float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// True when the keys of the valid lanes never decrease from one lane to the
// next, so that equal keys form contiguous runs and a segmented warp sum over
// runs is exact. `ok` marks the valid lanes, a prefix of the warp. Pair lists
// from amlp_pair_filter are sorted by (i, j); other callers may pass any order,
// and the scatters then fall back to one atomic per lane.
__device__ __forceinline__ bool warp_keys_sorted(int key, bool ok) {
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    return __all_sync(0xffffffffu, !ok || lane == 0 || prev <= key) != 0;
}

__device__ __forceinline__ float clip100(float v) { return v > 100.0f ? 100.0f : (v < -100.0f ? -100.0f : v); }

}  // namespace amlp

#define AMLP_CHECK_CUDA(call)                       \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) {                    \
            amlp::set_cuda_error(e_);               \
            return AMLP_ERR_CUDA;                   \
        }                                           \
    } while (0)
