// Pair filter of DescriptorGenerator.pos_to_pts (DescriptorGenerator.py:168-182):
// minimum-image translation in FP32 and |t| < cutoff (compared in double, the
// reference's cutoff being a Python float), keeping the Verlet order.
// Two passes over a fixed grid of chunks: count per chunk, then every block
// sums the counts of the chunks before it and writes its kept pairs in order.
#include "common.cuh"

namespace amlp {
namespace {

constexpr int kFilterBlocks = 4 * kNumSM;
constexpr int kFilterThreads = 256;

// Box of pair k: L, or with several systems in one launch the box of the
// system of body i.
struct BoxOf {
    float L;
    const int *rep;
    const amlp_replica *rp;
    __device__ __forceinline__ float operator()(int i) const { return rep ? rp[rep[i]].box : L; }
};

__device__ __forceinline__ bool keep_pair(const float *pos, const int *vp, long long k, BoxOf box, double cutoff) {
    float d;
    int i = vp[2 * k];
    min_image(pos, i, vp[2 * k + 1], box(i), &d);
    return (double)d < cutoff;
}

__device__ __forceinline__ void chunk_range(long long nv, long long *s, long long *e) {
    long long chunk = (nv + gridDim.x - 1) / gridDim.x;
    *s = min(nv, (long long)blockIdx.x * chunk);
    *e = min(nv, *s + chunk);
}

__global__ void __launch_bounds__(kFilterThreads) k_filter_count(const float *pos, BoxOf L, double cutoff, const int *vp,
                                                                 const long long *d_nv, long long cap, int *counts) {
    long long nv = min(*d_nv, cap), s, e;
    chunk_range(nv, &s, &e);
    int c = 0;
    for (long long k = s + threadIdx.x; k < e; k += blockDim.x) c += keep_pair(pos, vp, k, L, cutoff);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int ws[kFilterThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kFilterThreads / 32; ++w) t += ws[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kFilterThreads) k_filter_write(const float *pos, BoxOf L, double cutoff, const int *vp,
                                                                 const long long *d_nv, long long cap, const int *counts,
                                                                 int *out, long long *d_np) {
    __shared__ long long base_s;
    __shared__ int wsum[kFilterThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // offset of this chunk = sum of the counts of the chunks before it
    long long b = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) b += counts[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
    if (threadIdx.x == 0) base_s = 0;
    __syncthreads();
    if (lane == 0 && b) atomicAdd((unsigned long long *)&base_s, (unsigned long long)b);
    __syncthreads();
    long long base = base_s;
    long long nv = min(*d_nv, cap), s, e;
    chunk_range(nv, &s, &e);
    for (long long t0 = s; t0 < e; t0 += blockDim.x) {
        long long k = t0 + threadIdx.x;
        bool keep = k < e && keep_pair(pos, vp, k, L, cutoff);
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wsum[w] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int q = 0; q < kFilterThreads / 32; ++q) {
            before += q < w ? wsum[q] : 0;
            total += wsum[q];
        }
        if (keep) {
            long long o = base + before + __popc(m & ((1u << lane) - 1u));
            out[2 * o] = vp[2 * k];
            out[2 * o + 1] = vp[2 * k + 1];
        }
        base += total;
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *d_np = base;
}

}  // namespace
}  // namespace amlp

using namespace amlp;

extern "C" amlp_status amlp_filter_workspace_bytes(long long cap_verlet, size_t *bytes) {
    if (cap_verlet < 0 || !bytes) return AMLP_ERR_INVALID_ARG;
    *bytes = align_up(kFilterBlocks * sizeof(int));
    return AMLP_OK;
}

extern "C" amlp_status amlp_pair_filter(const float *d_pos, float box, double cutoff, const int *d_vpairs,
                                        const long long *d_nverlet, long long cap_verlet, int *d_pairs,
                                        long long *d_npairs, void *d_ws, size_t ws_bytes, void *stream) {
    if (!d_pos || !d_nverlet || !d_npairs || !(box > 0.f) || cap_verlet < 0) return AMLP_ERR_INVALID_ARG;
    if (!d_ws || ws_bytes < kFilterBlocks * sizeof(int)) return AMLP_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    int *counts = static_cast<int *>(d_ws);
    double c = cutoff;
    BoxOf b{box, nullptr, nullptr};
    k_filter_count<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, c, d_vpairs, d_nverlet, cap_verlet, counts);
    k_filter_write<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, c, d_vpairs, d_nverlet, cap_verlet, counts,
                                                            d_pairs, d_npairs);
    return check_launch();
}

extern "C" amlp_status amlp_multi_pair_filter(const float *d_pos, const int *d_rep, const amlp_replica *d_rp,
                                              double cutoff, const int *d_vpairs, const long long *d_nverlet,
                                              long long cap_verlet, int *d_pairs, long long *d_npairs, void *d_ws,
                                              size_t ws_bytes, void *stream) {
    if (!d_pos || !d_rep || !d_rp || !d_nverlet || !d_npairs || cap_verlet < 0) return AMLP_ERR_INVALID_ARG;
    if (!d_ws || ws_bytes < kFilterBlocks * sizeof(int)) return AMLP_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    int *counts = static_cast<int *>(d_ws);
    BoxOf b{0.f, d_rep, d_rp};
    k_filter_count<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, cutoff, d_vpairs, d_nverlet, cap_verlet, counts);
    k_filter_write<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, cutoff, d_vpairs, d_nverlet, cap_verlet, counts,
                                                            d_pairs, d_npairs);
    return check_launch();
}
