// Pair filter of DescriptorGenerator.pos_to_pts (DescriptorGenerator.py:168-182):
// minimum-image translation in FP32 and |t| < cutoff (compared in double, the
// reference's cutoff being a Python float), keeping the Verlet order.
// Two passes over a fixed grid of chunks: the first tests every pair, stores
// one keep bit per pair and counts per chunk; the second sums the counts of
// the chunks before its own and writes the kept pairs in order, reading the
// bits instead of testing the pairs again.
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
    int vec;  // the pair list is 16-byte aligned: vector loads allowed
    __device__ __forceinline__ float operator()(int i) const { return rep ? rp[rep[i]].box : L; }
};

__device__ __forceinline__ bool keep_ij(const float *pos, int i, int j, BoxOf box, double cutoff) {
    float d;
    min_image(pos, i, j, box(i), &d);
    return (double)d < cutoff;
}

// Each thread takes kFilterItems consecutive pairs per round (two 16-byte loads
// when the four lie inside the chunk), so a block covers 1024 pairs per round
// and every thread has four independent position gathers in flight.
constexpr int kFilterItems = 4;
constexpr int kFilterRound = kFilterThreads * kFilterItems;

// Bit u set when pair k0 + u (< e) is kept.
__device__ __forceinline__ unsigned keep_mask(const float *pos, const int *vp, long long k0, long long e, BoxOf box,
                                              double cutoff, int (&ij)[2 * kFilterItems]) {
    if (box.vec && k0 + kFilterItems <= e) {
        const int4 a = *reinterpret_cast<const int4 *>(vp + 2 * k0);
        const int4 b = *reinterpret_cast<const int4 *>(vp + 2 * k0 + 4);
        ij[0] = a.x; ij[1] = a.y; ij[2] = a.z; ij[3] = a.w;
        ij[4] = b.x; ij[5] = b.y; ij[6] = b.z; ij[7] = b.w;
    } else {
#pragma unroll
        for (int u = 0; u < kFilterItems; ++u) {
            const bool in = k0 + u < e;
            ij[2 * u] = in ? vp[2 * (k0 + u)] : 0;
            ij[2 * u + 1] = in ? vp[2 * (k0 + u) + 1] : 0;
        }
    }
    unsigned m = 0;
#pragma unroll
    for (int u = 0; u < kFilterItems; ++u)
        if (k0 + u < e && keep_ij(pos, ij[2 * u], ij[2 * u + 1], box, cutoff)) m |= 1u << u;
    return m;
}

// Chunks of whole 32-pair words of the keep bits (and so multiples of
// kFilterItems pairs: the 16-byte loads are aligned).
__device__ __forceinline__ void chunk_range(long long nv, long long *s, long long *e) {
    long long chunk = (nv + gridDim.x - 1) / gridDim.x;
    chunk = (chunk + 31) / 32 * 32;
    *s = min(nv, (long long)blockIdx.x * chunk);
    *e = min(nv, *s + chunk);
}

__global__ void __launch_bounds__(kFilterThreads) k_filter_count(const float *pos, BoxOf L, double cutoff,
                                                                 const int *vp, const long long *d_nv, long long cap,
                                                                 int *counts, unsigned *bits) {
    long long nv = min(*d_nv, cap), s, e;
    chunk_range(nv, &s, &e);
    const int lane = threadIdx.x & 31;
    int c = 0;
    int ij[2 * kFilterItems];
    // every thread of a warp runs the same rounds (a round starts at s + multiple of 1024)
    for (long long r0 = s; r0 < e; r0 += kFilterRound) {
        const long long k0 = r0 + (long long)threadIdx.x * kFilterItems;
        const unsigned m = k0 < e ? keep_mask(pos, vp, k0, e, L, cutoff, ij) : 0u;
        c += __popc(m);
        // eight lanes' four bits make the 32-bit word of pairs k0 - 4 (lane % 8) ...
        unsigned w = m << (4 * (lane & 7));
        w |= __shfl_xor_sync(0xffffffffu, w, 1);
        w |= __shfl_xor_sync(0xffffffffu, w, 2);
        w |= __shfl_xor_sync(0xffffffffu, w, 4);
        if ((lane & 7) == 0 && k0 < e) bits[k0 >> 5] = w;
    }
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

__global__ void __launch_bounds__(kFilterThreads) k_filter_write(const int *vp, const long long *d_nv, long long cap,
                                                                 const int *counts, const unsigned *bits, int vec,
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
    int ij[2 * kFilterItems];
    for (long long r0 = s; r0 < e; r0 += kFilterRound) {
        const long long k0 = r0 + (long long)threadIdx.x * kFilterItems;
        const unsigned m = k0 < e ? (bits[k0 >> 5] >> (k0 & 31)) & ((1u << kFilterItems) - 1u) : 0u;
        if (m) {  // the pair rows of this thread's group, only when one of them is kept
            if (vec && k0 + kFilterItems <= e) {
                const int4 a = *reinterpret_cast<const int4 *>(vp + 2 * k0);
                const int4 b = *reinterpret_cast<const int4 *>(vp + 2 * k0 + 4);
                ij[0] = a.x; ij[1] = a.y; ij[2] = a.z; ij[3] = a.w;
                ij[4] = b.x; ij[5] = b.y; ij[6] = b.z; ij[7] = b.w;
            } else {
#pragma unroll
                for (int u = 0; u < kFilterItems; ++u) {
                    const bool in = k0 + u < e;
                    ij[2 * u] = in ? vp[2 * (k0 + u)] : 0;
                    ij[2 * u + 1] = in ? vp[2 * (k0 + u) + 1] : 0;
                }
            }
        }
        // block-wide exclusive scan of the kept counts (thread order = pair order)
        const int cnt = __popc(m);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        int before = incl - cnt, total = 0;
#pragma unroll
        for (int q = 0; q < kFilterThreads / 32; ++q) {
            before += q < w ? wsum[q] : 0;
            total += wsum[q];
        }
        long long o = base + before;
#pragma unroll
        for (int u = 0; u < kFilterItems; ++u) {
            if (m & (1u << u)) {
                out[2 * o] = ij[2 * u];
                out[2 * o + 1] = ij[2 * u + 1];
                ++o;
            }
        }
        base += total;
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *d_np = base;
}

}  // namespace
}  // namespace amlp

using namespace amlp;

// Workspace: the per-chunk counts, then one keep bit per Verlet pair.
static size_t filter_ws_bytes(long long cap_verlet) {
    return align_up(kFilterBlocks * sizeof(int)) + align_up((size_t)((cap_verlet + 31) / 32 + 1) * sizeof(unsigned));
}

extern "C" amlp_status amlp_filter_workspace_bytes(long long cap_verlet, size_t *bytes) {
    if (cap_verlet < 0 || !bytes) return AMLP_ERR_INVALID_ARG;
    *bytes = filter_ws_bytes(cap_verlet);
    return AMLP_OK;
}

extern "C" amlp_status amlp_pair_filter(const float *d_pos, float box, double cutoff, const int *d_vpairs,
                                        const long long *d_nverlet, long long cap_verlet, int *d_pairs,
                                        long long *d_npairs, void *d_ws, size_t ws_bytes, void *stream) {
    if (!d_pos || !d_nverlet || !d_npairs || !(box > 0.f) || cap_verlet < 0) return AMLP_ERR_INVALID_ARG;
    if (!d_ws || ws_bytes < filter_ws_bytes(cap_verlet)) return AMLP_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    int *counts = static_cast<int *>(d_ws);
    unsigned *bits = reinterpret_cast<unsigned *>(static_cast<char *>(d_ws) + align_up(kFilterBlocks * sizeof(int)));
    double c = cutoff;
    BoxOf b{box, nullptr, nullptr, ((uintptr_t)d_vpairs & 15) == 0};
    k_filter_count<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, c, d_vpairs, d_nverlet, cap_verlet, counts, bits);
    k_filter_write<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_vpairs, d_nverlet, cap_verlet, counts, bits, b.vec,
                                                            d_pairs, d_npairs);
    return check_launch();
}

extern "C" amlp_status amlp_multi_pair_filter(const float *d_pos, const int *d_rep, const amlp_replica *d_rp,
                                              double cutoff, const int *d_vpairs, const long long *d_nverlet,
                                              long long cap_verlet, int *d_pairs, long long *d_npairs, void *d_ws,
                                              size_t ws_bytes, void *stream) {
    if (!d_pos || !d_rep || !d_rp || !d_nverlet || !d_npairs || cap_verlet < 0) return AMLP_ERR_INVALID_ARG;
    if (!d_ws || ws_bytes < filter_ws_bytes(cap_verlet)) return AMLP_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    int *counts = static_cast<int *>(d_ws);
    unsigned *bits = reinterpret_cast<unsigned *>(static_cast<char *>(d_ws) + align_up(kFilterBlocks * sizeof(int)));
    BoxOf b{0.f, d_rep, d_rp, ((uintptr_t)d_vpairs & 15) == 0};
    k_filter_count<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_pos, b, cutoff, d_vpairs, d_nverlet, cap_verlet, counts,
                                                            bits);
    k_filter_write<<<kFilterBlocks, kFilterThreads, 0, s>>>(d_vpairs, d_nverlet, cap_verlet, counts, bits, b.vec,
                                                            d_pairs, d_npairs);
    return check_launch();
}
