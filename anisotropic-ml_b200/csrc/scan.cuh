// Device-wide exclusive prefix sums (three passes: tile sums, scan of the tile
// sums in one block, tile scans with their offsets). out[0..n] receives n+1
// values, out[n] being the total; out may alias in (each tile is read before
// it is written). With a non-null gate every kernel returns at once when
// gate[0] == 0 (the scan is part of a pass that only runs when flagged).
#pragma once
#include "common.cuh"

namespace amlp {

constexpr int kScanTile = 1024;  // elements per block (one per thread)

inline size_t scan_tmp_elems(size_t n) { return (n + kScanTile - 1) / kScanTile + 2; }

template <class T>
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long *total) {
    __shared__ long long warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        long long s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    long long excl = x - v + (w > 0 ? warp_sums[w - 1] : 0);
    *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return excl;
}

template <class T>
__global__ void k_tile_sums(const T *in, long long n, long long *tsum, const int *gate) {
    if (gate && !*gate) return;
    long long i = (long long)blockIdx.x * kScanTile + threadIdx.x;
    long long v = i < n ? (long long)in[i] : 0;
    long long tot;
    block_exclusive_scan<T>(v, &tot);
    if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

// Exclusive scan of the tile sums in one block (any number of tiles).
__global__ void k_scan_tiles(long long *tsum, long long ntiles, const int *gate) {
    if (gate && !*gate) return;
    long long carry = 0;
    for (long long base = 0; base < ntiles; base += blockDim.x) {
        long long i = base + threadIdx.x;
        long long v = i < ntiles ? tsum[i] : 0;
        long long tot;
        long long e = block_exclusive_scan<long long>(v, &tot);
        if (i < ntiles) tsum[i] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) tsum[ntiles] = carry;
}

template <class T>
__global__ void k_tile_scan(const T *in, long long *out, long long n, const long long *tsum, long long ntiles,
                            const int *gate) {
    if (gate && !*gate) return;
    long long i = (long long)blockIdx.x * kScanTile + threadIdx.x;
    long long v = i < n ? (long long)in[i] : 0;
    long long tot;
    long long e = block_exclusive_scan<T>(v, &tot);
    if (i < n) out[i] = tsum[blockIdx.x] + e;
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tsum[ntiles];
}

template <class T>
inline amlp_status exclusive_scan(const T *in, long long *out, long long n, long long *tmp, cudaStream_t s,
                                  const int *gate = nullptr) {
    long long ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) ntiles = 1;
    k_tile_sums<T><<<(unsigned)ntiles, kScanTile, 0, s>>>(in, n, tmp, gate);
    k_scan_tiles<<<1, kScanTile, 0, s>>>(tmp, ntiles, gate);
    k_tile_scan<T><<<(unsigned)ntiles, kScanTile, 0, s>>>(in, out, n, tmp, ntiles, gate);
    return AMLP_OK;
}

inline amlp_status exclusive_scan_int(const int *in, long long *out, long long n, long long *tmp, cudaStream_t s,
                                      const int *gate = nullptr) {
    return exclusive_scan<int>(in, out, n, tmp, s, gate);
}
inline amlp_status exclusive_scan_ll(const long long *in, long long *out, long long n, long long *tmp,
                                     cudaStream_t s, const int *gate = nullptr) {
    return exclusive_scan<long long>(in, out, n, tmp, s, gate);
}

}  // namespace amlp
