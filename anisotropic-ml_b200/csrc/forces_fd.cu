// Finite-difference force path (the reference's method):
//   DescriptorGenerator.generate_nep_descriptors (DescriptorGenerator.py:136-161)
//   ForceEvaluator.evaluate_interactions        (ForceEvaluator.py:71-146)
// as three kernels that keep the reference's intermediate g_all in HBM
// (amlp_descriptors, amlp_mlp_energy, amlp_fd_scatter) and as one fused kernel
// (amlp_forces_fd) that keeps every intermediate on chip.
//
// Tile of the descriptor stage: 32 pairs x 10 variants = 320 rows, one thread
// per row; warp v evaluates variant v of the 32 pairs (lane = pair), so every
// branch on the variant is warp-uniform. The rotated body points of the tile
// are staged in shared memory once and each variant's points are derived from
// them on the fly. The fused kernel runs 12 warps: warps 8 and 9 take the first
// harmonic pass of variants 8 and 9 and warps 10 and 11 the second, so that each
// of the SM's four schedulers (warp % 4) holds five passes of the tile instead
// of six, six, four and four.
#include "descriptor.cuh"
#include "descriptor_direct.cuh"

namespace amlp {

constexpr int kPT = 32;             // pairs per tile
constexpr int kRows = 10 * kPT;     // rows (pair-variants) per tile
constexpr int kTileThreads = kRows;  // one thread per row
constexpr int kFusedThreads = kRows + 2 * kPT;  // the fused kernel: two more warps for the split variants
static_assert(kTileThreads % (2 * kPT) == 0 && kFusedThreads % (2 * kPT) == 0,
              "whole (pair, body) groups per thread stride");

struct TileGeom {
    int npts, nd, rs;  // points per body, points per cloud, floats per pair in R (odd)
};

__host__ __device__ inline TileGeom tile_geom(int npts) {
    TileGeom g;
    g.npts = npts;
    g.nd = 2 * npts;
    g.rs = 6 * npts + ((6 * npts) % 2 == 0 ? 1 : 0);
    return g;
}

// Rotated body points of the pairs [p0, p0 + kPT) (clamped to the last pair),
// the minimum-image translations and the pair indices. The pairs'
// orientations are read once into shared memory first. The caller's barrier
// must separate this from the previous use of R, t and ij.
__device__ void load_tile(const float *pos, const float *quat, float L, const int *pairs, long long P, long long p0,
                          const float *pts_s, const TileGeom &g, float *R, float *t, int *ij) {
    __shared__ float4 qs[2 * kPT];
    const int nthr = blockDim.x;
    for (int p = threadIdx.x; p < kPT; p += nthr) {
        long long pr = min(p0 + p, P - 1);
        int i = pairs[2 * pr], j = pairs[2 * pr + 1];
        qs[2 * p] = load_quat(quat, i);
        qs[2 * p + 1] = load_quat(quat, j);
        float d;
        float3 tt = min_image(pos, i, j, L, &d);
        t[3 * p] = tt.x;
        t[3 * p + 1] = tt.y;
        t[3 * p + 2] = tt.z;
        ij[2 * p] = i;
        ij[2 * p + 1] = j;
    }
    __syncthreads();
    // thread -> (pair, body) = tid % 64 and a stride of points tid / 64 (no index divisions)
    const int pb = threadIdx.x & (2 * kPT - 1), p = pb >> 1, body = pb & 1;
    const float4 qq = qs[2 * p + body];
    float *dst = R + p * g.rs + body * 3 * g.npts;
    for (int a = threadIdx.x / (2 * kPT); a < g.npts; a += nthr / (2 * kPT)) {
        float3 r = rotate_ref(qq, make_float3(pts_s[3 * a], pts_s[3 * a + 1], pts_s[3 * a + 2]));
        dst[3 * a] = r.x;
        dst[3 * a + 1] = r.y;
        dst[3 * a + 2] = r.z;
    }
}

// Descriptor of row (variant v, pair p = lane) of the staged tile into
// gT[d*ld + col], the harmonic passes in pass_mask.
template <class Cfg>
__device__ __forceinline__ void tile_descriptor_row(const float *R, const float *t, const TileGeom &g, float dx,
                                                    float dteta, float inv_rc, float *gT, int ld, int col, int v,
                                                    unsigned pass_mask = (1u << Cfg::NPASS) - 1u) {
    const int p = threadIdx.x & 31;
    VariantPoints vp;
    vp.Ri = R + p * g.rs;
    vp.Rj = vp.Ri + 3 * g.npts;
    vp.tx = t[3 * p];
    vp.ty = t[3 * p + 1];
    vp.tz = t[3 * p + 2];
    vp.h = g.npts;
    vp.v = v;
    vp.dx = dx;
    vp.q = variant_quat(v, dteta);
    nep_descriptor<Cfg>(vp, g.nd, inv_rc, gT + col, ld, pass_mask);
}

// The tile's 10 x kPT descriptor rows from gT (column v kPT + p, row stride ld,
// odd) to g_all, where rows v*P + p0 .. p0+valid-1 of variant v are
// contiguous: a warp per row, lanes over the D columns (coalesced stores,
// column reads on 32 banks), no index divisions.
template <int D>
__device__ __forceinline__ void store_tile_rows(const float *gT, int ld, float *g_out, long long P, long long p0,
                                                int valid) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < 10 * kPT; r += nw) {
        const int v = r / kPT, p = r - v * kPT;
        if (p >= valid) continue;
        float *dst = g_out + ((long long)v * P + p0 + p) * D;
        const float *src = gT + r;
        for (int d = lane; d < D; d += 32) dst[d] = src[d * ld];
    }
}

// ---------------------------------------------------------------- g_all to HBM
template <class Cfg>
__global__ void __launch_bounds__(kTileThreads) k_descriptors(const float *pos, const float *quat, float L,
                                                              const int *pairs, long long P, const float *pts,
                                                              int npts, float dx, float dteta, float inv_rc, float *g_out) {
    extern __shared__ float smem[];
    const TileGeom g = tile_geom(npts);
    constexpr int ld = kRows + 1;  // odd stride: conflict-free column reads below
    float *pts_s = smem;
    float *R = pts_s + 3 * npts;
    float *t = R + kPT * g.rs;
    int *ij = reinterpret_cast<int *>(t + 3 * kPT);
    float *gT = reinterpret_cast<float *>(ij + 2 * kPT);
    for (int k = threadIdx.x; k < 3 * npts; k += blockDim.x) pts_s[k] = pts[k];
    __syncthreads();
    long long ntiles = (P + kPT - 1) / kPT;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        long long p0 = tile * kPT;
        load_tile(pos, quat, L, pairs, P, p0, pts_s, g, R, t, ij);
        __syncthreads();
        tile_descriptor_row<Cfg>(R, t, g, dx, dteta, inv_rc, gT, ld, threadIdx.x, threadIdx.x >> 5);
        __syncthreads();
        int valid = (int)min((long long)kPT, P - p0);
        store_tile_rows<Cfg::D>(gT, ld, g_out, P, p0, valid);
        __syncthreads();
    }
}

// The same rows in the reference's direct form, g_ang[n,l] = sum_{a,b} f_n(a)
// f_n(b) P_l(rhat_a . rhat_b) (NepDescriptorKernels.py:3-144): cheaper than the
// harmonic passes for the clouds of the reference's th_v1 and cube_v2 shapes
// (8 and 12 points) and for the hypers (10, 10, 10), whose 120 harmonics take
// twelve passes. Each row thread centres its variant's cloud into its own
// float4 (rhat_a, d_a) slots of shared memory (point-major, threads innermost),
// then sums the unordered point pairs, doubled, plus the diagonal (c = 1,
// P_l(1) = 1), like the adjoint's direct forward pass.
template <int NR, int NA, int LM>
__device__ __forceinline__ void direct_row_descriptor(const VariantPoints &vp, int nd, float inv_rc, float4 *S,
                                                      int sstride, float *g, int gstride) {
    const float3 ps = vp.point_sum();
    const float inv_nd = 1.0f / (float)nd;
    const float cx = ps.x * inv_nd, cy = ps.y * inv_nd, cz = ps.z * inv_nd;
    for (int a = 0; a < nd; ++a) {
        const float3 p = vp(a);
        const float rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
        const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
        const float inv_d = rsqrtf(d2);
        S[a * sstride] = make_float4(rx * inv_d, ry * inv_d, rz * inv_d, d2 * inv_d);
    }
    float acc[NA][LM], rad[NR], dia[NA];
#pragma unroll
    for (int n = 0; n < NA; ++n) {
        dia[n] = 0.f;
#pragma unroll
        for (int l = 0; l < LM; ++l) acc[n][l] = 0.f;
    }
#pragma unroll
    for (int n = 0; n < NR; ++n) rad[n] = 0.f;
    for (int a = 0; a < nd; ++a) {
        const float4 A = S[a * sstride];
        float fa[NR];
        radial_basis<NR>(A.w, inv_rc, fa);
#pragma unroll
        for (int n = 0; n < NR; ++n) rad[n] += fa[n];
#pragma unroll
        for (int n = 0; n < NA; ++n) dia[n] = fmaf(fa[n], fa[n], dia[n]);
        for (int b = a + 1; b < nd; ++b) {
            const float4 B = S[b * sstride];
            const float c = fmaf(A.x, B.x, fmaf(A.y, B.y, A.z * B.z));
            float Pl[LM];
            Pl[0] = c;
            Pl[1] = direct::legendre_next(1, c, c, 1.0f);
#pragma unroll
            for (int l = 2; l < LM; ++l) Pl[l] = direct::legendre_next(l, c, Pl[l - 1], Pl[l - 2]);
            float fb[NR];
            radial_basis<NR>(B.w, inv_rc, fb);
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                const float ff = fa[n] * fb[n];
#pragma unroll
                for (int l = 0; l < LM; ++l) acc[n][l] = fmaf(ff, Pl[l], acc[n][l]);
            }
        }
    }
#pragma unroll
    for (int n = 0; n < NR; ++n) g[n * gstride] = rad[n];
#pragma unroll
    for (int n = 0; n < NA; ++n)
#pragma unroll
        for (int l = 0; l < LM; ++l) g[(NR + n * LM + l) * gstride] = fmaf(2.0f, acc[n][l], dia[n]);
}

template <int NR, int NA, int LM>
__global__ void __launch_bounds__(kTileThreads) k_descriptors_direct(const float *pos, const float *quat, float L,
                                                                     const int *pairs, long long P, const float *pts,
                                                                     int npts, float dx, float dteta, float inv_rc,
                                                                     float *g_out) {
    constexpr int D = NR + NA * LM;
    extern __shared__ __align__(16) float smem[];
    const TileGeom g = tile_geom(npts);
    constexpr int ld = kRows + 1;  // odd stride: conflict-free column reads below
    float4 *cloud = reinterpret_cast<float4 *>(smem);  // g.nd x kTileThreads
    float *pts_s = reinterpret_cast<float *>(cloud + (size_t)g.nd * kTileThreads);
    float *R = pts_s + 3 * npts;
    float *t = R + kPT * g.rs;
    int *ij = reinterpret_cast<int *>(t + 3 * kPT);
    float *gT = reinterpret_cast<float *>(ij + 2 * kPT);
    for (int k = threadIdx.x; k < 3 * npts; k += blockDim.x) pts_s[k] = pts[k];
    __syncthreads();
    const int v = threadIdx.x >> 5, p = threadIdx.x & 31;
    long long ntiles = (P + kPT - 1) / kPT;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        long long p0 = tile * kPT;
        load_tile(pos, quat, L, pairs, P, p0, pts_s, g, R, t, ij);
        __syncthreads();
        VariantPoints vp;
        vp.Ri = R + p * g.rs;
        vp.Rj = vp.Ri + 3 * g.npts;
        vp.tx = t[3 * p];
        vp.ty = t[3 * p + 1];
        vp.tz = t[3 * p + 2];
        vp.h = g.npts;
        vp.v = v;
        vp.dx = dx;
        vp.q = variant_quat(v, dteta);
        direct_row_descriptor<NR, NA, LM>(vp, g.nd, inv_rc, cloud + threadIdx.x, kTileThreads, gT + threadIdx.x, ld);
        __syncthreads();
        int valid = (int)min((long long)kPT, P - p0);
        store_tile_rows<D>(gT, ld, g_out, P, p0, valid);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- generic FP32 net
struct MlpDesc {
    int n_layers, act;
    int dims[AMLP_MAX_LAYERS + 1];
    long long woff[AMLP_MAX_LAYERS];  // offset of W_k in the packed weights; b_k follows
};

constexpr int kMlpRows = 128;

// One thread per row; activations of the 128-row tile in shared memory,
// transposed (feature-major); four outputs per pass share each input load.
__global__ void __launch_bounds__(kMlpRows) k_mlp(const float *g, long long rows, MlpDesc m, const float *w,
                                                  int amax, float *e_out) {
    extern __shared__ float smem[];
    float *A = smem, *B = smem + (size_t)amax * kMlpRows;
    const int r = threadIdx.x;
    for (long long r0 = (long long)blockIdx.x * kMlpRows; r0 < rows; r0 += (long long)gridDim.x * kMlpRows) {
        const int D = m.dims[0];
        for (int idx = threadIdx.x; idx < kMlpRows * D; idx += blockDim.x) {
            int rr = idx / D, d = idx - rr * D;
            A[d * kMlpRows + rr] = r0 + rr < rows ? g[(r0 + rr) * D + d] : 0.f;
        }
        __syncthreads();
        float *X = A, *Y = B;
        for (int L = 0; L < m.n_layers; ++L) {
            const int K = m.dims[L], N = m.dims[L + 1];
            const float *W = w + m.woff[L], *b = W + (size_t)N * K;
            const bool last = L == m.n_layers - 1;
            for (int n = 0; n < N; n += 4) {
                float acc[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = n + q < N ? __ldg(b + n + q) : 0.f;
                for (int k = 0; k < K; ++k) {
                    float x = X[k * kMlpRows + r];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (n + q < N) acc[q] = fmaf(__ldg(W + (size_t)(n + q) * K + k), x, acc[q]);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (n + q < N) Y[(n + q) * kMlpRows + r] = last ? acc[q] : act_f(m.act, acc[q]);
            }
            __syncthreads();
            float *tmp = X;
            X = Y;
            Y = tmp;
        }
        if (r0 + r < rows) e_out[r0 + r] = X[r];
        __syncthreads();
    }
}

// Register-tiled FP32 net for widths up to 160 (the reference's 150-wide models
// on its own finite-difference data flow): tiles of 128 rows, 512 threads (four
// warps per scheduler, which the shared memory of one tile allows). The
// activations are feature-major in one shared-memory buffer, XT[k][col] (row
// stride kTLd), with the tile's rows permuted so that thread rg's eight rows
// sit at columns 4 rg .. 4 rg + 3 and 64 + 4 rg .. + 3: a quarter warp's
// 16-byte loads cover 128 contiguous bytes. Each layer's weights are staged
// k-major, WT[k][n] (row stride kTWs), by cp.async in blocks of 8 k x 4 n per
// warp instruction (four 32-byte global segments, 32 different banks), so that
// every copy of a thread is in flight at once; the next layer's copies run
// while a layer's outputs are written. Thread t owns rows rg = t % 16 and, for
// a 160-wide layer, columns 4 cg .. 4 cg + 3 and 128 + cg (cg = t / 16): per k
// two 16-byte activation loads and two weight loads (16 and 4 bytes) feed 40
// multiply-adds, the next k's operands loading while this k's multiply-adds
// issue. Narrower layers take columns cg, cg + 32, ... below npad. The outputs
// stay in registers until every thread has read the layer's inputs, then
// overwrite them. Each hidden output is bias + sum_k x_k w_k in ascending k, one
// rounding per multiply-add; the energy (the one-column output layer) is the
// bias plus the 32 column groups' partial sums over k = cg, cg + 32, ...
constexpr int kTRows = 128, kTThreads = 512, kTMaxW = 160, kTGroups = kTThreads / 16;
constexpr int kTMaxCw = kTMaxW / kTGroups;  // outputs per row and thread: 5
constexpr int kTLd = kTRows + 4;  // activation row stride (16-byte aligned rows)
constexpr int kTWs = kTMaxW + 4;  // weight row stride: 16-byte aligned rows, 4 (mod 32) for the staging banks
constexpr int kTRowsK = kTMaxW + 2;  // rows of XT and WT: K <= 160 plus the two that a prefetch may read past K
__host__ __device__ constexpr int tiled_col(int r) { return ((r >> 2) & 1) * (kTRows / 2) + (r >> 3) * 4 + (r & 3); }

// Asynchronous 4-byte global -> shared copy (cp.async, no register staging).
__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Layer L's weights, k-major with zero columns up to npad, and its bias into
// WT and Bs, in blocks of 8 k x 4 n per warp instruction. Copies in flight
// until cp_async_wait_all.
__device__ __forceinline__ void stage_layer(const MlpDesc &m, const float *w, int L, float *WT, float *Bs) {
    const int K = m.dims[L], N = m.dims[L + 1], npad = (N + 15) / 16 * 16;
    const float *W = w + m.woff[L], *b = W + (size_t)N * K;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // warp w takes the column blocks w, w + 16, ... and walks each down k with
    // two pointer increments per copy (no index division)
    for (int nbi = warp; 4 * nbi < npad; nbi += kTThreads / 32) {
        const int n = 4 * nbi + (lane & 3);
        int k = lane >> 2;
        float *dst = WT + k * kTWs + n;
        if (n < N) {
            const float *src = W + (size_t)n * K + k;
            for (; k < K; k += 8, src += 8, dst += 8 * kTWs) cp_async4(dst, src);
        } else {
            for (; k < K; k += 8, dst += 8 * kTWs) *dst = 0.f;
        }
    }
    for (int n = t; n < npad; n += kTThreads) {
        if (n < N) cp_async4(Bs + n, b + n);
        else Bs[n] = 0.f;
    }
}

// Column of output c of thread group cg: a 160-wide layer (4 contiguous, then
// one of the last 32), or a narrower one (cg + 32 c; beyond npad unused).
__device__ __forceinline__ int wide_col(int cg, int c) { return c < 4 ? 4 * cg + c : 128 + cg; }
__device__ __forceinline__ int narrow_col(int cg, int c) { return cg + kTGroups * c; }

__global__ void __launch_bounds__(kTThreads) k_mlp_tiled(const float *g, long long rows, MlpDesc m, const float *w,
                                                         float *e_out) {
    extern __shared__ __align__(16) float smem[];
    float *XT = smem;                  // kTRowsK x kTLd
    float *WT = XT + kTRowsK * kTLd;   // kTRowsK x kTWs
    float *Bs = WT + kTRowsK * kTWs;   // kTMaxW
    const int t = threadIdx.x, rg = t & 15, cg = t >> 4;
    for (long long r0 = (long long)blockIdx.x * kTRows; r0 < rows; r0 += (long long)gridDim.x * kTRows) {
        const int D = m.dims[0];
        const int nr = (int)min((long long)kTRows, rows - r0);
        __syncthreads();  // the previous tile's last layer is done with XT, WT and Bs
        // the tile's g rows, a warp instruction per 4 rows x 8 columns (four 32-byte
        // global segments; columns 4 apart in XT, 32 different banks), walked by
        // pointer increments
        for (int rb = t >> 5; 4 * rb < kTRows; rb += kTThreads / 32) {
            const int rr = 4 * rb + (t & 3);
            int d = (t & 31) >> 2;
            float *dst = XT + d * kTLd + tiled_col(rr);
            if (rr < nr) {
                const float *src = g + (r0 + rr) * D + d;
                for (; d < D; d += 8, src += 8, dst += 8 * kTLd) cp_async4(dst, src);
            } else {
                for (; d < D; d += 8, dst += 8 * kTLd) *dst = 0.f;
            }
        }
        stage_layer(m, w, 0, WT, Bs);
        cp_async_wait_all();
        __syncthreads();
        for (int L = 0; L < m.n_layers; ++L) {
            const int K = m.dims[L], N = m.dims[L + 1];
            const int npad = (N + 15) / 16 * 16;
            const bool last = L == m.n_layers - 1, wide = npad == kTMaxW;
            const float *xk = XT + 4 * rg;
            if (last) {
                // the output layer (one column, N = 1): the 32 column groups split k (group
                // cg sums k = cg, cg + 32, ... in ascending order over its 8 rows), the
                // partial sums meet in the activation buffer and add up in group order
                // after the bias
                float part[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) part[i] = 0.f;
                for (int k = cg; k < K; k += kTGroups) {
                    const float4 x0 = *reinterpret_cast<const float4 *>(xk + k * kTLd);
                    const float4 x1 = *reinterpret_cast<const float4 *>(xk + k * kTLd + kTRows / 2);
                    const float wv = WT[k * kTWs];
                    const float xs[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
                    for (int i = 0; i < 8; ++i) part[i] = fmaf(xs[i], wv, part[i]);
                }
                __syncthreads();  // every thread has read the layer's inputs
                float *sp = XT + cg * kTRows + 8 * rg;  // [group][row], rows 8 rg .. 8 rg + 7
                *reinterpret_cast<float4 *>(sp) = make_float4(part[0], part[1], part[2], part[3]);
                *reinterpret_cast<float4 *>(sp + 4) = make_float4(part[4], part[5], part[6], part[7]);
                __syncthreads();
                if (t < nr) {
                    float e = Bs[0];
                    for (int gq = 0; gq < kTGroups; ++gq) e += XT[gq * kTRows + t];
                    e_out[r0 + t] = e;
                }
                break;
            }
            const int ncol = wide ? kTMaxCw : (npad - cg + kTGroups - 1) / kTGroups;  // this thread's columns
            float acc[8][kTMaxCw];
            if (wide) {
#pragma unroll
                for (int c = 0; c < kTMaxCw; ++c) {
                    const float bc = Bs[wide_col(cg, c)];
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[i][c] = bc;
                }
                // operands of row k: x (8 rows) and w (5 columns); two sets alternate so
                // that row k + 1 is loading while row k's 40 multiply-adds issue
                struct Ops {
                    float4 x0, x1, w0;
                    float w1;
                };
                auto load = [&](const float *px, const float *pw) {
                    Ops o;
                    o.x0 = *reinterpret_cast<const float4 *>(px);
                    o.x1 = *reinterpret_cast<const float4 *>(px + kTRows / 2);
                    o.w0 = *reinterpret_cast<const float4 *>(pw + 4 * cg);
                    o.w1 = pw[128 + cg];
                    return o;
                };
                auto fma40 = [&](const Ops &o) {
                    const float xs[8] = {o.x0.x, o.x0.y, o.x0.z, o.x0.w, o.x1.x, o.x1.y, o.x1.z, o.x1.w};
                    const float ws[kTMaxCw] = {o.w0.x, o.w0.y, o.w0.z, o.w0.w, o.w1};
#pragma unroll
                    for (int c = 0; c < kTMaxCw; ++c)
#pragma unroll
                        for (int i = 0; i < 8; ++i) acc[i][c] = fmaf(xs[i], ws[c], acc[i][c]);
                };
                const float *px = xk, *pw = WT;
                Ops a = load(px, pw);
                for (int k = 0; k < K; k += 2, px += 2 * kTLd, pw += 2 * kTWs) {
                    const Ops b = load(px + kTLd, pw + kTWs);  // row k + 1 (a padding row when k + 1 = K)
                    fma40(a);
                    if (k + 1 < K) {
                        a = load(px + 2 * kTLd, pw + 2 * kTWs);  // row k + 2 (<= K + 1)
                        fma40(b);
                    }
                }
            } else if (ncol == 1) {  // one column (a hidden layer of width 16 or less: column cg < 16)
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i][0] = Bs[cg];
                const float *px = xk, *pw = WT + cg;
                for (int k = 0; k < K; ++k, px += kTLd, pw += kTWs) {
                    const float4 x0 = *reinterpret_cast<const float4 *>(px);
                    const float4 x1 = *reinterpret_cast<const float4 *>(px + kTRows / 2);
                    const float wv = *pw;
                    const float xs[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[i][0] = fmaf(xs[i], wv, acc[i][0]);
                }
            } else if (ncol > 1) {
#pragma unroll
                for (int c = 0; c < kTMaxCw; ++c) {
                    const float bc = c < ncol ? Bs[narrow_col(cg, c)] : 0.f;
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[i][c] = bc;
                }
                for (int k = 0; k < K; ++k) {
                    const float4 x0 = *reinterpret_cast<const float4 *>(xk + k * kTLd);
                    const float4 x1 = *reinterpret_cast<const float4 *>(xk + k * kTLd + kTRows / 2);
                    const float xs[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
                    for (int c = 0; c < kTMaxCw; ++c) {
                        if (c < ncol) {
                            const float wv = WT[k * kTWs + narrow_col(cg, c)];
#pragma unroll
                            for (int i = 0; i < 8; ++i) acc[i][c] = fmaf(xs[i], wv, acc[i][c]);
                        }
                    }
                }
            }
            __syncthreads();  // every thread has read this layer's inputs and weights
            stage_layer(m, w, L + 1, WT, Bs);  // in flight while the outputs are written
#pragma unroll
            for (int c = 0; c < kTMaxCw; ++c) {
                if (c < ncol) {
                    float o[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) o[i] = act_f(m.act, acc[i][c]);
                    float *yp = XT + (wide ? wide_col(cg, c) : narrow_col(cg, c)) * kTLd + 4 * rg;
                    *reinterpret_cast<float4 *>(yp) = make_float4(o[0], o[1], o[2], o[3]);
                    *reinterpret_cast<float4 *>(yp + kTRows / 2) = make_float4(o[4], o[5], o[6], o[7]);
                }
            }
            cp_async_wait_all();
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------- differences + scatter
struct FdConst {
    float dx, dteta, en_min, en_range;
};

__device__ __forceinline__ float fd_value(float ev, float e0, float step, float en_range) {
    // -(e_v - e_0) / step * (en_max - en_min), then the +-100 clip
    // (ForceEvaluator.py:100-132), FP32 with the reference's rounding
    return clip100(__fmul_rn(__fdiv_rn(-__fsub_rn(ev, e0), step), en_range));
}

__global__ void k_fd_scatter(const float *e, long long P, const int *pairs, FdConst c, float *F, float *T, double *pe) {
    double local = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        float e0 = e[p];
        int i = pairs[2 * p], j = pairs[2 * p + 1];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float f = fd_value(e[(1 + k) * P + p], e0, c.dx, c.en_range);
            float ti = fd_value(e[(4 + k) * P + p], e0, c.dteta, c.en_range);
            float tj = fd_value(e[(7 + k) * P + p], e0, c.dteta, c.en_range);
            atomicAdd(F + 3 * i + k, f);
            atomicAdd(F + 3 * j + k, -f);
            atomicAdd(T + 3 * i + k, ti);
            atomicAdd(T + 3 * j + k, tj);
        }
        local += (double)c.en_min + (double)c.en_range * (double)e0;
    }
    if (pe) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
        if ((threadIdx.x & 31) == 0 && local != 0.0) atomicAdd(pe, local);
    }
}

// ---------------------------------------------------------------- fused plain path
constexpr int kFusedMaxWidth = 64;

struct FusedNet {
    int n_layers, act;
    int dims[AMLP_MAX_LAYERS + 1];
    int npad[AMLP_MAX_LAYERS];       // output width rounded up to 8 (hidden layers)
    int wt_off[AMLP_MAX_LAYERS];     // offset of layer k's transposed weights in smem
    int b_off[AMLP_MAX_LAYERS];      // offset of its bias
    long long woff[AMLP_MAX_LAYERS];  // offset in the packed global weights
    int wt_total;
};

// Activations of the fused net are feature-major, YT[n*kRows + col], with the
// rows permuted: row r = 8 rg + 4 hf + i (i < 4) sits at column
// hf * kRows/2 + 4 rg + i. A thread owns the 8 rows of one rg; the 8 threads
// of a quarter warp take consecutive rg, so their float4 loads and stores of
// activations cover 128 contiguous bytes (no bank conflicts) and they share
// the weight loads (broadcast).
static_assert(kRows % 8 == 0 && (kRows / 8) % 4 == 0, "rows come in groups of 8, a multiple of 4 groups");
static_assert(kFusedThreads % 128 == 0, "the fused kernel's warps are a multiple of four");
__host__ __device__ constexpr int act_col(int r) { return ((r >> 2) & 1) * (kRows / 2) + (r >> 3) * 4 + (r & 3); }

// YT[n][r] = act(b[n] + sum_k XT[k][r] WT[k*npad + n]) for n < npad, rows in the
// permuted layout above; 8x8 register tiles. The items are dealt to the SM's
// four schedulers (warp % 4) in four equal consecutive ranges, a quarter of the
// work each (the block holds the same number of warps per scheduler); inside a
// range the scheduler's warps take consecutive items.
__device__ __forceinline__ void tile_gemm(const float *XT, int K, const float *WT, const float *b, int npad, float *YT,
                                          int act) {
    constexpr int nrg = kRows / 8, hoff = kRows / 2;
    const int items = nrg * (npad / 8);  // a multiple of 4 (nrg is)
    const int per = items / 4, warp = threadIdx.x >> 5, per_sched = (blockDim.x >> 7) * 32;
    const int base = (warp & 3) * per;
    for (int li = (warp >> 2) * 32 + (threadIdx.x & 31); li < per; li += per_sched) {
        const int it = base + li;
        const int rg = it % nrg, cg = it / nrg;
        float acc[8][8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float bj = b[cg * 8 + j];
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[i][j] = bj;
        }
        // operands of row k; two sets alternate so that row k + 1 loads while row k's 64
        // multiply-adds issue. The load of row K (past the last) reads the next area of
        // the shared memory (the following activation buffer, bias or layer) and is unused.
        struct Ops {
            float4 x0, x1, w0, w1;
        };
        auto load = [&](const float *xp, const float *wp) {
            Ops o;
            o.x0 = *reinterpret_cast<const float4 *>(xp);
            o.x1 = *reinterpret_cast<const float4 *>(xp + hoff);
            o.w0 = *reinterpret_cast<const float4 *>(wp);
            o.w1 = *reinterpret_cast<const float4 *>(wp + 4);
            return o;
        };
        auto fma64 = [&](const Ops &o) {
            const float xs[8] = {o.x0.x, o.x0.y, o.x0.z, o.x0.w, o.x1.x, o.x1.y, o.x1.z, o.x1.w};
            const float ws[8] = {o.w0.x, o.w0.y, o.w0.z, o.w0.w, o.w1.x, o.w1.y, o.w1.z, o.w1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(xs[i], ws[j], acc[i][j]);
        };
        const float *xp = XT + rg * 4, *wp = WT + cg * 8;
        Ops a = load(xp, wp);
        for (int k = 0; k < K; k += 2, xp += 2 * kRows, wp += 2 * npad) {
            const Ops bo = load(xp + kRows, wp + npad);  // row k + 1 (row K when k + 1 = K: unused)
            fma64(a);
            if (k + 1 < K) {
                a = load(xp + 2 * kRows, wp + 2 * npad);  // row k + 2 (<= K)
                fma64(bo);
            }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float o[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) o[i] = act_f(act, acc[i][j]);
            float *yp = YT + (cg * 8 + j) * kRows + rg * 4;
            *reinterpret_cast<float4 *>(yp) = make_float4(o[0], o[1], o[2], o[3]);
            *reinterpret_cast<float4 *>(yp + hoff) = make_float4(o[4], o[5], o[6], o[7]);
        }
    }
}

// Segmented (by body index) sum over the lanes of a warp whose keys form
// contiguous runs; returns true on the last lane of each run.
__device__ __forceinline__ bool segmented_sum(int key, float *v, int nv) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ko = __shfl_up_sync(0xffffffffu, key, o);
        for (int q = 0; q < nv; ++q) {
            float y = __shfl_up_sync(0xffffffffu, v[q], o);
            if (lane >= o && ko == key) v[q] += y;
        }
    }
    int kn = __shfl_down_sync(0xffffffffu, key, 1);
    return lane == 31 || kn != key;
}

// Scatter of one tile's per-pair forces/torques, fd[p*9 + (F xyz, T_i xyz, T_j xyz)]:
// F[i] += F, F[j] -= F, T[i] += T_i, T[j] += T_j (ForceEvaluator.py:135-142).
// Warp 0, lane = pair. When the tile's pairs are sorted by i (lists from
// amlp_pair_filter), the i side is summed over runs of equal i first, so one
// atomic per run and component; otherwise one atomic per pair.
__device__ __forceinline__ void scatter_tile(const float *fd, const int *ij, int valid, float *F, float *T) {
    if (threadIdx.x >= 32) return;
    const int p = threadIdx.x;
    const bool ok = p < valid;
    const int i = ij[2 * p], j = ij[2 * p + 1];
    float v[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = ok ? fd[9 * p + k] : 0.f;
        v[3 + k] = ok ? fd[9 * p + 3 + k] : 0.f;
    }
    if (ok) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicAdd(F + 3 * j + k, -v[k]);
            atomicAdd(T + 3 * j + k, fd[9 * p + 6 + k]);
        }
    }
    const bool runs = warp_keys_sorted(i, ok);  // warp-uniform
    bool last = true;
    if (runs) last = segmented_sum(ok ? i : -1 - p, v, 6);
    if (ok && last) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicAdd(F + 3 * i + k, v[k]);
            atomicAdd(T + 3 * i + k, v[3 + k]);
        }
    }
}

template <class Cfg>
__global__ void __launch_bounds__(kFusedThreads, 1) k_forces_fd(const float *pos, const float *quat, float L,
                                                               const int *pairs, const long long *d_np, long long cap,
                                                               const float *pts, int npts, float inv_rc, FdConst c,
                                                               FusedNet net, const float *w, float *F, float *T,
                                                               double *pe, float *e_out) {
    extern __shared__ __align__(16) float smem[];
    const TileGeom g = tile_geom(npts);
    // layout: activations (2 x kFusedMaxWidth x kRows) | weights | e | fd | pts | R | t | ij
    float *bufA = smem;
    float *bufB = bufA + kFusedMaxWidth * kRows;
    float *wt = bufB + kFusedMaxWidth * kRows;
    float *e = wt + net.wt_total;
    float *fd = e + kRows;
    float *pts_s = fd + 9 * kPT;
    float *R = pts_s + 3 * npts;
    float *t = R + kPT * g.rs;
    int *ij = reinterpret_cast<int *>(t + 3 * kPT);
    __shared__ double pe_s[kFusedThreads / 32];
    static_assert(Cfg::NPASS == 2, "the variant split hands the second of two harmonic passes to warps 10 and 11");
    const int warp = threadIdx.x >> 5;
    // descriptor stage: (variant, passes) of this warp; warps 10 and 11 write the
    // second pass of variants 8 and 9 into bufB (free until the first layer),
    // column 32 (v - 8) + pair, and it is added to bufA after the stage
    const int dv = warp < 10 ? warp : warp - 2;
    const unsigned dmask = warp < 8 ? 3u : (warp < 10 ? 1u : 2u);

    for (int k = threadIdx.x; k < 3 * npts; k += blockDim.x) pts_s[k] = pts[k];
    // transposed, zero-padded weights of every layer
    for (int L2 = 0; L2 < net.n_layers; ++L2) {
        const int K = net.dims[L2], N = net.dims[L2 + 1], NP = net.npad[L2];
        const float *W = w + net.woff[L2], *b = W + (size_t)N * K;
        for (int idx = threadIdx.x; idx < K * NP; idx += blockDim.x) {
            int k = idx / NP, n = idx - k * NP;
            wt[net.wt_off[L2] + idx] = n < N ? W[(size_t)n * K + k] : 0.f;
        }
        for (int n = threadIdx.x; n < NP; n += blockDim.x) wt[net.b_off[L2] + n] = n < N ? b[n] : 0.f;
    }
    __syncthreads();

    const long long P = min(*d_np, cap);
    const long long ntiles = (P + kPT - 1) / kPT;
    double pe_acc = 0.0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long p0 = tile * kPT;
        const int valid = (int)min((long long)kPT, P - p0);
        load_tile(pos, quat, L, pairs, P, p0, pts_s, g, R, t, ij);
        __syncthreads();
        tile_descriptor_row<Cfg>(R, t, g, c.dx, c.dteta, inv_rc, warp < 10 ? bufA : bufB, warp < 10 ? kRows : 2 * kPT,
                                 warp < 10 ? act_col(threadIdx.x) : threadIdx.x - kRows, dv, dmask);
        __syncthreads();
        if (warp == 8 || warp == 9) {  // the second pass's angular sums (rows NR..D-1; zero where it has none)
            const int col = act_col(threadIdx.x), sc = threadIdx.x - 8 * kPT;
            for (int d = Cfg::NR; d < Cfg::D; ++d) bufA[d * kRows + col] += bufB[d * (2 * kPT) + sc];
        }
        __syncthreads();
        float *X = bufA, *Y = bufB;
        for (int L2 = 0; L2 + 1 < net.n_layers; ++L2) {
            tile_gemm(X, net.dims[L2], wt + net.wt_off[L2], wt + net.b_off[L2], net.npad[L2], Y, net.act);
            __syncthreads();
            float *tmp = X;
            X = Y;
            Y = tmp;
        }
        {   // last layer (width -> 1), one thread per row
            const int Ll = net.n_layers - 1, K = net.dims[Ll];
            const float *wl = wt + net.wt_off[Ll];
            float acc = wt[net.b_off[Ll]];
            if (threadIdx.x < kRows) {
                const int col = act_col(threadIdx.x);
                for (int k = 0; k < K; ++k) acc = fmaf(wl[k * net.npad[Ll]], X[k * kRows + col], acc);
                e[threadIdx.x] = acc;
                if (e_out && (threadIdx.x & 31) < valid)  // row (variant v, pair p) of e_all: e_out[v P + p0 + p]
                    e_out[(long long)(threadIdx.x >> 5) * P + p0 + (threadIdx.x & 31)] = acc;
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < 9 * kPT; idx += blockDim.x) {
            int p = idx / 9, q = idx - 9 * p;
            int v = 1 + q;  // 1..3 force, 4..6 torque on i, 7..9 torque on j
            fd[idx] = fd_value(e[v * kPT + p], e[p], q < 3 ? c.dx : c.dteta, c.en_range);
        }
        if (threadIdx.x < kPT && threadIdx.x < valid)
            pe_acc += (double)c.en_min + (double)c.en_range * (double)e[threadIdx.x];
        __syncthreads();
        scatter_tile(fd, ij, valid, F, T);
        __syncthreads();
    }
    if (pe) {
        double v = pe_acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) pe_s[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int k = 0; k < kFusedThreads / 32; ++k) s += pe_s[k];
            if (s != 0.0) atomicAdd(pe, s);
        }
    }
}

// ---------------------------------------------------------------- host side
using CfgA = NepCfg<10, 8, 4, 12>;    // D = 47 (the C104 models and every large-scale config)
constexpr int kDirectMaxNd47 = 12;    // clouds up to which the direct form is the cheaper one for D = 47
using CfgB = NepCfg<10, 10, 10, 10>;  // D = 121 (the C100 models)

int hyper_kind(const amlp_nep *n) {
    if (n->nrad == 10 && n->nang == 8 && n->lmax == 4) return 1;
    if (n->nrad == 10 && n->nang == 10 && n->lmax == 10) return 2;
    return 0;
}

amlp_status check_nep(const amlp_nep *n) {
    if (!n || !n->d_pts || n->npts <= 0 || n->npts > AMLP_MAX_PTS || !(n->nep_cutoff > 0.f) || !(n->cutoff > 0.0))
        return AMLP_ERR_INVALID_ARG;
    if (!hyper_kind(n)) return AMLP_ERR_UNSUPPORTED;
    return AMLP_OK;
}

amlp_status check_mlp(const amlp_mlp *m, int D) {
    if (!m || !m->d_w || m->n_layers < 1 || m->n_layers > AMLP_MAX_LAYERS || m->dims[0] != D ||
        m->dims[m->n_layers] != 1 || m->act < 0 || m->act > 2)
        return AMLP_ERR_INVALID_ARG;
    for (int k = 1; k < m->n_layers; ++k)
        if (m->dims[k] <= 0 || m->dims[k] > 1024) return AMLP_ERR_INVALID_ARG;
    return AMLP_OK;
}

int nep_D(const amlp_nep *n) { return (n->nrad + 1) + (n->nang + 1) * n->lmax; }

template <class K>
amlp_status set_smem(K kernel, size_t bytes) {
    if (bytes > 227 * 1024) return AMLP_ERR_UNSUPPORTED;
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return AMLP_OK;
}

}  // namespace amlp

using namespace amlp;

extern "C" amlp_status amlp_descriptors(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                        long long P, const amlp_nep *nep, float *d_g, void *stream) {
    amlp_status st = check_nep(nep);
    if (st) return st;
    if (P < 0 || !d_pos || !d_quat || (P > 0 && (!d_pairs || !d_g))) return AMLP_ERR_INVALID_ARG;
    if (P == 0) return AMLP_OK;
    cudaStream_t s = as_stream(stream);
    TileGeom g = tile_geom(nep->npts);
    int D = nep_D(nep);
    size_t smem = sizeof(float) * (3 * nep->npts + kPT * g.rs + 3 * kPT + 2 * kPT + (size_t)D * (kRows + 1));
    long long ntiles = (P + kPT - 1) / kPT;
    int grid = (int)std::min<long long>(ntiles, 8LL * kNumSM);
    float inv_rc = 1.0f / nep->nep_cutoff;
    // the direct form where it costs less (the rule of the adjoint's descriptor passes) and its
    // per-thread clouds fit the shared memory
    const size_t smem_direct = smem + sizeof(float4) * (size_t)g.nd * kTileThreads;
    const bool direct = (hyper_kind(nep) == 2 || g.nd <= kDirectMaxNd47) && smem_direct <= 227 * 1024;
    if (direct) {
        auto kern = hyper_kind(nep) == 2 ? k_descriptors_direct<11, 11, 10> : k_descriptors_direct<11, 9, 4>;
        if ((st = set_smem(kern, smem_direct))) return st;
        kern<<<grid, kTileThreads, smem_direct, s>>>(d_pos, d_quat, box, d_pairs, P, nep->d_pts, nep->npts, nep->dx,
                                                     nep->dteta, inv_rc, d_g);
    } else if (hyper_kind(nep) == 1) {
        if ((st = set_smem(k_descriptors<CfgA>, smem))) return st;
        k_descriptors<CfgA><<<grid, kTileThreads, smem, s>>>(d_pos, d_quat, box, d_pairs, P, nep->d_pts, nep->npts,
                                                             nep->dx, nep->dteta, inv_rc, d_g);
    } else {
        if ((st = set_smem(k_descriptors<CfgB>, smem))) return st;
        k_descriptors<CfgB><<<grid, kTileThreads, smem, s>>>(d_pos, d_quat, box, d_pairs, P, nep->d_pts, nep->npts,
                                                             nep->dx, nep->dteta, inv_rc, d_g);
    }
    return check_launch();
}

extern "C" amlp_status amlp_mlp_energy(const float *d_g, long long rows, const amlp_mlp *mlp, float *d_e,
                                       void *stream) {
    if (!mlp || rows < 0) return AMLP_ERR_INVALID_ARG;
    amlp_status st = check_mlp(mlp, mlp->dims[0]);
    if (st) return st;
    if (rows == 0) return AMLP_OK;
    if (!d_g || !d_e) return AMLP_ERR_INVALID_ARG;
    MlpDesc m;
    m.n_layers = mlp->n_layers;
    m.act = mlp->act;
    long long off = 0;
    int amax = 1;
    for (int k = 0; k <= mlp->n_layers; ++k) {
        m.dims[k] = mlp->dims[k];
        amax = std::max(amax, mlp->dims[k]);
    }
    for (int k = 0; k < mlp->n_layers; ++k) {
        m.woff[k] = off;
        off += (long long)mlp->dims[k + 1] * mlp->dims[k] + mlp->dims[k + 1];
    }
    if (amax <= kTMaxW) {  // the register-tiled kernel
        size_t smem = sizeof(float) * ((size_t)kTRowsK * kTLd + (size_t)kTRowsK * kTWs + kTMaxW);
        if ((st = set_smem(k_mlp_tiled, smem))) return st;
        long long tiles = (rows + kTRows - 1) / kTRows;
        int grid = (int)std::min<long long>(tiles, kNumSM);  // one CTA per SM (188 KB of shared memory)
        k_mlp_tiled<<<grid, kTThreads, smem, as_stream(stream)>>>(d_g, rows, m, mlp->d_w, d_e);
        return check_launch();
    }
    size_t smem = 2 * sizeof(float) * (size_t)amax * kMlpRows;
    if ((st = set_smem(k_mlp, smem))) return st;
    long long tiles = (rows + kMlpRows - 1) / kMlpRows;
    int grid = (int)std::min<long long>(tiles, 16LL * kNumSM);
    k_mlp<<<grid, kMlpRows, smem, as_stream(stream)>>>(d_g, rows, m, mlp->d_w, amax, d_e);
    return check_launch();
}

extern "C" amlp_status amlp_fd_scatter(const float *d_e, long long P, const int *d_pairs, const amlp_nep *nep,
                                       float *d_F, float *d_T, double *d_pe, void *stream) {
    if (!nep || P < 0 || !d_F || !d_T) return AMLP_ERR_INVALID_ARG;
    if (P == 0) return AMLP_OK;
    if (!d_e || !d_pairs) return AMLP_ERR_INVALID_ARG;
    FdConst c{nep->dx, nep->dteta, nep->en_min, nep->en_max - nep->en_min};
    int grid = (int)std::min<long long>((P + 255) / 256, 4LL * kNumSM);
    k_fd_scatter<<<grid, 256, 0, as_stream(stream)>>>(d_e, P, d_pairs, c, d_F, d_T, d_pe);
    return check_launch();
}

static amlp_status launch_fd(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                             const long long *d_npairs, long long cap, const amlp_nep *nep, const amlp_mlp *mlp,
                             float *d_F, float *d_T, double *d_pe, float *d_e, void *stream) {
    amlp_status st = check_nep(nep);
    if (st) return st;
    int D = nep_D(nep);
    if ((st = check_mlp(mlp, D))) return st;
    if (!d_pos || !d_quat || !d_npairs || !d_F || !d_T || cap < 0 || (cap > 0 && !d_pairs)) return AMLP_ERR_INVALID_ARG;
    if (cap == 0) return AMLP_OK;
    if (D > kFusedMaxWidth) return AMLP_ERR_UNSUPPORTED;
    FusedNet net;
    net.n_layers = mlp->n_layers;
    net.act = mlp->act;
    long long off = 0;
    int woff = 0;
    for (int k = 0; k <= mlp->n_layers; ++k) net.dims[k] = mlp->dims[k];
    for (int k = 0; k < mlp->n_layers; ++k) {
        if (k + 1 < mlp->n_layers && mlp->dims[k + 1] > kFusedMaxWidth) return AMLP_ERR_UNSUPPORTED;
        net.npad[k] = (mlp->dims[k + 1] + 7) / 8 * 8;
        net.woff[k] = off;
        off += (long long)mlp->dims[k + 1] * mlp->dims[k] + mlp->dims[k + 1];
        net.wt_off[k] = woff;
        woff += mlp->dims[k] * net.npad[k];
        net.b_off[k] = woff;
        woff += net.npad[k];
    }
    net.wt_total = (woff + 3) / 4 * 4;
    TileGeom g = tile_geom(nep->npts);
    size_t smem = sizeof(float) * (2 * (size_t)kFusedMaxWidth * kRows + net.wt_total + kRows + 9 * kPT + 3 * nep->npts +
                                   kPT * g.rs + 3 * kPT + 2 * kPT);
    FdConst c{nep->dx, nep->dteta, nep->en_min, nep->en_max - nep->en_min};
    float inv_rc = 1.0f / nep->nep_cutoff;
    cudaStream_t s = as_stream(stream);
    int grid = kNumSM;
    if (hyper_kind(nep) == 1) {
        if ((st = set_smem(k_forces_fd<CfgA>, smem))) return st;
        k_forces_fd<CfgA><<<grid, kFusedThreads, smem, s>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep->d_pts,
                                                           nep->npts, inv_rc, c, net, mlp->d_w, d_F, d_T, d_pe, d_e);
    } else {
        return AMLP_ERR_UNSUPPORTED;
    }
    return check_launch();
}

extern "C" amlp_status amlp_forces_fd(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                      const long long *d_npairs, long long cap, const amlp_nep *nep,
                                      const amlp_mlp *mlp, float *d_F, float *d_T, double *d_pe, void *stream) {
    return launch_fd(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep, mlp, d_F, d_T, d_pe, nullptr, stream);
}

extern "C" amlp_status amlp_forces_fd_energies(const float *d_pos, const float *d_quat, float box,
                                               const int *d_pairs, const long long *d_npairs, long long cap,
                                               const amlp_nep *nep, const amlp_mlp *mlp, float *d_F, float *d_T,
                                               double *d_pe, float *d_e, void *stream) {
    if (!d_e && cap > 0) return AMLP_ERR_INVALID_ARG;
    return launch_fd(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep, mlp, d_F, d_T, d_pe, d_e, stream);
}
