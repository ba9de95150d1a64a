// Weight gradient of the pair-energy net for a training step, the loss of the
// reference's training loop (05/FFNN.py:95-106, torch.nn.MSELoss over a batch)
// on energies normalised as 05/FFNN.py:59-63 does (the caller passes
// y = clamp((min(E, en_max) - en_min) / (en_max - en_min), 0, 1)):
//   L = (1/B) sum_r (net(g_r) - y_r)^2.
// The same kernel also backpropagates a given per-row upstream gradient dy_r
// (a vector-Jacobian product, sum_r dy_r d net(g_r) / d theta).
// Backpropagation into every weight and bias, FP32. A CTA takes 32 rows: the
// forward keeps pre-activations and activations of its rows in shared memory,
// the backward forms the deltas and adds its rows' share of dL/dW and dL/db to
// the caller's gradient buffer (one atomic per weight per CTA).
#include "common.cuh"

namespace amlp {
namespace {

constexpr int kTrainRows = 32;
constexpr int kTrainThreads = 128;
constexpr int kTrainMaxWidth = 256;

struct TrainNet {
    int n_layers, act;
    int dims[AMLP_MAX_LAYERS + 1];
    long long woff[AMLP_MAX_LAYERS];
    int aoff[AMLP_MAX_LAYERS + 1];  // float offset of layer k's activations (rows x dims[k]) in smem
    int total;                      // floats of activations (and as many for pre-activations / deltas)
};

__global__ void __launch_bounds__(kTrainThreads) k_mlp_loss_grad(const float *g, const float *y, const float *dy,
                                                                 long long rows, TrainNet net, const float *w,
                                                                 float *grad, double *loss) {
    extern __shared__ float sm[];
    float *act = sm;               // activations a_k[r][i], k = 0..n_layers (a_0 = g)
    float *pre = sm + net.total;   // pre-activations z_k (k >= 1), then deltas in place
    const int tid = threadIdx.x;
    const float inv_b = 1.0f / (float)rows;
    for (long long r0 = (long long)blockIdx.x * kTrainRows; r0 < rows; r0 += (long long)gridDim.x * kTrainRows) {
        const int nr = (int)min((long long)kTrainRows, rows - r0);
        const int D = net.dims[0];
        for (int idx = tid; idx < kTrainRows * D; idx += kTrainThreads) {
            int r = idx / D, d = idx - r * D;
            act[net.aoff[0] + idx] = r < nr ? g[(r0 + r) * D + d] : 0.f;
        }
        __syncthreads();
        // forward
        for (int L = 0; L < net.n_layers; ++L) {
            const int K = net.dims[L], N = net.dims[L + 1];
            const float *W = w + net.woff[L], *b = W + (size_t)N * K;
            const bool last = L == net.n_layers - 1;
            for (int n = tid; n < N; n += kTrainThreads) {
                float acc[kTrainRows];
#pragma unroll
                for (int r = 0; r < kTrainRows; ++r) acc[r] = __ldg(b + n);
                for (int k = 0; k < K; ++k) {
                    float wv = __ldg(W + (size_t)n * K + k);
#pragma unroll
                    for (int r = 0; r < kTrainRows; ++r) acc[r] = fmaf(wv, act[net.aoff[L] + r * K + k], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < kTrainRows; ++r) {
                    pre[net.aoff[L + 1] + r * N + n] = acc[r];
                    act[net.aoff[L + 1] + r * N + n] = last ? acc[r] : act_f(net.act, acc[r]);
                }
            }
            __syncthreads();
        }
        // output delta: dy, or dL/dz_last = 2 (net - y) / B and the loss
        const int Ll = net.n_layers;
        if (tid < kTrainRows) {
            float d = 0.f;
            double l = 0.0;
            if (tid < nr && dy) {
                d = dy[r0 + tid];
            } else if (tid < nr) {
                float e = act[net.aoff[Ll] + tid] - y[r0 + tid];
                d = 2.0f * e * inv_b;
                l = (double)e * (double)e / (double)rows;
            }
            pre[net.aoff[Ll] + tid] = d;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
            if (tid == 0 && loss) atomicAdd(loss, l);
        }
        __syncthreads();
        // backward: delta_L (rows x N) in pre[aoff[L+1]]
        for (int L = net.n_layers - 1; L >= 0; --L) {
            const int K = net.dims[L], N = net.dims[L + 1];
            const float *W = w + net.woff[L];
            float *gW = grad + net.woff[L], *gb = gW + (size_t)N * K;
            const float *delta = pre + net.aoff[L + 1];
            const float *a = act + net.aoff[L];
            for (int n = tid; n < N; n += kTrainThreads) {
                float sb = 0.f;
                for (int r = 0; r < nr; ++r) sb += delta[r * N + n];
                atomicAdd(gb + n, sb);
                for (int k = 0; k < K; ++k) {
                    float s = 0.f;
                    for (int r = 0; r < nr; ++r) s = fmaf(delta[r * N + n], a[r * K + k], s);
                    atomicAdd(gW + (size_t)n * K + k, s);
                }
            }
            if (L > 0) {
                // delta_{L-1}[r][k] = sum_n W[n][k] delta_L[r][n] * act'(z_{L-1}[r][k])
                float *dprev = pre + net.aoff[L];
                for (int k = tid; k < K; k += kTrainThreads) {
                    float s[kTrainRows];
#pragma unroll
                    for (int r = 0; r < kTrainRows; ++r) s[r] = 0.f;
                    for (int n = 0; n < N; ++n) {
                        float wv = __ldg(W + (size_t)n * K + k);
#pragma unroll
                        for (int r = 0; r < kTrainRows; ++r) s[r] = fmaf(wv, delta[r * N + n], s[r]);
                    }
#pragma unroll
                    for (int r = 0; r < kTrainRows; ++r) s[r] *= act_df(net.act, dprev[r * K + k]);
#pragma unroll
                    for (int r = 0; r < kTrainRows; ++r) dprev[r * K + k] = s[r];
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace

amlp_status check_mlp(const amlp_mlp *m, int D);

}  // namespace amlp

using namespace amlp;

static amlp_status launch_grad(const float *d_g, const float *d_y, const float *d_dy, long long rows,
                               const amlp_mlp *mlp, float *d_grad, double *d_loss, void *stream) {
    if (!mlp || rows < 0) return AMLP_ERR_INVALID_ARG;
    amlp_status st = check_mlp(mlp, mlp->dims[0]);
    if (st) return st;
    if (rows == 0) return AMLP_OK;
    if (!d_g || !(d_y || d_dy) || !d_grad) return AMLP_ERR_INVALID_ARG;
    TrainNet net{};
    net.n_layers = mlp->n_layers;
    net.act = mlp->act;
    long long off = 0;
    int aoff = 0;
    for (int k = 0; k <= mlp->n_layers; ++k) {
        net.dims[k] = mlp->dims[k];
        if (mlp->dims[k] > kTrainMaxWidth) return AMLP_ERR_UNSUPPORTED;
        net.aoff[k] = aoff;
        aoff += kTrainRows * mlp->dims[k];
    }
    for (int k = 0; k < mlp->n_layers; ++k) {
        net.woff[k] = off;
        off += (long long)mlp->dims[k + 1] * mlp->dims[k] + mlp->dims[k + 1];
    }
    net.total = aoff;
    size_t smem = (size_t)2 * aoff * sizeof(float);
    if (smem > 220 * 1024) return AMLP_ERR_UNSUPPORTED;
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(k_mlp_loss_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    long long tiles = (rows + kTrainRows - 1) / kTrainRows;
    int grid = (int)std::min<long long>(tiles, 4LL * kNumSM);
    k_mlp_loss_grad<<<grid, kTrainThreads, smem, as_stream(stream)>>>(d_g, d_y, d_dy, rows, net, mlp->d_w, d_grad,
                                                                      d_dy ? nullptr : d_loss);
    return check_launch();
}

extern "C" amlp_status amlp_mlp_loss_grad(const float *d_g, const float *d_y, long long rows, const amlp_mlp *mlp,
                                          float *d_grad, double *d_loss, void *stream) {
    if (!d_y && rows > 0) return AMLP_ERR_INVALID_ARG;
    return launch_grad(d_g, d_y, nullptr, rows, mlp, d_grad, d_loss, stream);
}

extern "C" amlp_status amlp_mlp_backward(const float *d_g, const float *d_dy, long long rows, const amlp_mlp *mlp,
                                         float *d_grad, void *stream) {
    if (!d_dy && rows > 0) return AMLP_ERR_INVALID_ARG;
    return launch_grad(d_g, nullptr, d_dy, rows, mlp, d_grad, nullptr, stream);
}
