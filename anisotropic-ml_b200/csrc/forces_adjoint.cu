// Adjoint force path: exact forces and torques of the pair energy
// E = en_min + (en_max - en_min) * net(g(cloud)) instead of the reference's
// ten finite-difference evaluations (ForceEvaluator.py:86-112).
//
// One CTA works on tiles of 128 pairs with 256 threads; thread t handles pair
// p = t % 128 and the half h = t / 128 of the harmonics (and the same TMEM
// lane p in the tensor-core epilogues). Per tile:
//   1  stage the rotated body points of the pairs in shared memory;
//   2  descriptor forward (FP32): g = [sum_a f_n(a) | sum_m A_{n,lm}^2];
//   3  net forward and backward on the tensor cores: every product is three
//      bf16 x bf16 -> fp32 MMAs (hi*hi + hi*lo + lo*hi of the bf16 splits of
//      activations and weights), accumulators in TMEM; gives dE/dg;
//   4  descriptor backward (FP32): the per-point quantities are recomputed
//      instead of stored (only the per-pair sums A stay in registers across the
//      net): dE/dA = 2 dE/dg_ang A, then per point
//      dE/dr_a = sum_n dE/df_n f_n'(d) rhat + sum_lm dE/dY_lm grad Y_lm;
//   5  F_pair = -sum_{a in i} dE/dp_a, T_i = -sum_{a in i} p_a x dE/dp_a,
//      T_j = -sum_{a in j} (p_a - t) x dE/dp_a (dE/dp_a = dE/dr_a minus the mean,
//      the centroid moving with every point), times (en_max - en_min), clipped
//      to [-100, 100] and scattered like the reference (ForceEvaluator.py:119-142).
// Nets: 1 to 3 hidden layers of width <= 64, D <= 64.
#include "descriptor.cuh"
#include "descriptor_direct.cuh"
#include "tcgen05.cuh"

namespace amlp {

__device__ unsigned int g_amlp_device_error = 0;
// Test hook (amlp_test_first_wait_limit): polls allowed to the first MMA-completion
// wait of every CTA of k_forces_adjoint; -1 keeps the normal limit. 0 makes that
// wait give up at once, which exercises the abort path without any fault.
__device__ int g_amlp_first_wait_limit = -1;

namespace {

constexpr int kAP = 128;          // pairs per tile (MMA M)
constexpr int kAThreads = 256;
constexpr int kMaxHidden = 3;      // hidden layers of the fused kernel
constexpr int kMaxHiddenWide = 4;  // hidden layers of the wide path: layer_first + 3 (TheEnergyNet(150, 3, D))
constexpr int kWpad = 64;          // hidden widths padded to 64 in TMEM regions
constexpr uint32_t kErrMbarTimeout = 1u;
// Shared-memory row strides of per-pair arrays, odd so that the 32 pairs of a
// warp (thread = pair) hit 32 different banks.
constexpr int kGS = 49;           // descriptor partials / dE/dg rows (48 used)
constexpr int kPartStride = 13;   // gradient partial sums (12 used)

struct AdjNet {
    int nh;                              // hidden layers
    int act;
    int kin[kMaxHiddenWide + 1];         // padded input width of hidden layer k (multiple of 16)
    int nout[kMaxHiddenWide + 1];        // padded output width of hidden layer k (multiple of 16)
    int dims[kMaxHiddenWide + 2];        // true dims: D, h1, .., h_nh, 1
    long long woff[kMaxHiddenWide + 1];  // offset of W_k in the packed global weights (k = 0..nh)
    int wsm_off[kMaxHiddenWide];         // byte offset of W_k (hi) in the weight area; lo follows (the wide
                                         // path: in the pre-split global copy of the weights)
    int wsm_total;                       // bytes of the weight area
    int bias_off[kMaxHiddenWide + 1];    // float offsets of b_k in the fp32 parameter area; last = w_last
    int par_total;
    // k_mlp_grad only (set by wide_net): row strides of the g and dE/dg rows, widest
    // hidden layer, TMEM columns of the product region, act'(z) as bits (ReLU),
    // shared-memory carve-up and whether the next tile's g rows are prefetched
    int g_ld, gp, wmax, zbw, relu_bits;
    int wbuf_off, par_off, eps_off, gbuf_off, prefetch_g, smem;
};

// Activation and its derivative from one exponential, for the tensor-core
// epilogues (the net there is accurate to about 1e-5 relative, so the fast
// exponential's few-ulp error does not show): tanh(z) = 1 - 2 / (1 + e^(2z)),
// tanh' = 1 - tanh^2; silu(z) = z s, silu' = s (1 + z (1 - s)), s = 1 / (1 + e^-z).
__device__ __forceinline__ void act_pair(int act, float z, float &f, float &df) {
    if (act == AMLP_ACT_RELU) {
        f = fmaxf(z, 0.0f);
        df = z > 0.0f ? 1.0f : 0.0f;
    } else if (act == AMLP_ACT_TANH) {
        const float t = 1.0f - __fdividef(2.0f, 1.0f + __expf(2.0f * z));
        f = t;
        df = fmaf(-t, t, 1.0f);
    } else {
        const float sg = __fdividef(1.0f, 1.0f + __expf(-z));
        f = z * sg;
        df = sg * fmaf(z, 1.0f - sg, 1.0f);
    }
}

// Radial basis f_n of the adjoint kernels, with the cutoff function from the
// hardware sine/cosine (__sincosf: a few 1e-7 absolute error for the
// arguments here, far below the tensor-core net's 1e-5), used by both their
// forward and their backward so that the forces stay the exact derivative of
// the energy they compute.
template <int NR>
__device__ __forceinline__ void radial_basis_fast(float d, float inv_rc, float *f) {
    const float u = d * inv_rc, um1 = u - 1.0f;
    const float x = fmaf(2.0f * um1, um1, -1.0f);
    float s, c;
    __sincosf(3.14159265358979f * u, &s, &c);
    const float hfc = fmaf(0.25f, c, 0.25f);  // fc / 2
    float tm1 = 1.0f, t = x;
    f[0] = 2.0f * hfc;
    if (NR > 1) f[1] = fmaf(hfc, x, hfc);
#pragma unroll
    for (int n = 2; n < NR; ++n) {
        const float tn = fmaf(2.0f * x, t, -tm1);
        tm1 = t;
        t = tn;
        f[n] = fmaf(hfc, tn, hfc);
    }
}

// Derivative of f_n with respect to the distance d, together with f_n (same
// arithmetic as radial_basis_fast for f_n).
template <int NR>
__device__ __forceinline__ void radial_basis_grad(float d, float inv_rc, float *f, float *df) {
    const float u = d * inv_rc, um1 = u - 1.0f;
    const float x = fmaf(2.0f * um1, um1, -1.0f);
    float s, c;
    __sincosf(3.14159265358979f * u, &s, &c);
    const float hfc = fmaf(0.25f, c, 0.25f);                        // fc / 2
    const float hdfc = -0.25f * 3.14159265358979f * s * inv_rc;      // (dfc/dd) / 2
    const float hdxfc = 4.0f * um1 * inv_rc * hfc;                   // (dx/dd) fc / 2
    float tm1 = 1.0f, t = x, dtm1 = 0.0f, dt = 1.0f;                // T_n and dT_n/dx
    f[0] = 2.0f * hfc;
    df[0] = 2.0f * hdfc;
    if (NR > 1) {
        f[1] = fmaf(hfc, x, hfc);
        df[1] = fmaf(hdfc, x, hdfc) + hdxfc;
    }
#pragma unroll
    for (int n = 2; n < NR; ++n) {
        const float tn = fmaf(2.0f * x, t, -tm1);
        const float dtn = fmaf(2.0f * x, dt, fmaf(2.0f, t, -dtm1));
        tm1 = t;
        t = tn;
        dtm1 = dt;
        dt = dtn;
        f[n] = fmaf(hfc, tn, hfc);
        df[n] = fmaf(dtn, hdxfc, fmaf(hdfc, tn, hdfc));
    }
}

// The recurrences behind the harmonics: C_m + i S_m = (x + i y)^m (m <= LMAX)
// and Q[l][m] = d^m P_l / dz^m (m <= l + 1 <= LMAX + 1; 0 above l).
template <int LMAX>
__device__ __forceinline__ void sh_recurrences(float x, float y, float z, float *C, float *S,
                                               float (&Q)[LMAX + 2][LMAX + 2]) {
    C[0] = 1.0f;
    S[0] = 0.0f;
#pragma unroll
    for (int m = 1; m <= LMAX; ++m) {
        C[m] = fmaf(x, C[m - 1], -y * S[m - 1]);
        S[m] = fmaf(x, S[m - 1], y * C[m - 1]);
    }
#pragma unroll
    for (int l = 0; l <= LMAX + 1; ++l)
#pragma unroll
        for (int m = 0; m <= LMAX + 1; ++m) Q[l][m] = 0.0f;
#pragma unroll
    for (int m = 0; m <= LMAX; ++m) {
#pragma unroll
        for (int l = m; l <= LMAX; ++l) {
            if (l == m) Q[l][m] = (float)dfact_odd(m);
            else if (l == m + 1) Q[l][m] = (float)(2 * m + 1) * z * Q[l - 1][m];
            else
                Q[l][m] = ((float)(2 * l - 1) * z * Q[l - 1][m] - (float)(l + m - 1) * Q[l - 2][m]) *
                          (1.0f / (float)(l - m));
        }
    }
}

__host__ __device__ constexpr int sh_m_of(int k) {  // m of harmonic index k (order m = 0, (cos, sin) m = 1..l)
    return (k + 1 - sh_l_of(k) * sh_l_of(k) + 1) / 2;
}
__host__ __device__ constexpr bool sh_is_sin(int k) {
    return sh_m_of(k) > 0 && ((k + 1 - sh_l_of(k) * sh_l_of(k)) % 2 == 0);
}

// Weight of harmonic k in the angular descriptor when the harmonics are kept
// unnormalised (Q_l^m {C_m, S_m}): N_lm^2 = 2 (l-m)! / (l+m)! for m >= 1, 1 for
// m = 0, so that g[n][l] = sum_m N_lm^2 (sum_a f_n Q_l^m {C_m, S_m})^2.
__host__ __device__ constexpr float sh_weight(int k) {
    const int l = sh_l_of(k), m = sh_m_of(k);
    if (m == 0) return 1.0f;
    double num = 2.0, den = 1.0;
    for (int v = 2; v <= l - m; ++v) num *= v;
    for (int v = 2; v <= l + m; ++v) den *= v;
    return (float)(num / den);
}

// The unnormalised harmonics Q_l^m {C_m, S_m} (m > 0) and Q_l^0 of this half
// (indices k0 .. k0 + KC - 1, zero past K) from the recurrences.
template <class Cfg, int KC, int k0>
__device__ __forceinline__ void sh_half_u(const float *C, const float *Sn,
                                          const float (&Q)[Cfg::LMAX + 2][Cfg::LMAX + 2], float *Y) {
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
        const int k = k0 + kk;
        if (k < Cfg::K) {
            const int l = sh_l_of(k), m = sh_m_of(k);
            Y[kk] = m == 0 ? Q[l][0] : Q[l][m] * (sh_is_sin(k) ? Sn[m] : C[m]);
        } else {
            Y[kk] = 0.f;
        }
    }
}

template <class Cfg>
struct Half {
    static constexpr int KC = (Cfg::K + 1) / 2;  // harmonics per half
};

// sum_a f_n(a) Y_k(a) for this half's harmonics k0..k0+KC-1, unnormalised (and
// the radial sums). r holds the pair's nd centred points (x, y, z each).
template <class Cfg, int KC, int k0>
__device__ __forceinline__ void accumulate_A(const float *r, int nd, float inv_rc, float (*A)[KC], float *R) {
#pragma unroll
    for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) A[n][kk] = 0.f;
#pragma unroll
    for (int n = 0; n < Cfg::NR; ++n) R[n] = 0.f;
    for (int a = 0; a < nd; ++a) {
        const float rx = r[3 * a], ry = r[3 * a + 1], rz = r[3 * a + 2];
        float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
        float inv_d = rsqrtf(d2);
        float f[Cfg::NR];
        radial_basis_fast<Cfg::NR>(d2 * inv_d, inv_rc, f);
#pragma unroll
        for (int n = 0; n < Cfg::NR; ++n) R[n] += f[n];
        constexpr int LM = Cfg::LMAX;
        float C[LM + 1], Sn[LM + 1], Q[LM + 2][LM + 2];
        sh_recurrences<LM>(rx * inv_d, ry * inv_d, rz * inv_d, C, Sn, Q);
        float Y[KC];
        sh_half_u<Cfg, KC, k0>(C, Sn, Q, Y);
#pragma unroll
        for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
            for (int kk = 0; kk < KC; ++kk)
                if (k0 + kk < Cfg::K) A[n][kk] = fmaf(f[n], Y[kk], A[n][kk]);
    }
}

// Forward of one half of the harmonics: radial sums (half 0) and the partial
// sums of weighted squares of this half's harmonics, written to gp[0..47]
// (zeros elsewhere). The unnormalised sums A of this half stay in the caller's
// registers for the backward.
template <class Cfg, int H>
__device__ __forceinline__ void half_forward(const float *r, int nd, float inv_rc, float *gp,
                                             float (&A)[Cfg::NA][Half<Cfg>::KC]) {
    constexpr int KC = Half<Cfg>::KC;
    float Rr[Cfg::NR];
    accumulate_A<Cfg, KC, H * KC>(r, nd, inv_rc, A, Rr);
    for (int k = 0; k < 48; ++k) gp[k] = 0.f;
    if (H == 0) {
#pragma unroll
        for (int n = 0; n < Cfg::NR; ++n) gp[n] = Rr[n];
    }
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
        if (H * KC + kk < Cfg::K) {
            const int l = sh_l_of(H * KC + kk);
            const float w = sh_weight(H * KC + kk);
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n)
                gp[Cfg::NR + n * Cfg::LMAX + l - 1] = fmaf(w * A[n][kk], A[n][kk], gp[Cfg::NR + n * Cfg::LMAX + l - 1]);
        }
    }
}

// Backward of one half: given dE/dg (dg) and the forward sums A of this half
// (overwritten), the partial sums over the centred points r_a of dE/dr_a
// needed for the pair force and torques: sum_{a in i} G_a, sum_a G_a,
// sum_{a in i} r_a x G_a, sum_{a in j} r_a x G_a -> out[12] (the caller adds
// the centroid terms).
template <class Cfg, int H>
__device__ __forceinline__ void half_backward(const float *r, int npts, float inv_rc, const float *dg, float *out,
                                              float (&A)[Cfg::NA][Half<Cfg>::KC]) {
    constexpr int KC = Half<Cfg>::KC;
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
        if (H * KC + kk < Cfg::K) {
            const int l = sh_l_of(H * KC + kk);
            const float w2 = 2.0f * sh_weight(H * KC + kk);
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n) A[n][kk] *= w2 * dg[Cfg::NR + n * Cfg::LMAX + l - 1];
        } else {
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n) A[n][kk] = 0.f;
        }
    }
    float grad_rad[Cfg::NR];
#pragma unroll
    for (int n = 0; n < Cfg::NR; ++n) grad_rad[n] = H == 0 ? dg[n] : 0.f;
    float Si[3] = {0, 0, 0}, Sj[3] = {0, 0, 0}, Xi[3] = {0, 0, 0}, Xj[3] = {0, 0, 0};
    const int nd = 2 * npts;
    for (int a = 0; a < nd; ++a) {
        const float rx = r[3 * a], ry = r[3 * a + 1], rz = r[3 * a + 2];
        float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
        float inv_d = rsqrtf(d2);
        float d = d2 * inv_d;
        float ux = rx * inv_d, uy = ry * inv_d, uz = rz * inv_d;
        float f[Cfg::NR], df[Cfg::NR];
        radial_basis_grad<Cfg::NR>(d, inv_rc, f, df);
        constexpr int LM = Cfg::LMAX;
        float C[LM + 1], Sn[LM + 1], Q[LM + 2][LM + 2];
        sh_recurrences<LM>(ux, uy, uz, C, Sn, Q);
        float Y[KC];
        sh_half_u<Cfg, KC, H * KC>(C, Sn, Q, Y);
        float gr = 0.f;
#pragma unroll
        for (int n = 0; n < Cfg::NR; ++n) {
            float s = grad_rad[n];
            if (n < Cfg::NA) {
#pragma unroll
                for (int kk = 0; kk < KC; ++kk)
                    if (H * KC + kk < Cfg::K) s = fmaf(A[n][kk], Y[kk], s);
            }
            gr = fmaf(s, df[n], gr);
        }
        // gradient of sum_k s_k Y_k grouped by m: with U_m, V_m the sums of
        // s m Q_l^m over the cos / sin harmonics of order m and Wc_m, Ws_m those
        // of s Q_l^(m+1),
        //   gx = sum_m U_m C_(m-1) + V_m S_(m-1), gy = sum_m V_m C_(m-1) - U_m S_(m-1),
        //   gz = sum_m Wc_m C_m + Ws_m S_m.
        float U[LM + 1], V[LM + 1], Wc[LM + 1], Ws[LM + 1];
#pragma unroll
        for (int m = 0; m <= LM; ++m) U[m] = V[m] = Wc[m] = Ws[m] = 0.f;
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            const int k = H * KC + kk;
            if (k < Cfg::K) {
                float s = 0.f;
#pragma unroll
                for (int n = 0; n < Cfg::NA; ++n) s = fmaf(A[n][kk], f[n], s);
                const int l = sh_l_of(k), m = sh_m_of(k);
                if (sh_is_sin(k)) {
                    V[m] = fmaf(s, m == 1 ? Q[l][m] : (float)m * Q[l][m], V[m]);
                    Ws[m] = fmaf(s, Q[l][m + 1], Ws[m]);
                } else {
                    if (m > 0) U[m] = fmaf(s, m == 1 ? Q[l][m] : (float)m * Q[l][m], U[m]);
                    Wc[m] = fmaf(s, Q[l][m + 1], Wc[m]);
                }
            }
        }
        float gx = 0.f, gy = 0.f, gz = Wc[0];
#pragma unroll
        for (int m = 1; m <= LM; ++m) {
            gx = fmaf(U[m], C[m - 1], fmaf(V[m], Sn[m - 1], gx));
            gy = fmaf(V[m], C[m - 1], fmaf(-U[m], Sn[m - 1], gy));
            gz = fmaf(Wc[m], C[m], fmaf(Ws[m], Sn[m], gz));
        }
        // dE/dr = gr rhat + (g - rhat (rhat . g)) / d = rhat (gr - (rhat . g) / d) + g / d
        const float dot = ux * gx + uy * gy + uz * gz;
        const float c1 = fmaf(-dot, inv_d, gr);
        const float Gx = fmaf(ux, c1, gx * inv_d);
        const float Gy = fmaf(uy, c1, gy * inv_d);
        const float Gz = fmaf(uz, c1, gz * inv_d);
        if (a < npts) {
            Si[0] += Gx;
            Si[1] += Gy;
            Si[2] += Gz;
            Xi[0] += ry * Gz - rz * Gy;
            Xi[1] += rz * Gx - rx * Gz;
            Xi[2] += rx * Gy - ry * Gx;
        } else {
            Sj[0] += Gx;
            Sj[1] += Gy;
            Sj[2] += Gz;
            Xj[0] += ry * Gz - rz * Gy;
            Xj[1] += rz * Gx - rx * Gz;
            Xj[2] += rx * Gy - ry * Gx;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        out[k] = Si[k];
        out[3 + k] = Si[k] + Sj[k];
        out[6 + k] = Xi[k];
        out[9 + k] = Xj[k];
    }
}

struct AdjShared {
    float *R;          // rotated body points, kAP x rs (aliases the MLP operand area)
    char *ops;         // MLP operand area (bf16 hi/lo tiles)
    char *wts;         // weights (bf16 hi/lo), resident
    float *par;        // biases + last-layer weights (fp32)
    float *g0, *g1;    // per-half descriptor partials, kAP x kGS each; g0 later holds dE/dg
    float *t;          // translations, kAP x 3
    float *cen;        // centroids, kAP x 3
    float *part;       // per-half gradient partial sums, 2 x kAP x kPartStride
    float *eps;        // per-half energy partials, 2 x kAP
    float *fd;         // per-pair F, T_i, T_j, kAP x 9
    int *ij;           // pair indices, kAP x 2
    float *pts;        // body points
    float4 *q;         // orientations of the tile's pairs, kAP x 2 (i, j)
    float *psum;       // sum of the body points (body frame), 3
};

// Sum of the body-frame points into S.psum (one warp; call before a barrier).
__device__ __forceinline__ void body_point_sum(const AdjShared &S, int npts) {
    if (threadIdx.x < 32) {
        float v[3] = {0.f, 0.f, 0.f};
        for (int a = threadIdx.x; a < npts; a += 32)
#pragma unroll
            for (int k = 0; k < 3; ++k) v[k] += S.pts[3 * a + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < 3; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < 3; ++k) S.psum[k] = v[k];
    }
}

// Activation tile of layer k in the operand area (hi at its base, lo after it).
// Only two are live at a time (the one an MMA reads and the one its epilogue
// writes), so the layers alternate between two buffers.
__device__ __forceinline__ char *op_tile(char *ops, int k) { return ops + (k & 1) * (2 * kAP * kWpad * 2); }

// A (128 x K) times B, three split terms, into TMEM columns at d_tmem.
// STEP_DESC: build the four descriptors of K-step 0 once and move only their
// start address (bits 0-13, in 16-byte units, below 2^14 for any shared-memory
// address) from step to step; otherwise build them per MMA. Measured: stepping
// is 0.4 % faster in the fused kernel (K <= 64) and 0.7 % slower in k_mlp_grad.
template <bool STEP_DESC>
__device__ __forceinline__ void mma3(uint32_t d_tmem, const char *a_hi, int K, const char *b_hi, size_t b_lo_off,
                                     int N, bool b_mn, int b_kstride /* bytes per K-step of 16 */, uint32_t b_lbo,
                                     uint32_t b_sbo) {
    const uint32_t idesc = tc::idesc_bf16(N, b_mn ? 1 : 0);
    const uint32_t a0 = tc::smem_u32(a_hi), a1 = a0 + (uint32_t)(kAP * K * 2);
    const uint32_t b0 = tc::smem_u32(b_hi), b1 = b0 + (uint32_t)b_lo_off;
    const uint32_t a_sbo = (uint32_t)K * 16;
    if constexpr (STEP_DESC) {
        const uint64_t da = tc::smem_desc(a0, 128, a_sbo), da1 = tc::smem_desc(a1, 128, a_sbo);
        const uint64_t db = tc::smem_desc(b0, b_lbo, b_sbo), db1 = tc::smem_desc(b1, b_lbo, b_sbo);
        for (int ks = 0; ks < K / 16; ++ks) {
            const uint64_t oa = (uint64_t)(ks * 16), ob = (uint64_t)((ks * b_kstride) >> 4);
            tc::mma_bf16(d_tmem, da + oa, db + ob, idesc, ks > 0 ? 1u : 0u);
            tc::mma_bf16(d_tmem, da + oa, db1 + ob, idesc, 1u);
            tc::mma_bf16(d_tmem, da1 + oa, db + ob, idesc, 1u);
        }
    } else {
        for (int ks = 0; ks < K / 16; ++ks) {
            const uint32_t ao = ks * 256, bo = ks * b_kstride;
            tc::mma_bf16(d_tmem, tc::smem_desc(a0 + ao, 128, a_sbo), tc::smem_desc(b0 + bo, b_lbo, b_sbo), idesc,
                         ks > 0 ? 1u : 0u);
            tc::mma_bf16(d_tmem, tc::smem_desc(a0 + ao, 128, a_sbo), tc::smem_desc(b1 + bo, b_lbo, b_sbo), idesc,
                         1u);
            tc::mma_bf16(d_tmem, tc::smem_desc(a1 + ao, 128, a_sbo), tc::smem_desc(b0 + bo, b_lbo, b_sbo), idesc,
                         1u);
        }
    }
}

// Write 8 consecutive values of row p, columns c0..c0+7 into a K-major bf16
// hi/lo tile of width K.
// The splits are rounded two at a time (one packed conversion per pair, the
// same round-to-nearest-even values as tc::split_bf16).
__device__ __forceinline__ void store_split8(char *tile_hi, int K, int p, int c0, const float *v) {
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
        const float2 hf = __bfloat1622float2(h2);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
        hi[k] = *reinterpret_cast<const uint32_t *>(&h2);
        lo[k] = *reinterpret_cast<const uint32_t *>(&l2);
    }
    uint32_t off = tc::kmajor_offset(p, c0, K);
    *reinterpret_cast<uint4 *>(tile_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4 *>(tile_hi + kAP * K * 2 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// Centroid of pair q's cloud into S.cen from its orientations and translation
// (S.q, S.t): c = (R_i s + R_j s + npts t) / (2 npts), s the sum of the
// body-frame points. Called by the thread that wrote pair q's S.q and S.t.
__device__ __forceinline__ void store_centroid(const AdjShared &S, int q, int npts) {
    const float3 ps = make_float3(S.psum[0], S.psum[1], S.psum[2]);
    const float3 a = rotate_ref(S.q[2 * q], ps), b = rotate_ref(S.q[2 * q + 1], ps);
    const float inv = 1.0f / (float)(2 * npts), n = (float)npts;
    S.cen[3 * q] = fmaf(n, S.t[3 * q], a.x + b.x) * inv;
    S.cen[3 * q + 1] = fmaf(n, S.t[3 * q + 1], a.y + b.y) * inv;
    S.cen[3 * q + 2] = fmaf(n, S.t[3 * q + 2], a.z + b.z) * inv;
}

// Centred cloud points of the tile's pairs into S.R: row q holds body i's
// points R_i b_a - c, then body j's R_j b_a + t - c (c = S.cen). Thread
// (q, body) = (tid % kAP, tid / kAP) rotates all points of one body of one pair
// (body points broadcast from shared memory, rows of odd stride rs: no bank
// conflicts, no index divisions) with the matrix of q v q* for q = (w, u),
// (w^2 - |u|^2) I + 2 u u^T + 2 w [u]x, built once: 9 FMAs per point.
__device__ __forceinline__ void rotate_tile(const AdjShared &S, int npts, int rs) {
    static_assert(kAThreads == 2 * kAP, "one thread per (pair, body)");
    const int q = threadIdx.x & (kAP - 1), body = threadIdx.x / kAP;
    const float4 qq = S.q[2 * q + body];
    const float w = qq.x, x = qq.y, y = qq.z, z = qq.w;
    const float a0 = w * w - (x * x + y * y + z * z);
    const float m00 = fmaf(2.f * x, x, a0), m01 = 2.f * (x * y - w * z), m02 = 2.f * (x * z + w * y);
    const float m10 = 2.f * (x * y + w * z), m11 = fmaf(2.f * y, y, a0), m12 = 2.f * (y * z - w * x);
    const float m20 = 2.f * (x * z - w * y), m21 = 2.f * (y * z + w * x), m22 = fmaf(2.f * z, z, a0);
    const float ox = body ? S.t[3 * q] - S.cen[3 * q] : -S.cen[3 * q];
    const float oy = body ? S.t[3 * q + 1] - S.cen[3 * q + 1] : -S.cen[3 * q + 1];
    const float oz = body ? S.t[3 * q + 2] - S.cen[3 * q + 2] : -S.cen[3 * q + 2];
    float *dst = S.R + q * rs + body * 3 * npts;
    for (int a = 0; a < npts; ++a) {
        const float px = S.pts[3 * a], py = S.pts[3 * a + 1], pz = S.pts[3 * a + 2];
        dst[3 * a] = fmaf(m00, px, fmaf(m01, py, fmaf(m02, pz, ox)));
        dst[3 * a + 1] = fmaf(m10, px, fmaf(m11, py, fmaf(m12, pz, oy)));
        dst[3 * a + 2] = fmaf(m20, px, fmaf(m21, py, fmaf(m22, pz, oz)));
    }
}

// Torque sums about the body origins from those about the centroid:
// sum_{a in i} (r_a + c) x G_a = Xi + c x Si and
// sum_{a in j} (r_a + c - t) x G_a = Xj + (c - t) x (Sa - Si).
__device__ __forceinline__ void add_centroid_terms(const AdjShared &S, int q, const float *Si, const float *Sa,
                                                   float *Xi, float *Xj) {
    const float c[3] = {S.cen[3 * q], S.cen[3 * q + 1], S.cen[3 * q + 2]};
    const float e[3] = {c[0] - S.t[3 * q], c[1] - S.t[3 * q + 1], c[2] - S.t[3 * q + 2]};
    const float Sj[3] = {Sa[0] - Si[0], Sa[1] - Si[1], Sa[2] - Si[2]};
    Xi[0] += c[1] * Si[2] - c[2] * Si[1];
    Xi[1] += c[2] * Si[0] - c[0] * Si[2];
    Xi[2] += c[0] * Si[1] - c[1] * Si[0];
    Xj[0] += e[1] * Sj[2] - e[2] * Sj[1];
    Xj[1] += e[2] * Sj[0] - e[0] * Sj[2];
    Xj[2] += e[0] * Sj[1] - e[1] * Sj[0];
}

// MULTI: the pairs come from many systems in one launch; body i's system is
// rep[i], its box rp[rep[i]].box, and the pair energies are summed per system
// into pe[rep[i]].
template <class Cfg, bool MULTI>
__global__ void __launch_bounds__(kAThreads, 1) k_forces_adjoint(const float *pos, const float *quat, float L,
                                                                const int *pairs, const long long *d_np, long long cap,
                                                                const float *pts, int npts, float inv_rc, float en_min,
                                                                float en_range, AdjNet net, const float *w, float *F,
                                                                float *T, double *pe, const int *rep,
                                                                const amlp_replica *rp, int keep_r) {
    constexpr int KC = Half<Cfg>::KC;
    constexpr int DP = kGS;  // row stride of the fp32 descriptor staging
    extern __shared__ __align__(128) char smem_raw[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ double pe_s[kAThreads / 32];
    __shared__ float psum_s[3];

    const int tid = threadIdx.x, p = tid & (kAP - 1), h = tid >> 7, warp = tid >> 5, lane = tid & 31;
    const int rs = 6 * npts + 1 - ((6 * npts) & 1);
    const int Kg = net.kin[0];
    const int first_limit = g_amlp_first_wait_limit;

    // ---- shared memory carve-up (offsets are multiples of 128 bytes)
    AdjShared S;
    size_t off = 0;
    // Two layouts. keep_r: the rotated points R have their own area and the
    // descriptor partials g0, g1 live in the two operand tiles (free whenever
    // the partials are), so R survives the net and is rotated once per tile.
    // Otherwise (when that does not fit) R shares its area with the operand
    // tiles and is rotated again after the net.
    const size_t r_bytes = (size_t)kAP * rs * 4, ops_bytes = (size_t)2 * 2 * kAP * kWpad * 2;
    if (keep_r) {
        S.R = reinterpret_cast<float *>(smem_raw);
        off = align_up(r_bytes, 128);
        S.ops = smem_raw + off;
        off += align_up(ops_bytes, 128);
    } else {
        S.ops = smem_raw;
        S.R = reinterpret_cast<float *>(smem_raw);
        off = align_up(r_bytes > ops_bytes ? r_bytes : ops_bytes, 128);
    }
    S.wts = smem_raw + off;
    off += align_up(net.wsm_total, 128);
    S.par = reinterpret_cast<float *>(smem_raw + off);
    off += align_up((size_t)net.par_total * 4, 128);
    if (keep_r) {
        S.g0 = reinterpret_cast<float *>(op_tile(S.ops, 0));
        S.g1 = reinterpret_cast<float *>(op_tile(S.ops, 1));
    } else {
        S.g0 = reinterpret_cast<float *>(smem_raw + off);
        off += (size_t)kAP * DP * 4;
        S.g1 = reinterpret_cast<float *>(smem_raw + off);
        off += (size_t)kAP * DP * 4;
    }
    S.t = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 3 * 4;
    S.cen = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 3 * 4;
    S.part = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)2 * kAP * kPartStride * 4;
    S.eps = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)2 * kAP * 4;
    S.fd = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 9 * 4;
    S.ij = reinterpret_cast<int *>(smem_raw + off);
    off += (size_t)kAP * 2 * 4;
    S.pts = reinterpret_cast<float *>(smem_raw + off);
    off = align_up(off + (size_t)3 * npts * 4, 16);
    S.q = reinterpret_cast<float4 *>(smem_raw + off);
    S.psum = psum_s;

    // ---- one-time set-up: weights (bf16 hi/lo, K-major), biases, TMEM, mbarrier
    for (int k = tid; k < 3 * npts; k += kAThreads) S.pts[k] = pts[k];
    __syncthreads();
    body_point_sum(S, npts);
    for (int L2 = 0; L2 < net.nh; ++L2) {
        const int K = net.dims[L2], N = net.dims[L2 + 1], Kp = net.kin[L2], Np = net.nout[L2];
        const float *W = w + net.woff[L2];
        char *hi = S.wts + net.wsm_off[L2];
        char *lo = hi + Np * Kp * 2;
        for (int idx = tid; idx < Np * Kp; idx += kAThreads) {
            int n = idx / Kp, k = idx - n * Kp;
            float v = (n < N && k < K) ? W[(size_t)n * K + k] : 0.f;
            __nv_bfloat16 a, b;
            tc::split_bf16(v, a, b);
            uint32_t o = tc::kmajor_offset(n, k, Kp);
            *reinterpret_cast<__nv_bfloat16 *>(hi + o) = a;
            *reinterpret_cast<__nv_bfloat16 *>(lo + o) = b;
        }
        const float *b = W + (size_t)N * K;
        for (int n = tid; n < Np; n += kAThreads) S.par[net.bias_off[L2] + n] = n < N ? b[n] : 0.f;
    }
    {
        const int K = net.dims[net.nh];
        const float *Wl = w + net.woff[net.nh];
        for (int k = tid; k < kWpad; k += kAThreads) S.par[net.bias_off[net.nh] + k] = k < K ? Wl[k] : 0.f;
        if (tid == 0) S.par[net.bias_off[net.nh] + kWpad] = Wl[K];  // last bias
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, 512);
    if (tid == 0) tc::mbar_init(&mbar, 1);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t bar = tc::smem_u32(&mbar);
    uint32_t phase = 0;
    // A bounded wait that gives up sets gave_up in its thread; the barrier that
    // ends each net stage ORs it over the block into `aborted`, so that every
    // thread agrees on it: no further MMA is issued or waited for, the tile loop
    // ends, and the MMA still in flight is drained before TMEM is released.
    bool gave_up = false, aborted = false;
    int waits = 0, commits = 0;
    // TMEM column regions: Z_k (hidden layer k) at 64k, backward product at 192, dE/dg at 192 too,
    // act'(Z_k) of the hidden layers before the last at 256 + 64k
    auto zcol = [&](int k) { return (uint32_t)(k * kWpad); };
    const uint32_t bcol = (uint32_t)(3 * kWpad);
    auto dfcol = [&](int k) { return (uint32_t)(4 * kWpad + k * kWpad); };
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;

    auto wait_mma = [&]() {
        if (aborted) return;  // nothing was issued
        const int limit = (waits++ == 0 && first_limit >= 0) ? first_limit : tc::kWaitLimit;
        if (!tc::mbar_wait(bar, phase, limit)) gave_up = true;
        phase ^= 1u;
        tc::fence_after();
    };

    const long long P = min(*d_np, cap);
    const long long ntiles = (P + kAP - 1) / kAP;
    double pe_acc = 0.0;
    const int nd = 2 * npts;

    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long p0 = tile * kAP;
        const int valid = (int)min((long long)kAP, P - p0);
        // ---- 1. pair indices, orientations, translations, then the rotated body points
        if (tid < kAP) {
            long long pr = min(p0 + tid, P - 1);
            int i = pairs[2 * pr], j = pairs[2 * pr + 1];
            S.q[2 * tid] = load_quat(quat, i);
            S.q[2 * tid + 1] = load_quat(quat, j);
            float dd;
            float3 tt = min_image(pos, i, j, MULTI ? rp[rep[i]].box : L, &dd);
            S.t[3 * tid] = tt.x;
            S.t[3 * tid + 1] = tt.y;
            S.t[3 * tid + 2] = tt.z;
            S.ij[2 * tid] = i;
            S.ij[2 * tid + 1] = j;
            store_centroid(S, tid, npts);
        }
        __syncthreads();
        rotate_tile(S, npts, rs);
        __syncthreads();
        // ---- 2. descriptor forward
        const float *Rp = S.R + p * rs;  // the pair's centred points
        float A[Cfg::NA][KC];  // this half's sum_a f_n Y_k, kept in registers for the backward
        if (h == 0) half_forward<Cfg, 0>(Rp, nd, inv_rc, S.g0 + p * DP, A);
        else half_forward<Cfg, 1>(Rp, nd, inv_rc, S.g1 + p * DP, A);
        __syncthreads();
        // ---- 3. net forward + backward on the tensor cores
        {
            char *tG = op_tile(S.ops, 0);
            // this thread's half of its row of g (kin[0] = 48 columns, set by the
            // launcher, 24 per half), read completely before the tile is written:
            // with keep_r, g0 and g1 occupy the operand tiles
            float v[24];
#pragma unroll
            for (int k = 0; k < 24; ++k) {
                int d = h * 24 + k;
                v[k] = d < Cfg::D ? S.g0[p * DP + d] + S.g1[p * DP + d] : 0.f;
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < 3; ++c) store_split8(tG, Kg, p, h * 24 + 8 * c, v + 8 * c);
        }
        tc::fence_async_smem();
        __syncthreads();
        // forward layers
        for (int L2 = 0; L2 < net.nh; ++L2) {
            const int Kp = net.kin[L2], Np = net.nout[L2];
            if (tid == 0 && !aborted) {
                tc::fence_after();
                const char *wb = S.wts + net.wsm_off[L2];
                mma3<true>(tmem + zcol(L2), op_tile(S.ops, L2), Kp, wb, (size_t)Np * Kp * 2, Np, false, 256, 128,
                     (uint32_t)Kp * 16);
                tc::commit(bar);
                ++commits;
            }
            wait_mma();
            // epilogue: a = act(z + b) into the next operand tile; the last hidden
            // layer also forms e and delta = w_last * act'(z)
            const bool last = L2 == net.nh - 1;
            const float *bias = S.par + net.bias_off[L2];
            const float *wl = S.par + net.bias_off[net.nh];
            char *dst = op_tile(S.ops, L2 + 1);
            float esum = 0.f;
            // this thread's Np / 2 columns from cb: nch chunks of 8, two per TMEM wait
            const int cb = h * (Np / 2), nch = Np / 16;
            for (int g = 0; g < nch; g += 2) {
                float z[2 * 8];
                tc::tmem_ld8_many<2>(tmem + lane_base + zcol(L2) + cb + 8 * g, min(2, nch - g), z);
#pragma unroll
                for (int ch = 0; ch < 2; ++ch) {
                    if (g + ch < nch) {
                        const int c0 = cb + 8 * (g + ch);
                        float v[8], dv[8], bb[8], ww[8];
                        // bias_off is a multiple of 16 floats and c0 of 8: 16-byte loads
                        *reinterpret_cast<float4 *>(bb) = *reinterpret_cast<const float4 *>(bias + c0);
                        *reinterpret_cast<float4 *>(bb + 4) = *reinterpret_cast<const float4 *>(bias + c0 + 4);
                        if (last) {
                            *reinterpret_cast<float4 *>(ww) = *reinterpret_cast<const float4 *>(wl + c0);
                            *reinterpret_cast<float4 *>(ww + 4) = *reinterpret_cast<const float4 *>(wl + c0 + 4);
                        }
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            float zz = z[8 * ch + k] + bb[k], fz, dfz;
                            act_pair(net.act, zz, fz, dfz);
                            if (last) {
                                esum = fmaf(ww[k], fz, esum);
                                v[k] = ww[k] * dfz;
                            } else {
                                v[k] = fz;
                                dv[k] = dfz;
                            }
                        }
                        store_split8(dst, Np, p, c0, v);
                        if (!last) tc::tmem_st8(tmem + lane_base + dfcol(L2) + c0, dv);  // for the backward
                    }
                }
            }
            if (last) S.eps[h * kAP + p] = esum;
            else tc::tmem_wait_st();
            tc::fence_before();
            tc::fence_async_smem();
            aborted = __syncthreads_or(gave_up) != 0;
        }
        // backward layers: delta_{k-1} = (delta_k W_k) * act'(z_{k-1}); dE/dg = delta_1 W_1
        for (int L2 = net.nh - 1; L2 >= 0; --L2) {
            const int Kp = net.kin[L2], Np = net.nout[L2];
            if (tid == 0 && !aborted) {
                tc::fence_after();
                const char *wb = S.wts + net.wsm_off[L2];
                // B = W_k read as MN-major (the transpose): N' = Kp, K' = Np
                mma3<true>(tmem + bcol, op_tile(S.ops, L2 + 1), Np, wb, (size_t)Np * Kp * 2, Kp, true,
                     2 * Kp * 16, (uint32_t)Kp * 16, 128);
                tc::commit(bar);
                ++commits;
            }
            wait_mma();
            if (L2 > 0) {
                char *dst = op_tile(S.ops, L2);
                const int cb = h * (Kp / 2), nch = Kp / 16;
                for (int ch = 0; ch < nch; ++ch) {  // a chunk of dz and of act'(z) per TMEM wait
                    const int c0 = cb + 8 * ch;
                    uint32_t r[16];
                    float x[16];
                    tc::tmem_ld8_issue(tmem + lane_base + bcol + c0, r);
                    tc::tmem_ld8_issue(tmem + lane_base + dfcol(L2 - 1) + c0, r + 8);
                    tc::tmem_wait_ld<16>(r, x);
                    float v[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[k] = x[k] * x[8 + k];
                    store_split8(dst, Kp, p, c0, v);
                }
                tc::fence_async_smem();
            } else {
                const int cb = h * (Kp / 2), nch = Kp / 16;
                for (int g = 0; g < nch; g += 2) {
                    float dg[2 * 8];
                    tc::tmem_ld8_many<2>(tmem + lane_base + bcol + cb + 8 * g, min(2, nch - g), dg);
#pragma unroll
                    for (int ch = 0; ch < 2; ++ch)
                        if (g + ch < nch)
#pragma unroll
                            for (int k = 0; k < 8; ++k) S.g0[p * DP + cb + 8 * (g + ch) + k] = dg[8 * ch + k];
                }
            }
            tc::fence_before();
            aborted = __syncthreads_or(gave_up) != 0;
        }
        if (aborted) break;  // the net's outputs are not to be trusted: no forces from this tile
        if (!MULTI && h == 0 && p < valid)
            pe_acc += (double)en_min +
                      (double)en_range * (double)(S.eps[p] + S.eps[kAP + p] + S.par[net.bias_off[net.nh] + kWpad]);
        // ---- 4. recompute the rotated points (their area held the MLP tiles)
        if (!keep_r) {
            rotate_tile(S, npts, rs);
            __syncthreads();
        }
        // ---- descriptor backward
        if (h == 0) half_backward<Cfg, 0>(Rp, npts, inv_rc, S.g0 + p * DP, S.part + p * kPartStride, A);
        else half_backward<Cfg, 1>(Rp, npts, inv_rc, S.g0 + p * DP, S.part + (kAP + p) * kPartStride, A);
        __syncthreads();
        // ---- 5. per-pair forces and torques
        if (tid < kAP) {
            const float *a0 = S.part + p * kPartStride, *a1 = S.part + (kAP + p) * kPartStride;
            float Si[3], Sa[3], Xi[3], Xj[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                Si[k] = a0[k] + a1[k];
                Sa[k] = a0[3 + k] + a1[3 + k];
                Xi[k] = a0[6 + k] + a1[6 + k];
                Xj[k] = a0[9 + k] + a1[9 + k];
            }
            add_centroid_terms(S, p, Si, Sa, Xi, Xj);
            // sums of the rotated points of i and of j: the rotation of the point sum
            const float3 ps = make_float3(S.psum[0], S.psum[1], S.psum[2]);
            const float3 pi3 = rotate_ref(S.q[2 * p], ps), qj3 = rotate_ref(S.q[2 * p + 1], ps);
            const float Pi[3] = {pi3.x, pi3.y, pi3.z}, Qj[3] = {qj3.x, qj3.y, qj3.z};
            const float inv_nd = 1.0f / (float)nd;
            float Gm[3] = {Sa[0] * inv_nd, Sa[1] * inv_nd, Sa[2] * inv_nd};  // mean gradient
            float Fp[3], Ti[3], Tj[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) Fp[k] = -(Si[k] - (float)npts * Gm[k]);
            Ti[0] = -(Xi[0] - (Pi[1] * Gm[2] - Pi[2] * Gm[1]));
            Ti[1] = -(Xi[1] - (Pi[2] * Gm[0] - Pi[0] * Gm[2]));
            Ti[2] = -(Xi[2] - (Pi[0] * Gm[1] - Pi[1] * Gm[0]));
            Tj[0] = -(Xj[0] - (Qj[1] * Gm[2] - Qj[2] * Gm[1]));
            Tj[1] = -(Xj[1] - (Qj[2] * Gm[0] - Qj[0] * Gm[2]));
            Tj[2] = -(Xj[2] - (Qj[0] * Gm[1] - Qj[1] * Gm[0]));
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                S.fd[9 * p + k] = clip100(Fp[k] * en_range);
                S.fd[9 * p + 3 + k] = clip100(Ti[k] * en_range);
                S.fd[9 * p + 6 + k] = clip100(Tj[k] * en_range);
            }
        }
        __syncthreads();
        // ---- scatter: warps 0..3, lane = pair within a 32-pair group
        if (warp < 4) {
            const int q = warp * 32 + lane;
            const bool ok = q < valid;
            const int i = S.ij[2 * q], j = S.ij[2 * q + 1];
            float v[6];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                v[k] = ok ? S.fd[9 * q + k] : 0.f;
                v[3 + k] = ok ? S.fd[9 * q + 3 + k] : 0.f;
            }
            if (ok) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    atomicAdd(F + 3 * j + k, -v[k]);
                    atomicAdd(T + 3 * j + k, S.fd[9 * q + 6 + k]);
                }
            }
            const bool runs = warp_keys_sorted(i, ok);  // every lane takes part (warp vote)
            int key = ok && runs ? i : -1 - q;  // unsorted pairs: no merging
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int ko = __shfl_up_sync(0xffffffffu, key, o);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    float y = __shfl_up_sync(0xffffffffu, v[k], o);
                    if (lane >= o && ko == key) v[k] += y;
                }
            }
            int kn = __shfl_down_sync(0xffffffffu, key, 1);
            if (ok && (lane == 31 || kn != key)) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    atomicAdd(F + 3 * i + k, v[k]);
                    atomicAdd(T + 3 * i + k, v[3 + k]);
                }
            }
            if (MULTI && pe) {  // pair energies summed per system (systems own contiguous bodies)
                double e = ok ? (double)en_min + (double)en_range *
                                    (double)(S.eps[q] + S.eps[kAP + q] + S.par[net.bias_off[net.nh] + kWpad])
                              : 0.0;
                const int sys = ok ? rep[i] : 0;
                const bool sys_runs = warp_keys_sorted(sys, ok);
                int rk = ok && sys_runs ? sys : -1 - lane;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int ro = __shfl_up_sync(0xffffffffu, rk, o);
                    double y = __shfl_up_sync(0xffffffffu, e, o);
                    if (lane >= o && ro == rk) e += y;
                }
                int rn = __shfl_down_sync(0xffffffffu, rk, 1);
                if (ok && (lane == 31 || rn != rk)) atomicAdd(pe + sys, e);
            }
        }
        __syncthreads();
    }
    // ---- pair-energy sum, TMEM release
    if (!MULTI && pe) {
        double v = pe_acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) pe_s[warp] = v;
    }
    tc::fence_before();
    __syncthreads();
    if (!MULTI && pe && tid == 0) {
        double s = 0.0;
        for (int k = 0; k < kAThreads / 32; ++k) s += pe_s[k];
        if (s != 0.0) atomicAdd(pe, s);
    }
    if (aborted && tid == 0) {
        atomicOr(&g_amlp_device_error, kErrMbarTimeout);
        // the last MMA issued may still be in flight (thread 0 flipped `phase` after waiting for it):
        // let it finish, with the normal limit, before TMEM is released
        if (commits > 0) tc::mbar_wait(bar, phase ^ 1u, tc::kWaitLimit);
    }
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

// ============================================================================
// Wide nets (hidden widths up to 128): three kernels instead of one, since the
// descriptor state and the resident weights of a 128-wide net do not share one
// CTA's shared memory. g, dE/dg and the net output go through a caller
// workspace:
//   k_adj_desc<..., false>  descriptor forward per pair -> g (P x 48 fp32);
//   k_mlp_grad              net forward + backward on the tensor cores per row,
//                           weights staged layer by layer -> y and dE/dg;
//   k_adj_desc<..., true>   recomputes the per-pair sums, descriptor backward,
//                           forces, torques, scatter.
// ============================================================================
constexpr int kWideMax = 160;  // hidden widths up to 150 (the reference's nets), padded to 160
constexpr int kGP = 48;  // padded descriptor width in the workspace rows
// Row stride of the descriptor rows in the workspace and in k_mlp_grad's shared
// copy: 52 floats, 13 units of 16 bytes, odd, so that the 16-byte reads of 32
// consecutive rows by a warp fall in distinct bank groups.
constexpr int kGRow = 52;
// The same for the hypers (10, 10, 10), D = 121: padded to 128, rows of 132 floats (33 x 16 bytes)
constexpr int kGP2 = 128;
constexpr int kGRow2 = 132;
constexpr size_t kWeightSplitBytes = (size_t)kMaxHiddenWide * kWideMax * kWideMax * 4;  // bf16 hi/lo, every layer
constexpr size_t kAdjAFloats = 2 * 9 * 12;  // harmonic sums per pair kept between the passes (two halves of 9 x 12)

__host__ __device__ inline size_t adj_a_bytes(long long cap) {
    return (size_t)((cap + 127) / 128) * 128 * kAdjAFloats * 4;
}

// Per-pair force/torque from the two halves' partial sums, scaled, clipped
// (unless clip == 0), then scattered with runs of equal i summed in the warp
// (warps 0..3, lane = pair).
template <bool MULTI>
__device__ __forceinline__ void adj_finish_tile(const AdjShared &S, int rs, int npts, int valid, float en_min,
                                                float en_range, const float *y_rows, long long p0, float *F, float *T,
                                                double *pe, const int *rep, double &pe_acc, int clip) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nd = 2 * npts;
    if (tid < kAP) {
        const int p = tid;
        const float *a0 = S.part + p * kPartStride, *a1 = S.part + (kAP + p) * kPartStride;
        float Si[3], Sa[3], Xi[3], Xj[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Si[k] = a0[k] + a1[k];
            Sa[k] = a0[3 + k] + a1[3 + k];
            Xi[k] = a0[6 + k] + a1[6 + k];
            Xj[k] = a0[9 + k] + a1[9 + k];
        }
        add_centroid_terms(S, p, Si, Sa, Xi, Xj);
        const float3 ps = make_float3(S.psum[0], S.psum[1], S.psum[2]);
        const float3 pi3 = rotate_ref(S.q[2 * p], ps), qj3 = rotate_ref(S.q[2 * p + 1], ps);
        const float Pi[3] = {pi3.x, pi3.y, pi3.z}, Qj[3] = {qj3.x, qj3.y, qj3.z};
        const float inv_nd = 1.0f / (float)nd;
        float Gm[3] = {Sa[0] * inv_nd, Sa[1] * inv_nd, Sa[2] * inv_nd};
        float Fp[3], Ti[3], Tj[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) Fp[k] = -(Si[k] - (float)npts * Gm[k]);
        Ti[0] = -(Xi[0] - (Pi[1] * Gm[2] - Pi[2] * Gm[1]));
        Ti[1] = -(Xi[1] - (Pi[2] * Gm[0] - Pi[0] * Gm[2]));
        Ti[2] = -(Xi[2] - (Pi[0] * Gm[1] - Pi[1] * Gm[0]));
        Tj[0] = -(Xj[0] - (Qj[1] * Gm[2] - Qj[2] * Gm[1]));
        Tj[1] = -(Xj[1] - (Qj[2] * Gm[0] - Qj[0] * Gm[2]));
        Tj[2] = -(Xj[2] - (Qj[0] * Gm[1] - Qj[1] * Gm[0]));
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float f = Fp[k] * en_range, ti = Ti[k] * en_range, tj = Tj[k] * en_range;
            S.fd[9 * p + k] = clip ? clip100(f) : f;
            S.fd[9 * p + 3 + k] = clip ? clip100(ti) : ti;
            S.fd[9 * p + 6 + k] = clip ? clip100(tj) : tj;
        }
        if (!MULTI && p < valid) pe_acc += (double)en_min + (double)en_range * (double)y_rows[p0 + p];
    }
    __syncthreads();
    if (warp < 4) {
        const int q = warp * 32 + lane;
        const bool ok = q < valid;
        const int i = S.ij[2 * q], j = S.ij[2 * q + 1];
        float v[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = ok ? S.fd[9 * q + k] : 0.f;
            v[3 + k] = ok ? S.fd[9 * q + 3 + k] : 0.f;
        }
        if (ok) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                atomicAdd(F + 3 * j + k, -v[k]);
                atomicAdd(T + 3 * j + k, S.fd[9 * q + 6 + k]);
            }
        }
        const bool runs = warp_keys_sorted(i, ok);  // every lane takes part (warp vote)
        int key = ok && runs ? i : -1 - q;  // unsorted pairs: no merging
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int ko = __shfl_up_sync(0xffffffffu, key, o);
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                float yv = __shfl_up_sync(0xffffffffu, v[k], o);
                if (lane >= o && ko == key) v[k] += yv;
            }
        }
        int kn = __shfl_down_sync(0xffffffffu, key, 1);
        if (ok && (lane == 31 || kn != key)) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                atomicAdd(F + 3 * i + k, v[k]);
                atomicAdd(T + 3 * i + k, v[3 + k]);
            }
        }
        if (MULTI && pe) {
            double e = ok ? (double)en_min + (double)en_range * (double)y_rows[p0 + q] : 0.0;
            const int sys = ok ? rep[i] : 0;
            const bool sys_runs = warp_keys_sorted(sys, ok);
            int rk = ok && sys_runs ? sys : -1 - lane;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int ro = __shfl_up_sync(0xffffffffu, rk, o);
                double yv = __shfl_up_sync(0xffffffffu, e, o);
                if (lane >= o && ro == rk) e += yv;
            }
            int rn = __shfl_down_sync(0xffffffffu, rk, 1);
            if (ok && (lane == 31 || rn != rk)) atomicAdd(pe + sys, e);
        }
    }
    __syncthreads();
}

// dE/dg rows of the tile's pairs into S.g0 (row stride kGS), weighted by wt
// when given; rows past `valid` are zero. One row per warp, lanes over columns.
__device__ __forceinline__ void load_dg_rows(const AdjShared &S, const float *dg_rows, const float *wt, long long p0,
                                             int valid) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = warp; q < kAP; q += kAThreads / 32) {
        const float w = q < valid ? (wt ? wt[p0 + q] : 1.0f) : 0.f;
        for (int d = lane; d < kGP; d += 32) S.g0[q * kGS + d] = q < valid ? w * dg_rows[(p0 + q) * kGP + d] : 0.f;
    }
}

// Descriptor pass of the wide path: BWD = false writes g rows (row stride
// g_ld >= D, zero padded); BWD = true reads dE/dg rows (stride kGP) and the net
// outputs and produces forces, torques and energies. wt (BWD, may be null)
// weights pair p's dE/dg by wt[p] (a vector-Jacobian product); clip = 0 turns
// the +-100 clip of the per-pair forces and torques off.
template <class Cfg, bool MULTI, bool BWD>
__global__ void __launch_bounds__(kAThreads, 1) k_adj_desc(const float *pos, const float *quat, float L,
                                                          const int *pairs, const long long *d_np, long long cap,
                                                          const float *pts, int npts, float inv_rc, float en_min,
                                                          float en_range, float *g_rows, int g_ld,
                                                          const float *dg_rows, const float *y_rows, const float *wt,
                                                          int clip, float *F, float *T, double *pe, const int *rep,
                                                          const amlp_replica *rp, float *a_rows) {
    constexpr int KC = Half<Cfg>::KC;
    static_assert(2 * Cfg::NA * KC == kAdjAFloats, "harmonic sums per pair in the workspace");
    extern __shared__ __align__(128) char smem_raw[];
    __shared__ double pe_s[kAThreads / 32];
    __shared__ float psum_s[3];
    const int tid = threadIdx.x, p = tid & (kAP - 1), h = tid >> 7, warp = tid >> 5, lane = tid & 31;
    const int rs = 6 * npts + 1 - ((6 * npts) & 1);
    const int nd = 2 * npts;
    AdjShared S;
    S.psum = psum_s;
    size_t off = 0;
    S.R = reinterpret_cast<float *>(smem_raw);
    off = align_up((size_t)kAP * rs * 4, 128);
    S.g0 = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * kGS * 4;
    S.g1 = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * kGS * 4;
    S.t = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 3 * 4;
    S.cen = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 3 * 4;
    S.part = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)2 * kAP * kPartStride * 4;
    S.fd = reinterpret_cast<float *>(smem_raw + off);
    off += (size_t)kAP * 9 * 4;
    S.ij = reinterpret_cast<int *>(smem_raw + off);
    off += (size_t)kAP * 2 * 4;
    S.pts = reinterpret_cast<float *>(smem_raw + off);
    off = align_up(off + (size_t)3 * npts * 4, 16);
    S.q = reinterpret_cast<float4 *>(smem_raw + off);
    for (int k = tid; k < 3 * npts; k += kAThreads) S.pts[k] = pts[k];
    __syncthreads();
    body_point_sum(S, npts);
    __syncthreads();
    const long long P = min(*d_np, cap);
    const long long ntiles = (P + kAP - 1) / kAP;
    double pe_acc = 0.0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long p0 = tile * kAP;
        const int valid = (int)min((long long)kAP, P - p0);
        // this thread's harmonic sums: computed by the forward pass (and stored
        // for the backward pass when a_rows is given), read back by the backward
        // pass; layout [tile][half][n][kk][pair] so that a warp's accesses coalesce
        float A[Cfg::NA][KC];
        float *a_tile = a_rows ? a_rows + ((size_t)tile * 2 + h) * (Cfg::NA * KC) * kAP + p : nullptr;
        if (BWD && a_rows && tid == 0 && tile + gridDim.x < ntiles) {
            // the next tile's harmonic sums and dE/dg rows into L2 while this tile runs
            const long long nt = tile + gridDim.x;
            const char *an = reinterpret_cast<const char *>(a_rows + (size_t)nt * 2 * (Cfg::NA * KC) * kAP);
            constexpr uint32_t kABytes = 2u * Cfg::NA * KC * kAP * 4u, kPiece = 16384u;
            for (uint32_t o = 0; o < kABytes; o += kPiece) tc::bulk_prefetch_l2(an + o, min(kPiece, kABytes - o));
            const uint32_t gb = (uint32_t)(min((long long)kAP, P - nt * kAP) * kGP * 4);
            tc::bulk_prefetch_l2(dg_rows + nt * kAP * kGP, gb);
        }
        if (BWD && a_rows) {
            // the backward's inputs first, so that their loads overlap the rotation pass
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
                for (int kk = 0; kk < KC; ++kk) A[n][kk] = a_tile[(n * KC + kk) * kAP];
            load_dg_rows(S, dg_rows, wt, p0, valid);
        }
        if (tid < kAP) {
            long long pr = min(p0 + tid, P - 1);
            int i = pairs[2 * pr], j = pairs[2 * pr + 1];
            S.q[2 * tid] = load_quat(quat, i);
            S.q[2 * tid + 1] = load_quat(quat, j);
            float dd;
            float3 tt = min_image(pos, i, j, MULTI ? rp[rep[i]].box : L, &dd);
            S.t[3 * tid] = tt.x;
            S.t[3 * tid + 1] = tt.y;
            S.t[3 * tid + 2] = tt.z;
            S.ij[2 * tid] = i;
            S.ij[2 * tid + 1] = j;
            store_centroid(S, tid, npts);
        }
        __syncthreads();
        rotate_tile(S, npts, rs);
        __syncthreads();
        const float *Rp = S.R + p * rs;  // the pair's centred points
        if (!BWD || !a_rows) {
            if (h == 0) half_forward<Cfg, 0>(Rp, nd, inv_rc, S.g0 + p * kGS, A);
            else half_forward<Cfg, 1>(Rp, nd, inv_rc, S.g1 + p * kGS, A);
            if (!BWD && a_tile) {
#pragma unroll
                for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) a_tile[(n * KC + kk) * kAP] = A[n][kk];
            }
        }
        __syncthreads();
        if (!BWD) {
            for (int q = warp; q < valid; q += kAThreads / 32)  // one row per warp: coalesced
                for (int d = lane; d < g_ld; d += 32)
                    g_rows[(p0 + q) * g_ld + d] = d < Cfg::D ? S.g0[q * kGS + d] + S.g1[q * kGS + d] : 0.f;
            __syncthreads();
            continue;
        }
        if (!a_rows) {  // the forward partials held S.g0 until now
            load_dg_rows(S, dg_rows, wt, p0, valid);
        }
        __syncthreads();
        if (h == 0) half_backward<Cfg, 0>(Rp, npts, inv_rc, S.g0 + p * kGS, S.part + p * kPartStride, A);
        else half_backward<Cfg, 1>(Rp, npts, inv_rc, S.g0 + p * kGS, S.part + (kAP + p) * kPartStride, A);
        __syncthreads();
        adj_finish_tile<MULTI>(S, rs, npts, valid, en_min, en_range, y_rows, p0, F, T, pe, rep, pe_acc, clip);
    }
    if (BWD && !MULTI && pe) {
        double v = pe_acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) pe_s[warp] = v;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int k = 0; k < kAThreads / 32; ++k) s += pe_s[k];
            if (s != 0.0) atomicAdd(pe, s);
        }
    }
}

// The hidden layers' weights split into bf16 hi/lo once per launch, in the
// K-major layout of the shared-memory operand (per layer: hi, then lo), so that
// k_mlp_grad loads a layer with one bulk copy.
__global__ void k_split_weights(AdjNet net, const float *w, char *dst) {
    for (int L2 = 0; L2 < net.nh; ++L2) {
        const int K = net.dims[L2], N = net.dims[L2 + 1], Kp = net.kin[L2], Np = net.nout[L2];
        const float *W = w + net.woff[L2];
        char *hi = dst + net.wsm_off[L2], *lo = hi + (size_t)Np * Kp * 2;
        for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < Np * Kp; idx += gridDim.x * blockDim.x) {
            int n = idx / Kp, k = idx - n * Kp;
            float v = (n < N && k < K) ? W[(size_t)n * K + k] : 0.f;
            __nv_bfloat16 a, bb;
            tc::split_bf16(v, a, bb);
            uint32_t o = tc::kmajor_offset(n, k, Kp);
            *reinterpret_cast<__nv_bfloat16 *>(hi + o) = a;
            *reinterpret_cast<__nv_bfloat16 *>(lo + o) = bb;
        }
    }
}

// Net forward and backward over rows of g on the tensor cores (bf16x3 splits,
// fp32 TMEM accumulators), hidden layers up to 160 wide and up to four of them
// (the reference's TheEnergyNet(150, 3, D): layer_first and three hidden
// layers). 16 warps: warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31 (its
// rows) and, of every layer's columns, the 8-column chunks c with
// c % 4 == w / 4, so that four warps share each epilogue's rows.
// Shared memory holds one operand tile: each epilogue overwrites the tile its
// MMA read, complete by then. One layer's weights at a time sit beside it,
// brought in by a bulk copy from the pre-split copy (k_split_weights) that
// thread 0 starts as soon as the previous layer's MMAs are done, so that it
// overlaps the epilogue; the layer order fwd 0..nh-1, bwd nh-1..0 reuses the
// last forward layer and, across tiles, layer 0. One TMEM region (net.zbw
// columns) takes every product in turn. The forward epilogues keep act'(z) of
// each hidden layer but the last for the backward: for ReLU (derivative 0 or
// 1) as bits in registers, otherwise in TMEM after the product region.
// Outputs per row: y = net(g) and dE/dg (net.gp floats).
constexpr int kMQ = 4;                  // column groups of the k_mlp_grad epilogues
constexpr int kMThreads = kMQ * kAP;    // 512
static_assert(kWideMax <= 8 * kMQ * 8, "a thread's 8-column chunks of a layer fit one 64-bit mask");
__global__ void __launch_bounds__(kMThreads, 1) k_mlp_grad(const float *g_rows, const long long *d_np, long long cap,
                                                          AdjNet net, const float *w, const char *wsplit,
                                                          float *y_rows, float *dg_rows) {
    extern __shared__ __align__(128) char smem_raw[];
    __shared__ uint64_t mbar, wbar, gbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, p = tid & (kAP - 1), h = tid >> 7, warp = tid >> 5;
    char *tile = smem_raw;  // the operand tile: bf16 hi, then lo
    char *wbuf = smem_raw + net.wbuf_off;
    float *par = reinterpret_cast<float *>(smem_raw + net.par_off);
    float *eps = reinterpret_cast<float *>(smem_raw + net.eps_off);
    float *gbuf = reinterpret_cast<float *>(smem_raw + net.gbuf_off);
    for (int L2 = 0; L2 < net.nh; ++L2) {
        const int N = net.dims[L2 + 1], Np = net.nout[L2];
        const float *b = w + net.woff[L2] + (size_t)N * net.dims[L2];
        for (int n = tid; n < Np; n += kMThreads) par[net.bias_off[L2] + n] = n < N ? b[n] : 0.f;
    }
    {
        const int K = net.dims[net.nh];
        const float *Wl = w + net.woff[net.nh];
        for (int k = tid; k < kWideMax; k += kMThreads) par[net.bias_off[net.nh] + k] = k < K ? Wl[k] : 0.f;
        if (tid == 0) par[net.bias_off[net.nh] + kWideMax] = Wl[K];
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, 512);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::mbar_init(&wbar, 1);
        tc::mbar_init(&gbar, 1);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tmem_slot, bar = tc::smem_u32(&mbar);
    uint32_t phase = 0;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    auto dfcol = [&](int k) { return (uint32_t)(net.zbw + k * net.wmax); };  // act'(z_k), smooth activations
    const bool relu = net.relu_bits != 0;
    // A bounded wait that gives up sets gave_up in its thread; the barriers that
    // end the stages OR it over the block into `aborted`: no further MMA or copy
    // is issued, the tile loop ends and what is in flight is drained at the end.
    bool gave_up = false, aborted = false;
    int commits = 0;
    auto wait_mma = [&]() {
        if (aborted) return;  // nothing was issued
        if (!tc::mbar_wait(bar, phase)) gave_up = true;
        phase ^= 1u;
        tc::fence_after();
    };
    // weights: `in_buf` (tracked identically by every thread) is the layer whose
    // weights are in wbuf or on their way; thread 0 starts the copies and waits
    // for them before its MMAs.
    int in_buf = -1;
    bool w_pending = false;
    uint32_t wphase = 0;
    const uint32_t wb_u32 = tc::smem_u32(wbuf), wbar_u32 = tc::smem_u32(&wbar);
    auto request = [&](int L2) {
        if (L2 == in_buf) return;
        in_buf = L2;
        if (tid == 0 && !aborted && !gave_up) {
            const uint32_t bytes = (uint32_t)(4 * net.nout[L2] * net.kin[L2]);
            tc::mbar_arrive_expect_tx(wbar_u32, bytes);
            tc::bulk_g2s(wb_u32, wsplit + net.wsm_off[L2], bytes, wbar_u32);
            w_pending = true;
        }
    };
    auto ensure = [&]() {  // thread 0 only
        if (!w_pending) return;
        if (!tc::mbar_wait(wbar_u32, wphase)) gave_up = true;
        wphase ^= 1u;
        w_pending = false;
    };
    request(0);
    const long long P = min(*d_np, cap);
    const long long ntiles = (P + kAP - 1) / kAP;
    const int Kg = net.kin[0];
    // descriptor rows of tile tl into gbuf (thread 0; rows r0 .. r0 + valid are contiguous)
    bool g_pending = false;
    uint32_t gphase = 0;
    const uint32_t gbuf_u32 = tc::smem_u32(gbuf), gbar_u32 = tc::smem_u32(&gbar);
    auto request_g = [&](long long tl) {
        if (!net.prefetch_g || tid != 0 || aborted || gave_up || tl >= ntiles) return;
        const long long r0 = tl * kAP;
        const uint32_t bytes = (uint32_t)(min((long long)kAP, P - r0) * net.g_ld * 4);
        tc::mbar_arrive_expect_tx(gbar_u32, bytes);
        tc::bulk_g2s(gbuf_u32, g_rows + r0 * net.g_ld, bytes, gbar_u32);
        g_pending = true;
    };
    request_g(blockIdx.x);
    for (long long tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
        if (aborted) break;
        const long long r0 = tl * kAP;
        const int valid = (int)min((long long)kAP, P - r0);
        if (net.prefetch_g) {  // every thread reads gbuf
            if (!tc::mbar_wait(gbar_u32, gphase)) gave_up = true;
            gphase ^= 1u;
            if (tid == 0) g_pending = false;
        }
        for (int c0 = 8 * h; c0 < Kg; c0 += 8 * kMQ) {
            float v[8];
            const float *src = net.prefetch_g ? gbuf + p * net.g_ld + c0 : g_rows + (r0 + p) * net.g_ld + c0;
            const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 lo4 = p < valid ? reinterpret_cast<const float4 *>(src)[0] : zero4;
            const float4 hi4 = p < valid ? reinterpret_cast<const float4 *>(src)[1] : zero4;
            v[0] = lo4.x, v[1] = lo4.y, v[2] = lo4.z, v[3] = lo4.w;
            v[4] = hi4.x, v[5] = hi4.y, v[6] = hi4.z, v[7] = hi4.w;
            store_split8(tile, Kg, p, c0, v);
        }
        uint64_t m0 = 0, m1 = 0, m2 = 0;  // ReLU: act'(z) bits of hidden layers 0, 1, 2 (this thread's chunks)
        for (int L2 = 0; L2 < net.nh; ++L2) {
            const int Kp = net.kin[L2], Np = net.nout[L2];
            request(L2);
            if (L2 == 0) {  // later layers start right after the previous epilogue's barrier
                tc::fence_async_smem();
                aborted = __syncthreads_or(gave_up) != 0;
                request_g(tl + gridDim.x);  // gbuf has been read: prefetch the next tile
            }
            if (tid == 0) ensure();
            if (tid == 0 && !aborted && !gave_up) {
                tc::fence_after();
                mma3<false>(tmem, tile, Kp, wbuf, (size_t)Np * Kp * 2, Np, false, 256, 128, (uint32_t)Kp * 16);
                tc::commit(bar);
                ++commits;
            }
            wait_mma();
            if (L2 + 1 < net.nh) request(L2 + 1);  // overlaps this layer's epilogue
            const bool last = L2 == net.nh - 1;
            const float *bias = par + net.bias_off[L2];
            const float *wl = par + net.bias_off[net.nh];
            float esum = 0.f;
            uint64_t bits = 0;
            for (int j = 0, c0 = 8 * h; c0 < Np; ++j, c0 += 8 * kMQ) {
                float z[8], v[8], dv[8], bb[8], ww[8];
                tc::tmem_ld8(tmem + lane_base + c0, z);
                *reinterpret_cast<float4 *>(bb) = *reinterpret_cast<const float4 *>(bias + c0);
                *reinterpret_cast<float4 *>(bb + 4) = *reinterpret_cast<const float4 *>(bias + c0 + 4);
                if (last) {
                    *reinterpret_cast<float4 *>(ww) = *reinterpret_cast<const float4 *>(wl + c0);
                    *reinterpret_cast<float4 *>(ww + 4) = *reinterpret_cast<const float4 *>(wl + c0 + 4);
                }
                uint32_t b8 = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    float zz = z[k] + bb[k], fz, dfz;
                    act_pair(net.act, zz, fz, dfz);
                    if (last) {
                        esum = fmaf(ww[k], fz, esum);
                        v[k] = ww[k] * dfz;
                    } else {
                        v[k] = fz;
                        dv[k] = dfz;
                        b8 |= (dfz != 0.f ? 1u : 0u) << k;
                    }
                }
                if (!last) bits |= (uint64_t)b8 << (8 * j);
                store_split8(tile, Np, p, c0, v);  // the MMA that read the tile is complete
                if (!last && !relu) tc::tmem_st8(tmem + lane_base + dfcol(L2) + c0, dv);  // for the backward
            }
            if (last) {
                eps[h * kAP + p] = esum;
            } else if (relu) {
                if (L2 == 0) m0 = bits;
                else if (L2 == 1) m1 = bits;
                else m2 = bits;
            } else {
                tc::tmem_wait_st();
            }
            tc::fence_before();
            tc::fence_async_smem();
            aborted = __syncthreads_or(gave_up) != 0;
        }
        if (tid < kAP && p < valid)
        {
            float ysum = par[net.bias_off[net.nh] + kWideMax];
#pragma unroll
            for (int g = 0; g < kMQ; ++g) ysum += eps[g * kAP + p];
            y_rows[r0 + p] = ysum;
        }
        // backward: delta_{k-1} = (delta_k W_k) * act'(z_{k-1}); dE/dg = delta_0 W_0
        for (int L2 = net.nh - 1; L2 >= 0; --L2) {  // each layer starts right after the previous barrier
            const int Kp = net.kin[L2], Np = net.nout[L2];
            request(L2);
            if (tid == 0) ensure();
            if (tid == 0 && !aborted && !gave_up) {
                tc::fence_after();
                // B = W_k read as MN-major (the transpose): N' = Kp, K' = Np
                mma3<false>(tmem, tile, Np, wbuf, (size_t)Np * Kp * 2, Kp, true, 2 * Kp * 16, (uint32_t)Kp * 16, 128);
                tc::commit(bar);
                ++commits;
            }
            wait_mma();
            request(L2 > 0 ? L2 - 1 : 0);  // the next layer needed (layer 0 again for the next tile)
            if (L2 > 0) {
                const uint64_t bits = L2 == 1 ? m0 : (L2 == 2 ? m1 : m2);
                for (int j = 0, c0 = 8 * h; c0 < Kp; ++j, c0 += 8 * kMQ) {
                    float dz[8], df[8], v[8];
                    tc::tmem_ld8(tmem + lane_base + c0, dz);
                    if (relu) {
                        const uint32_t b8 = (uint32_t)(bits >> (8 * j));
#pragma unroll
                        for (int k = 0; k < 8; ++k) v[k] = (b8 >> k) & 1u ? dz[k] : 0.f;
                    } else {
                        tc::tmem_ld8(tmem + lane_base + dfcol(L2 - 1) + c0, df);
#pragma unroll
                        for (int k = 0; k < 8; ++k) v[k] = dz[k] * df[k];
                    }
                    store_split8(tile, Kp, p, c0, v);
                }
            } else {
                for (int c0 = 8 * h; c0 < Kp; c0 += 8 * kMQ) {
                    float dg[8];
                    tc::tmem_ld8(tmem + lane_base + c0, dg);
                    if (p < valid) {
                        float4 *dst = reinterpret_cast<float4 *>(dg_rows + (r0 + p) * net.gp + c0);
                        dst[0] = make_float4(dg[0], dg[1], dg[2], dg[3]);
                        dst[1] = make_float4(dg[4], dg[5], dg[6], dg[7]);
                    }
                }
            }
            tc::fence_before();
            tc::fence_async_smem();
            aborted = __syncthreads_or(gave_up) != 0;
        }
    }
    aborted = __syncthreads_or(gave_up) != 0;
    if (tid == 0) {
        bool drained = true;
        // the last MMA issued (commit number `commits`, parity (commits - 1) & 1) may still be in flight
        if (commits > 0) drained &= tc::mbar_wait(bar, (uint32_t)((commits - 1) & 1));
        if (w_pending) drained &= tc::mbar_wait(wbar_u32, wphase);  // no copy may still write shared memory
        if (g_pending) drained &= tc::mbar_wait(gbar_u32, gphase);
        if (aborted || !drained) atomicOr(&g_amlp_device_error, kErrMbarTimeout);
    }
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

}  // namespace

amlp_status check_nep(const amlp_nep *n);
int hyper_kind(const amlp_nep *n);
int nep_D(const amlp_nep *n);
amlp_status check_mlp(const amlp_mlp *m, int D);

}  // namespace amlp

using namespace amlp;

static amlp_status launch_adjoint(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                  const long long *d_npairs, long long cap, const amlp_nep *nep, const amlp_mlp *mlp,
                                  float *d_F, float *d_T, double *d_pe, const int *d_rep, const amlp_replica *d_rp,
                                  void *stream) {
    amlp_status st = check_nep(nep);
    if (st) return st;
    const int D = nep_D(nep);
    if ((st = check_mlp(mlp, D))) return st;
    if (!d_pos || !d_quat || !d_npairs || !d_F || !d_T || cap < 0 || (cap > 0 && !d_pairs)) return AMLP_ERR_INVALID_ARG;
    if (cap == 0) return AMLP_OK;
    if (hyper_kind(nep) != 1 || D > 48) return AMLP_ERR_UNSUPPORTED;
    const int nh = mlp->n_layers - 1;
    if (nh < 1 || nh > kMaxHidden) return AMLP_ERR_UNSUPPORTED;
    AdjNet net{};
    net.nh = nh;
    net.act = mlp->act;
    long long off = 0;
    int wsm = 0, par = 0;
    for (int k = 0; k <= mlp->n_layers; ++k) net.dims[k] = mlp->dims[k];
    for (int k = 0; k <= nh; ++k) {
        net.woff[k] = off;
        off += (long long)mlp->dims[k + 1] * mlp->dims[k] + mlp->dims[k + 1];
    }
    for (int k = 0; k < nh; ++k) {
        if (mlp->dims[k + 1] > kWpad) return AMLP_ERR_UNSUPPORTED;
        net.kin[k] = k == 0 ? 48 : net.nout[k - 1];
        net.nout[k] = (mlp->dims[k + 1] + 15) / 16 * 16;
        net.wsm_off[k] = wsm;
        wsm += 2 * net.nout[k] * net.kin[k] * 2;
        net.bias_off[k] = par;
        par += net.nout[k];
    }
    net.bias_off[nh] = par;
    par += kWpad + 4;
    net.wsm_total = wsm;
    net.par_total = par;
    const int npts = nep->npts;
    const int rs = 6 * npts + 1 - ((6 * npts) & 1);
    size_t r_bytes = (size_t)kAP * rs * 4, ops_bytes = (size_t)2 * 2 * kAP * kWpad * 2;
    static_assert((size_t)kAP * kGS * 4 <= (size_t)2 * kAP * kWpad * 2, "descriptor partials fit an operand tile");
    const size_t tail = (size_t)kAP * 3 * 4 * 2 + (size_t)2 * kAP * kPartStride * 4 + (size_t)2 * kAP * 4 +
                        (size_t)kAP * 9 * 4 + (size_t)kAP * 2 * 4 + (size_t)3 * npts * 4 + (size_t)kAP * 32 + 16 + 128;
    // R kept apart from the operand tiles (one rotation pass per tile) when it fits
    const size_t smem_keep = align_up(r_bytes, 128) + align_up(ops_bytes, 128) + align_up(wsm, 128) +
                             align_up((size_t)par * 4, 128) + tail;
    const size_t smem_shared = align_up(std::max(r_bytes, ops_bytes), 128) + align_up(wsm, 128) +
                               align_up((size_t)par * 4, 128) + (size_t)kAP * kGS * 4 * 2 + tail;
    const int keep_r = smem_keep <= 220 * 1024 ? 1 : 0;
    const size_t smem = keep_r ? smem_keep : smem_shared;
    if (smem > 220 * 1024) return AMLP_ERR_UNSUPPORTED;
    using Cfg = NepCfg<10, 8, 4, 12>;
    cudaStream_t s = as_stream(stream);
    const float inv_rc = 1.0f / nep->nep_cutoff, rng = nep->en_max - nep->en_min;
    if (d_rep) {
        AMLP_CHECK_CUDA(cudaFuncSetAttribute(k_forces_adjoint<Cfg, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        k_forces_adjoint<Cfg, true><<<kNumSM, kAThreads, smem, s>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap,
                                                                    nep->d_pts, npts, inv_rc, nep->en_min, rng, net,
                                                                    mlp->d_w, d_F, d_T, d_pe, d_rep, d_rp, keep_r);
    } else {
        AMLP_CHECK_CUDA(cudaFuncSetAttribute(k_forces_adjoint<Cfg, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        k_forces_adjoint<Cfg, false><<<kNumSM, kAThreads, smem, s>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap,
                                                                     nep->d_pts, npts, inv_rc, nep->en_min, rng, net,
                                                                     mlp->d_w, d_F, d_T, d_pe, nullptr, nullptr,
                                                                     keep_r);
    }
    return check_launch();
}

extern "C" amlp_status amlp_forces_adjoint(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                           const long long *d_npairs, long long cap, const amlp_nep *nep,
                                           const amlp_mlp *mlp, float *d_F, float *d_T, double *d_pe,
                                           void *stream) {
    return launch_adjoint(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep, mlp, d_F, d_T, d_pe, nullptr, nullptr,
                          stream);
}

extern "C" amlp_status amlp_multi_forces_adjoint(const float *d_pos, const float *d_quat, const int *d_rep,
                                                 const amlp_replica *d_rp, const int *d_pairs,
                                                 const long long *d_npairs, long long cap, const amlp_nep *nep,
                                                 const amlp_mlp *mlp, float *d_F, float *d_T, double *d_pe,
                                                 void *stream) {
    if (!d_rep || !d_rp) return AMLP_ERR_INVALID_ARG;
    return launch_adjoint(d_pos, d_quat, 0.f, d_pairs, d_npairs, cap, nep, mlp, d_F, d_T, d_pe, d_rep, d_rp, stream);
}


constexpr size_t kMlpSmemMax = 226 * 1024;  // dynamic shared memory of k_mlp_grad

// The net of the wide path and k_mlp_grad's geometry: Kg = padded descriptor
// width (the first layer's K), g_ld = row stride of the g rows.
static amlp_status wide_net(const amlp_mlp *mlp, int Kg, int g_ld, AdjNet *net) {
    const int nh = mlp->n_layers - 1;
    if (nh < 1 || nh > kMaxHiddenWide) return AMLP_ERR_UNSUPPORTED;
    *net = AdjNet{};
    net->nh = nh;
    net->act = mlp->act;
    long long off = 0;
    int par = 0, wbytes = 0;
    for (int k = 0; k <= mlp->n_layers; ++k) net->dims[k] = mlp->dims[k];
    for (int k = 0; k <= nh; ++k) {
        net->woff[k] = off;
        off += (long long)mlp->dims[k + 1] * mlp->dims[k] + mlp->dims[k + 1];
    }
    for (int k = 0; k < nh; ++k) {
        if (mlp->dims[k + 1] > kWideMax) return AMLP_ERR_UNSUPPORTED;
        net->kin[k] = k == 0 ? Kg : net->nout[k - 1];
        net->nout[k] = (mlp->dims[k + 1] + 15) / 16 * 16;
        net->bias_off[k] = par;
        par += net->nout[k];
        net->wsm_off[k] = net->wsm_total;  // pre-split weights of layer k: hi then lo
        net->wsm_total += 4 * net->nout[k] * net->kin[k];
        wbytes = std::max(wbytes, 4 * net->nout[k] * net->kin[k]);
        net->wmax = std::max(net->wmax, net->nout[k]);
    }
    net->bias_off[nh] = par;
    par += kWideMax + 4;
    net->par_total = par;
    net->g_ld = g_ld;
    net->gp = Kg;
    net->zbw = std::max(Kg, net->wmax);
    net->relu_bits = mlp->act == AMLP_ACT_RELU ? 1 : 0;
    // smooth activations keep act'(z) of nh - 1 layers in TMEM beside the product region
    if (!net->relu_bits && net->zbw + (nh - 1) * net->wmax > 512) return AMLP_ERR_UNSUPPORTED;
    size_t o = align_up((size_t)2 * kAP * net->zbw * 2, 128);  // operand tile, bf16 hi + lo
    net->wbuf_off = (int)o;
    o += align_up((size_t)wbytes, 128);
    net->par_off = (int)o;
    o += align_up((size_t)par * 4, 128);
    net->eps_off = (int)o;
    o += align_up((size_t)kMQ * kAP * 4, 128);
    net->gbuf_off = (int)o;
    const size_t with_g = o + (size_t)kAP * g_ld * 4;
    net->prefetch_g = with_g <= kMlpSmemMax ? 1 : 0;
    net->smem = (int)(net->prefetch_g ? with_g : o);
    if ((size_t)net->smem > kMlpSmemMax) return AMLP_ERR_UNSUPPORTED;
    return AMLP_OK;
}

extern "C" amlp_status amlp_adjoint_workspace_bytes(long long cap, size_t *bytes) {
    if (cap < 0 || !bytes) return AMLP_ERR_INVALID_ARG;
    *bytes = align_up((size_t)cap * kGRow * 4) + align_up((size_t)cap * kGP * 4) + align_up((size_t)cap * 4) +
             align_up(kWeightSplitBytes) + align_up(adj_a_bytes(cap)) + 256;
    return AMLP_OK;
}

static size_t wide_desc_smem(int npts) {
    const int rs = 6 * npts + 1 - ((6 * npts) & 1);
    return align_up((size_t)kAP * rs * 4, 128) + (size_t)kAP * kGS * 4 * 2 + (size_t)kAP * 3 * 4 * 2 +
           (size_t)2 * kAP * kPartStride * 4 + (size_t)kAP * 9 * 4 + (size_t)kAP * 2 * 4 + (size_t)3 * npts * 4 +
           (size_t)kAP * 32 + 16;
}

static amlp_status check_pair_args(const float *d_pos, const float *d_quat, const int *d_pairs,
                                   const long long *d_npairs, long long cap, const amlp_nep *nep) {
    amlp_status st = check_nep(nep);
    if (st) return st;
    if (!d_pos || !d_quat || !d_npairs || cap < 0 || (cap > 0 && !d_pairs)) return AMLP_ERR_INVALID_ARG;
    if (hyper_kind(nep) == 2) return 2 * nep->npts <= direct::kMaxNd ? AMLP_OK : AMLP_ERR_UNSUPPORTED;
    if (hyper_kind(nep) != 1 || nep_D(nep) > kGP) return AMLP_ERR_UNSUPPORTED;
    return AMLP_OK;
}

// The wide path and amlp_pair_descriptors take the direct-form descriptor
// passes for the hypers (10, 10, 10) and, for (10, 8, 4), for clouds of at most
// 12 points (th_v1, cube_v2), where the O(Nd^2) sum costs less than the
// harmonic form; the multi-system path keeps the harmonic form.
constexpr int kDirectMaxNd47 = 12;
static bool use_direct(const amlp_nep *nep) {
    return hyper_kind(nep) == 2 || (hyper_kind(nep) == 1 && 2 * nep->npts <= kDirectMaxNd47);
}

// Launch of a direct-form descriptor kernel: one thread per pair, grid-stride
// over at most 16 blocks per SM, one float4 of shared memory per point and thread.
template <class K, class... Args>
static amlp_status launch_direct(K kernel, long long cap, int npts, cudaStream_t s, Args... args) {
    const size_t smem = direct::smem_bytes(2 * npts);
    if (smem > 48 * 1024)
        AMLP_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long blocks = min((cap + direct::kThreads - 1) / direct::kThreads, (long long)kNumSM * 16);
    kernel<<<(unsigned)blocks, direct::kThreads, smem, s>>>(args...);
    return AMLP_OK;
}

// Stage events of the wide path (amlp_stage_timing): one set for the library,
// recorded by the last call on its stream.
static bool g_stage_timing = false;
static bool g_stage_recorded = false;
static cudaEvent_t g_stage_ev[4];

static void stage_mark(int k, cudaStream_t s) {
    if (!g_stage_timing) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;  // not in graphs
    cudaEventRecord(g_stage_ev[k], s);
    if (k == 3) g_stage_recorded = true;
}

static amlp_status launch_adjoint_wide(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                       const long long *d_npairs, long long cap, const amlp_nep *nep,
                                       const amlp_mlp *mlp, const float *d_wt, int clip, float *d_F, float *d_T,
                                       double *d_pe, const int *d_rep, const amlp_replica *d_rp, void *d_ws,
                                       size_t ws_bytes, void *stream) {
    amlp_status st = check_pair_args(d_pos, d_quat, d_pairs, d_npairs, cap, nep);
    if (st) return st;
    if ((st = check_mlp(mlp, nep_D(nep)))) return st;
    if (!d_F || !d_T) return AMLP_ERR_INVALID_ARG;
    if (cap == 0) return AMLP_OK;
    size_t need;
    amlp_adjoint_workspace_bytes(cap, &need);
    if (!d_ws || ws_bytes < need) return AMLP_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    const float inv_rc = 1.0f / nep->nep_cutoff, rng = nep->en_max - nep->en_min;
    AdjNet net;
    if (hyper_kind(nep) == 2 || (use_direct(nep) && !d_rep)) {  // the direct-form passes around the same net kernel
        if (d_rep) return AMLP_ERR_UNSUPPORTED;
        const bool k2 = hyper_kind(nep) == 2;
        const int gp = k2 ? kGP2 : kGP, grow = k2 ? kGRow2 : kGRow;
        if ((st = wide_net(mlp, gp, grow, &net))) return st;
        Carver c(d_ws, ws_bytes);
        float *g_rows = c.take<float>((size_t)cap * grow);
        float *dg_rows = c.take<float>((size_t)cap * gp);
        float *y_rows = c.take<float>((size_t)cap);
        char *wsplit = c.take<char>(kWeightSplitBytes);
        if (!c.ok()) return AMLP_ERR_WORKSPACE;
        AMLP_CHECK_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, net.smem));
        const int npts = nep->npts;
        auto fwd = k2 ? direct::k_desc_direct_fwd<11, 11, 10> : direct::k_desc_direct_fwd<11, 9, 4>;
        auto bwd = k2 ? direct::k_desc_direct_bwd<11, 11, 10> : direct::k_desc_direct_bwd<11, 9, 4>;
        stage_mark(0, s);
        if ((st = launch_direct(fwd, cap, npts, s, d_pos, d_quat, box, d_pairs, d_npairs, cap,
                                (const float *)nep->d_pts, npts, inv_rc, g_rows, grow)))
            return st;
        stage_mark(1, s);
        k_split_weights<<<64, 256, 0, s>>>(net, mlp->d_w, wsplit);
        k_mlp_grad<<<kNumSM, kMThreads, net.smem, s>>>(g_rows, d_npairs, cap, net, mlp->d_w, wsplit, y_rows, dg_rows);
        stage_mark(2, s);
        if ((st = launch_direct(bwd, cap, npts, s, d_pos, d_quat, box, d_pairs, d_npairs, cap,
                                (const float *)nep->d_pts, npts, inv_rc, nep->en_min, rng, (const float *)dg_rows, gp,
                                (const float *)y_rows, d_wt, clip, d_F, d_T, d_pe)))
            return st;
        stage_mark(3, s);
        return check_launch();
    }
    if ((st = wide_net(mlp, kGP, kGRow, &net))) return st;
    Carver c(d_ws, ws_bytes);
    float *g_rows = c.take<float>((size_t)cap * kGRow);
    float *dg_rows = c.take<float>((size_t)cap * kGP);
    float *y_rows = c.take<float>((size_t)cap);
    char *wsplit = c.take<char>(kWeightSplitBytes);
    float *a_rows = c.take<float>(adj_a_bytes(cap) / 4);
    const int npts = nep->npts;
    const size_t smem_desc = wide_desc_smem(npts);
    const size_t smem_mlp = (size_t)net.smem;
    if (smem_desc > 220 * 1024) return AMLP_ERR_UNSUPPORTED;
    using Cfg = NepCfg<10, 8, 4, 12>;
    const bool multi = d_rep != nullptr;
    auto fwd = multi ? k_adj_desc<Cfg, true, false> : k_adj_desc<Cfg, false, false>;
    auto bwd = multi ? k_adj_desc<Cfg, true, true> : k_adj_desc<Cfg, false, true>;
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_desc));
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_desc));
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_mlp));
    stage_mark(0, s);
    fwd<<<kNumSM, kAThreads, smem_desc, s>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep->d_pts, npts, inv_rc,
                                             nep->en_min, rng, g_rows, kGRow, nullptr, nullptr, nullptr, clip, d_F,
                                             d_T, d_pe, d_rep, d_rp, a_rows);
    stage_mark(1, s);
    k_split_weights<<<64, 256, 0, s>>>(net, mlp->d_w, wsplit);
    k_mlp_grad<<<kNumSM, kMThreads, smem_mlp, s>>>(g_rows, d_npairs, cap, net, mlp->d_w, wsplit, y_rows, dg_rows);
    stage_mark(2, s);
    bwd<<<kNumSM, kAThreads, smem_desc, s>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep->d_pts, npts, inv_rc,
                                             nep->en_min, rng, nullptr, kGP, dg_rows, y_rows, d_wt, clip, d_F, d_T,
                                             d_pe, d_rep, d_rp, a_rows);
    stage_mark(3, s);
    return check_launch();
}

extern "C" amlp_status amlp_forces_adjoint_wide(const float *d_pos, const float *d_quat, float box,
                                                const int *d_pairs, const long long *d_npairs, long long cap,
                                                const amlp_nep *nep, const amlp_mlp *mlp, float *d_F, float *d_T,
                                                double *d_pe, void *d_ws, size_t ws_bytes, void *stream) {
    return launch_adjoint_wide(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep, mlp, nullptr, 1, d_F, d_T, d_pe,
                               nullptr, nullptr, d_ws, ws_bytes, stream);
}

extern "C" amlp_status amlp_multi_forces_adjoint_wide(const float *d_pos, const float *d_quat, const int *d_rep,
                                                      const amlp_replica *d_rp, const int *d_pairs,
                                                      const long long *d_npairs, long long cap, const amlp_nep *nep,
                                                      const amlp_mlp *mlp, float *d_F, float *d_T, double *d_pe,
                                                      void *d_ws, size_t ws_bytes, void *stream) {
    if (!d_rep || !d_rp) return AMLP_ERR_INVALID_ARG;
    return launch_adjoint_wide(d_pos, d_quat, 0.f, d_pairs, d_npairs, cap, nep, mlp, nullptr, 1, d_F, d_T, d_pe,
                               d_rep, d_rp, d_ws, ws_bytes, stream);
}

extern "C" amlp_status amlp_pair_energy_vjp(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                            const long long *d_npairs, long long cap, const amlp_nep *nep,
                                            const amlp_mlp *mlp, const float *d_wt, int clip, float *d_F,
                                            float *d_T, double *d_pe, void *d_ws, size_t ws_bytes, void *stream) {
    return launch_adjoint_wide(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep, mlp, d_wt, clip ? 1 : 0, d_F, d_T,
                               d_pe, nullptr, nullptr, d_ws, ws_bytes, stream);
}

extern "C" amlp_status amlp_pair_descriptors(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                             const long long *d_npairs, long long cap, const amlp_nep *nep,
                                             float *d_g, int ld_g, void *stream) {
    amlp_status st = check_pair_args(d_pos, d_quat, d_pairs, d_npairs, cap, nep);
    if (st) return st;
    if (!d_g || ld_g < nep_D(nep)) return AMLP_ERR_INVALID_ARG;
    if (cap == 0) return AMLP_OK;
    if (use_direct(nep)) {
        auto fwd = hyper_kind(nep) == 2 ? direct::k_desc_direct_fwd<11, 11, 10> : direct::k_desc_direct_fwd<11, 9, 4>;
        if ((st = launch_direct(fwd, cap, nep->npts, as_stream(stream), d_pos, d_quat, box, d_pairs, d_npairs, cap,
                                (const float *)nep->d_pts, nep->npts, 1.0f / nep->nep_cutoff, d_g, ld_g)))
            return st;
        return check_launch();
    }
    const size_t smem = wide_desc_smem(nep->npts);
    if (smem > 220 * 1024) return AMLP_ERR_UNSUPPORTED;
    using Cfg = NepCfg<10, 8, 4, 12>;
    auto fwd = k_adj_desc<Cfg, false, false>;
    AMLP_CHECK_CUDA(cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fwd<<<kNumSM, kAThreads, smem, as_stream(stream)>>>(d_pos, d_quat, box, d_pairs, d_npairs, cap, nep->d_pts,
                                                        nep->npts, 1.0f / nep->nep_cutoff, nep->en_min,
                                                        nep->en_max - nep->en_min, d_g, ld_g, nullptr, nullptr,
                                                        nullptr, 1, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                        nullptr);
    return check_launch();
}

extern "C" amlp_status amlp_stage_timing(int enable) {
    if (enable && !g_stage_ev[0]) {
        for (auto &e : g_stage_ev) AMLP_CHECK_CUDA(cudaEventCreate(&e));
    }
    g_stage_timing = enable != 0;
    return AMLP_OK;
}

extern "C" amlp_status amlp_stage_times(float *h_ms3) {
    if (!h_ms3) return AMLP_ERR_INVALID_ARG;
    if (!g_stage_recorded) return AMLP_ERR_INVALID_ARG;  // no call recorded its stages yet
    AMLP_CHECK_CUDA(cudaEventSynchronize(g_stage_ev[3]));
    for (int k = 0; k < 3; ++k) AMLP_CHECK_CUDA(cudaEventElapsedTime(h_ms3 + k, g_stage_ev[k], g_stage_ev[k + 1]));
    return AMLP_OK;
}

extern "C" amlp_status amlp_test_first_wait_limit(int polls) {
    if (polls < -1) return AMLP_ERR_INVALID_ARG;
    AMLP_CHECK_CUDA(cudaMemcpyToSymbol(g_amlp_first_wait_limit, &polls, sizeof(int)));
    return AMLP_OK;
}

// The sticky flags as a status, for the handles' synchronisation points (reads
// the flags without clearing them).
amlp_status amlp::device_wait_status() {
    unsigned int f = 0;
    AMLP_CHECK_CUDA(cudaMemcpyFromSymbol(&f, g_amlp_device_error, sizeof(unsigned int)));
    return f ? AMLP_ERR_DEVICE_WAIT : AMLP_OK;
}

extern "C" amlp_status amlp_device_error(unsigned int *flags, int clear) {
    if (!flags) return AMLP_ERR_INVALID_ARG;
    AMLP_CHECK_CUDA(cudaMemcpyFromSymbol(flags, g_amlp_device_error, sizeof(unsigned int)));
    if (clear) {
        unsigned int z = 0;
        AMLP_CHECK_CUDA(cudaMemcpyToSymbol(g_amlp_device_error, &z, sizeof(unsigned int)));
    }
    return AMLP_OK;
}
