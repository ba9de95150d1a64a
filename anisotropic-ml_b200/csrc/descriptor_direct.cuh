// Adjoint descriptor passes in the reference's direct form
// (NepDescriptorKernels.py:3-144, DescriptorGenerator.py:296-442):
//   g_rad[n]   = sum_a f_n(a),                              n < NR = nrad + 1
//   g_ang[n,l] = sum_{a,b} f_n(a) f_n(b) P_l(c_ab),         n < NA = nang + 1, 1 <= l <= LM = lmax
// (c_ab = rhat_a . rhat_b), diagonal included, over the Nd points of the pair's
// cloud centred on their centroid. Used for the hypers (10, 10, 10), D = 121, of
// the reference's C100 models, whose 11 x 120 harmonic sums would not fit in
// registers, and for (10, 8, 4), D = 47, when the clouds are small (Nd <= 12:
// th_v1 and cube_v2, 4 and 6 points per body), where the O(Nd^2) sum costs less
// than the harmonic form's per-point work.
//
// Gradient with respect to the centred point r_a (d_a = |r_a|, G = dE/dg_ang,
// R = dE/dg_rad):
//   dE/dr_a = (sum_n R_n f_n'(a)) rhat_a
//           + 2 sum_b [alpha_ab rhat_a + beta_ab (rhat_b - c_ab rhat_a) / d_a],
//   alpha_ab = sum_{n,l} G_nl f_n(b) f_n'(a) P_l(c_ab),
//   beta_ab  = sum_{n,l} G_nl f_n(b) f_n(a) P_l'(c_ab)
// (for b = a the P_l' term vanishes: rhat_a - c_aa rhat_a = 0).
//
// One thread per pair. The thread's cloud sits in shared memory as one float4
// (rhat_a, d_a) per point, laid out point-major with the block's threads
// innermost, so that the 32 lanes of a warp read 32 consecutive float4. The sum
// runs over the unordered point pairs a < b, doubled, plus the diagonal, where
// c_aa = 1 and P_l(1) = 1 exactly; the backward differentiates that same sum.
// No warp reductions: every accumulator stays in its thread's registers.
//
// For b != a the backward needs, per unordered pair, H_n(c) = sum_l G_nl P_l(c)
// and H'_n(c) = sum_l G_nl P_l'(c); then
//   alpha_ab = sum_n f_n'(a) f_n(b) H_n,  alpha_ba = sum_n f_n'(b) f_n(a) H_n,
//   beta     = sum_n f_n(a) f_n(b) H'_n  (= beta_ab = beta_ba),
// and point a gets 2 alpha_ab rhat_a + 2 beta (rhat_b - c rhat_a) / d_a, point b
// the same with a and b swapped. The diagonal adds 2 sum_n f_n'(a) f_n(a) H_n(1)
// to point a along rhat_a. f_n(b) and f_n'(b) are recomputed for every pair
// (a, b) instead of stored, which keeps the shared memory at 16 bytes per point
// and the occupancy bound by registers alone.
// The cloud is built like the other adjoint kernels': rotated by the
// orientation's 3x3 matrix, centred on the centroid of the rotated body-frame
// point sums.
#pragma once
#include "common.cuh"

namespace amlp {
namespace direct {

constexpr int kThreads = 64;  // pairs per block, one thread each
constexpr int kMaxNd = 64;

// Dynamic shared memory of the direct kernels: one float4 per point and thread.
inline size_t smem_bytes(int nd) { return (size_t)nd * kThreads * sizeof(float4); }

// Cutoff-scaled Chebyshev radial basis f_n(d), n < NR, and (with DER) df_n/dd,
// the cutoff cosine from the hardware sine/cosine. The forward and the backward
// pass run this same arithmetic, so that the forces are the exact derivative of
// the energy the forward computed.
template <int NR, bool DER>
__device__ __forceinline__ void radial(float dist, float inv_rc, float *f, float *df) {
    const float u = dist * inv_rc, um1 = u - 1.0f;
    const float x = fmaf(2.0f * um1, um1, -1.0f);
    float s, c;
    __sincosf(3.14159265358979f * u, &s, &c);
    const float hfc = fmaf(0.25f, c, 0.25f);  // fc / 2
    float tm1 = 1.0f, t = x;
    f[0] = 2.0f * hfc;
    f[1] = fmaf(hfc, x, hfc);
    if (DER) {
        const float hdfc = -0.25f * 3.14159265358979f * s * inv_rc;  // (dfc/dd) / 2
        const float hdxfc = 4.0f * um1 * inv_rc * hfc;                // (dx/dd) fc / 2
        float dtm1 = 0.0f, dt = 1.0f;                                 // dT_n/dx
        df[0] = 2.0f * hdfc;
        df[1] = fmaf(hdfc, x, hdfc) + hdxfc;
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
    } else {
#pragma unroll
        for (int n = 2; n < NR; ++n) {
            const float tn = fmaf(2.0f * x, t, -tm1);
            tm1 = t;
            t = tn;
            f[n] = fmaf(hfc, tn, hfc);
        }
    }
}

// One step of the Legendre recurrence: P_{l+1}(c) from P_l = p and P_{l-1} = pm1,
// (l + 1) P_{l+1} = (2l + 1) c P_l - l P_{l-1}, with explicit roundings so that
// both passes get the same values.
__device__ __forceinline__ float legendre_next(int l, float c, float p, float pm1) {
    const float a = (float)(2 * l + 1) / (float)(l + 1), b = (float)l / (float)(l + 1);
    return fmaf(a * c, p, -(b * pm1));
}

// Rotation matrix of the unit quaternion (w, x, y, z): (w^2 - |u|^2) I + 2 u u^T + 2 w [u]x.
__device__ __forceinline__ void quat_matrix(float4 q, float *m) {
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    const float a0 = w * w - (x * x + y * y + z * z);
    m[0] = fmaf(2.f * x, x, a0), m[1] = 2.f * (x * y - w * z), m[2] = 2.f * (x * z + w * y);
    m[3] = 2.f * (x * y + w * z), m[4] = fmaf(2.f * y, y, a0), m[5] = 2.f * (y * z - w * x);
    m[6] = 2.f * (x * z - w * y), m[7] = 2.f * (y * z + w * x), m[8] = fmaf(2.f * z, z, a0);
}

__device__ __forceinline__ float3 mat_apply(const float *m, float px, float py, float pz) {
    return make_float3(fmaf(m[0], px, fmaf(m[1], py, m[2] * pz)), fmaf(m[3], px, fmaf(m[4], py, m[5] * pz)),
                       fmaf(m[6], px, fmaf(m[7], py, m[8] * pz)));
}

// Sum of the body-frame points (the same for every pair).
__device__ __forceinline__ float3 point_sum(const float *pts, int npts) {
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int a = 0; a < npts; ++a) sx += pts[3 * a], sy += pts[3 * a + 1], sz += pts[3 * a + 2];
    return make_float3(sx, sy, sz);
}

// The cloud of pair (i, j) into S[a * kThreads] = (rhat_a, d_a), a < 2 npts
// (S already offset by the thread's index). Returns the translation
// t = pos_j - pos_i, the centroid c and the rotation matrices of both bodies.
__device__ __forceinline__ void build_cloud(float4 *S, const float *pos, const float *quat, float L, int i, int j,
                                            const float *pts, int npts, float3 psum, float3 &t, float3 &cen,
                                            float *mi, float *mj) {
    float dd;
    t = min_image(pos, i, j, L, &dd);
    quat_matrix(load_quat(quat, i), mi);
    quat_matrix(load_quat(quat, j), mj);
    const float3 si = mat_apply(mi, psum.x, psum.y, psum.z), sj = mat_apply(mj, psum.x, psum.y, psum.z);
    const float inv = 1.0f / (float)(2 * npts), n = (float)npts;
    cen = make_float3(fmaf(n, t.x, si.x + sj.x) * inv, fmaf(n, t.y, si.y + sj.y) * inv,
                      fmaf(n, t.z, si.z + sj.z) * inv);
    for (int a = 0; a < 2 * npts; ++a) {
        const int b = a < npts ? a : a - npts;
        const float px = pts[3 * b], py = pts[3 * b + 1], pz = pts[3 * b + 2];
        float3 r = a < npts ? mat_apply(mi, px, py, pz) : mat_apply(mj, px, py, pz);
        if (a >= npts) r.x += t.x, r.y += t.y, r.z += t.z;
        r.x -= cen.x, r.y -= cen.y, r.z -= cen.z;
        const float d2 = fmaf(r.x, r.x, fmaf(r.y, r.y, r.z * r.z));
        const float inv_d = rsqrtf(d2);
        S[a * kThreads] = make_float4(r.x * inv_d, r.y * inv_d, r.z * inv_d, d2 * inv_d);
    }
}

extern __shared__ float4 direct_smem[];

// Forward: row q of g (D values, then zeros up to g_ld) for every filtered pair.
template <int NR, int NA, int LM>
__global__ void __launch_bounds__(kThreads) k_desc_direct_fwd(const float *pos, const float *quat, float L,
                                                              const int *pairs, const long long *d_np, long long cap,
                                                              const float *pts, int npts, float inv_rc, float *g_rows,
                                                              int g_ld) {
    static_assert(NA <= NR && LM >= 2, "angular radial functions are the first NA of the NR");
    constexpr int D = NR + NA * LM;
    float4 *S = direct_smem + threadIdx.x;
    const int nd = 2 * npts;
    const float3 psum = point_sum(pts, npts);
    const long long P = min(*d_np, cap);
    const bool vec = (g_ld & 3) == 0 && (reinterpret_cast<uintptr_t>(g_rows) & 15) == 0;
    for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < P; q += (long long)gridDim.x * kThreads) {
        float3 t, cen;
        float mi[9], mj[9];
        build_cloud(S, pos, quat, L, pairs[2 * q], pairs[2 * q + 1], pts, npts, psum, t, cen, mi, mj);
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
            const float4 A = S[a * kThreads];
            float fa[NR];
            radial<NR, false>(A.w, inv_rc, fa, nullptr);
#pragma unroll
            for (int n = 0; n < NR; ++n) rad[n] += fa[n];
#pragma unroll
            for (int n = 0; n < NA; ++n) dia[n] = fmaf(fa[n], fa[n], dia[n]);
            for (int b = a + 1; b < nd; ++b) {
                const float4 B = S[b * kThreads];
                const float c = fmaf(A.x, B.x, fmaf(A.y, B.y, A.z * B.z));
                float Pl[LM];
                Pl[0] = c;
                Pl[1] = legendre_next(1, c, c, 1.0f);
#pragma unroll
                for (int l = 2; l < LM; ++l) Pl[l] = legendre_next(l, c, Pl[l - 1], Pl[l - 2]);
                float fb[NR];
                radial<NR, false>(B.w, inv_rc, fb, nullptr);
#pragma unroll
                for (int n = 0; n < NA; ++n) {
                    const float ff = fa[n] * fb[n];
#pragma unroll
                    for (int l = 0; l < LM; ++l) acc[n][l] = fmaf(ff, Pl[l], acc[n][l]);
                }
            }
        }
        // g_ang = diagonal + twice the sum over a < b
        float *row = g_rows + q * g_ld;
        auto col_value = [&](int col) -> float {
            if (col < NR) return rad[col];
            if (col < D) {
                const int n = (col - NR) / LM, l = (col - NR) % LM;
                return fmaf(2.0f, acc[n][l], dia[n]);
            }
            return 0.f;
        };
        if (vec) {
#pragma unroll
            for (int c4 = 0; c4 < (D + 3) / 4; ++c4)
                reinterpret_cast<float4 *>(row)[c4] =
                    make_float4(col_value(4 * c4), col_value(4 * c4 + 1), col_value(4 * c4 + 2), col_value(4 * c4 + 3));
            for (int col = 4 * ((D + 3) / 4); col < g_ld; col += 4)
                *reinterpret_cast<float4 *>(row + col) = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
#pragma unroll
            for (int col = 0; col < D; ++col) row[col] = col_value(col);
            for (int col = D; col < g_ld; ++col) row[col] = 0.f;
        }
    }
}

// Backward: dE/dg rows (stride gp >= 4 ceil(D / 4), a multiple of 4 floats,
// 16-byte aligned) and net outputs y in; forces, torques and pair energies out
// (the scaling, clip and scatter of ForceEvaluator.py:119-142). wt (may be null)
// weights pair q's dE/dg by wt[q]; clip = 0 leaves out the clip.
template <int NR, int NA, int LM>
__global__ void __launch_bounds__(kThreads) k_desc_direct_bwd(const float *pos, const float *quat, float L,
                                                              const int *pairs, const long long *d_np, long long cap,
                                                              const float *pts, int npts, float inv_rc, float en_min,
                                                              float en_range, const float *dg_rows, int gp,
                                                              const float *y_rows, const float *wt, int clip,
                                                              float *F, float *T, double *pe) {
    static_assert(NA <= NR && LM >= 2, "angular radial functions are the first NA of the NR");
    constexpr int D = NR + NA * LM;
    float4 *S = direct_smem + threadIdx.x;
    const int nd = 2 * npts;
    const float3 psum = point_sum(pts, npts);
    const long long P = min(*d_np, cap);
    double pe_acc = 0.0;
    for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < P; q += (long long)gridDim.x * kThreads) {
        const int i = pairs[2 * q], j = pairs[2 * q + 1];
        float3 t, cen;
        float mi[9], mj[9];
        build_cloud(S, pos, quat, L, i, j, pts, npts, psum, t, cen, mi, mj);
        const float w = wt ? wt[q] : 1.0f;
        float G[NA][LM], R[NR], Hd[NA];
        {
            const float4 *dg4 = reinterpret_cast<const float4 *>(dg_rows + q * gp);
#pragma unroll
            for (int c4 = 0; c4 < (D + 3) / 4; ++c4) {
                const float4 v4 = dg4[c4];
                const float v[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int col = 4 * c4 + k;
                    if (col < NR) R[col] = w * v[k];
                    else if (col < D) G[(col - NR) / LM][(col - NR) % LM] = w * v[k];
                }
            }
        }
#pragma unroll
        for (int n = 0; n < NA; ++n) {
            float h = 0.f;
#pragma unroll
            for (int l = 0; l < LM; ++l) h += G[n][l];
            Hd[n] = h;  // H_n(1): P_l(1) = 1
        }
        // sums over the points of dE/dr_a (centred r_a): over body i, over all,
        // and the moments r_a x dE/dr_a over body i and over body j
        float Si[3] = {0, 0, 0}, Sa[3] = {0, 0, 0}, Xi[3] = {0, 0, 0}, Xj[3] = {0, 0, 0};
        auto add_grad = [&](int a, const float4 &U, float gx, float gy, float gz) {
            const float rx = U.x * U.w, ry = U.y * U.w, rz = U.z * U.w;
            const float cx = ry * gz - rz * gy, cy = rz * gx - rx * gz, cz = rx * gy - ry * gx;
            Sa[0] += gx, Sa[1] += gy, Sa[2] += gz;
            if (a < npts) {
                Si[0] += gx, Si[1] += gy, Si[2] += gz;
                Xi[0] += cx, Xi[1] += cy, Xi[2] += cz;
            } else {
                Xj[0] += cx, Xj[1] += cy, Xj[2] += cz;
            }
        };
        for (int a = 0; a < nd; ++a) {
            const float4 A = S[a * kThreads];
            float fa[NR], dfa[NR];
            radial<NR, true>(A.w, inv_rc, fa, dfa);
            // radial part and the diagonal: (sum_n R_n f_n'(a) + 2 sum_n f_n'(a) f_n(a) H_n(1)) rhat_a
            float ga = 0.f;
#pragma unroll
            for (int n = 0; n < NR; ++n) ga = fmaf(R[n], dfa[n], ga);
#pragma unroll
            for (int n = 0; n < NA; ++n) ga = fmaf(2.0f * dfa[n] * fa[n], Hd[n], ga);
            float gx = ga * A.x, gy = ga * A.y, gz = ga * A.z;  // dE/dr_a, completed over b below
            const float inv_da = 1.0f / A.w;
            for (int b = a + 1; b < nd; ++b) {
                const float4 B = S[b * kThreads];
                const float c = fmaf(A.x, B.x, fmaf(A.y, B.y, A.z * B.z));
                float H[NA], Hp[NA];
                {
                    // l = 1: P_1 = c, P_1' = 1; then P_{l+1} by the recurrence and
                    // P'_{l+1} = (2l + 1) P_l + P'_{l-1}
                    float pm1 = 1.0f, p = c, dpm1 = 0.0f, dp = 1.0f;
#pragma unroll
                    for (int n = 0; n < NA; ++n) H[n] = G[n][0] * p, Hp[n] = G[n][0];
#pragma unroll
                    for (int l = 1; l < LM; ++l) {
                        const float pn = legendre_next(l, c, p, pm1);
                        const float dpn = fmaf((float)(2 * l + 1), p, dpm1);
                        pm1 = p, p = pn, dpm1 = dp, dp = dpn;
#pragma unroll
                        for (int n = 0; n < NA; ++n) {
                            H[n] = fmaf(G[n][l], p, H[n]);
                            Hp[n] = fmaf(G[n][l], dp, Hp[n]);
                        }
                    }
                }
                float fb[NR], dfb[NR];
                radial<NR, true>(B.w, inv_rc, fb, dfb);
                float al_ab = 0.f, al_ba = 0.f, be = 0.f;
#pragma unroll
                for (int n = 0; n < NA; ++n) {
                    al_ab = fmaf(dfa[n] * fb[n], H[n], al_ab);
                    al_ba = fmaf(dfb[n] * fa[n], H[n], al_ba);
                    be = fmaf(fa[n] * fb[n], Hp[n], be);
                }
                // a: 2 alpha_ab rhat_a + 2 beta (rhat_b - c rhat_a) / d_a; b likewise
                // 2 beta / d_b with the hardware reciprocal (a few ulp; the exact quotient costs an
                // IEEE division per point pair)
                const float wa = 2.0f * be * inv_da, wb = __fdividef(2.0f * be, B.w);
                const float ca = fmaf(-wa, c, 2.0f * al_ab), cb = fmaf(-wb, c, 2.0f * al_ba);
                gx += fmaf(ca, A.x, wa * B.x), gy += fmaf(ca, A.y, wa * B.y), gz += fmaf(ca, A.z, wa * B.z);
                add_grad(b, B, fmaf(cb, B.x, wb * A.x), fmaf(cb, B.y, wb * A.y), fmaf(cb, B.z, wb * A.z));
            }
            add_grad(a, A, gx, gy, gz);
        }
        // torques about the body origins, then the centroid moving with every point
        const float c3[3] = {cen.x, cen.y, cen.z}, e3[3] = {cen.x - t.x, cen.y - t.y, cen.z - t.z};
        const float Sj[3] = {Sa[0] - Si[0], Sa[1] - Si[1], Sa[2] - Si[2]};
        Xi[0] += c3[1] * Si[2] - c3[2] * Si[1], Xi[1] += c3[2] * Si[0] - c3[0] * Si[2];
        Xi[2] += c3[0] * Si[1] - c3[1] * Si[0];
        Xj[0] += e3[1] * Sj[2] - e3[2] * Sj[1], Xj[1] += e3[2] * Sj[0] - e3[0] * Sj[2];
        Xj[2] += e3[0] * Sj[1] - e3[1] * Sj[0];
        const float3 pi3 = mat_apply(mi, psum.x, psum.y, psum.z), qj3 = mat_apply(mj, psum.x, psum.y, psum.z);
        const float Pi[3] = {pi3.x, pi3.y, pi3.z}, Qj[3] = {qj3.x, qj3.y, qj3.z};
        const float inv_nd = 1.0f / (float)nd;
        const float Gm[3] = {Sa[0] * inv_nd, Sa[1] * inv_nd, Sa[2] * inv_nd};
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
            if (clip) f = clip100(f), ti = clip100(ti), tj = clip100(tj);
            atomicAdd(F + 3 * i + k, f);
            atomicAdd(F + 3 * j + k, -f);
            atomicAdd(T + 3 * i + k, ti);
            atomicAdd(T + 3 * j + k, tj);
        }
        pe_acc += (double)en_min + (double)en_range * (double)y_rows[q];
    }
    if (pe) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pe_acc += __shfl_xor_sync(0xffffffffu, pe_acc, o);
        if ((threadIdx.x & 31) == 0 && pe_acc != 0.0) atomicAdd(pe, pe_acc);
    }
}

}  // namespace direct
}  // namespace amlp
