// Adjoint descriptor passes for the hypers (nrad, nang, lmax) = (10, 10, 10),
// D = 121, of the reference's C100 models, in the reference's direct form
// (NepDescriptorKernels.py:3-144, DescriptorGenerator.py:296-442):
//   g_rad[n]   = sum_a f_n(a)
//   g_ang[n,l] = sum_{a,b} f_n(a) f_n(b) P_l(c_ab),  c_ab = rhat_a . rhat_b,
// diagonal included, over the Nd points of the pair's cloud centred on their
// centroid. The shapes these models belong to have few points (th_v1 4, cube_v2
// 6, pbp_v3 7 per body), so the O(Nd^2) sum is cheaper here than 11 x 120
// harmonic sums per point.
//
// Gradient with respect to the centred point r_a (d_a = |r_a|, G = dE/dg_ang,
// R = dE/dg_rad):
//   dE/dr_a = (sum_n R_n f_n'(a)) rhat_a
//           + 2 sum_b [alpha_ab rhat_a + beta_ab (rhat_b - c_ab rhat_a) / d_a],
//   alpha_ab = sum_{n,l} G_nl f_n(b) f_n'(a) P_l(c_ab),
//   beta_ab  = sum_{n,l} G_nl f_n(b) f_n(a) P_l'(c_ab)
// (for b = a the P_l' term vanishes: rhat_a - c_aa rhat_a = 0).
//
// One warp per pair; lane a holds points a and a + 32 (Nd <= 64). The cloud is
// built like the other adjoint kernels': rotated by the orientation's 3x3
// matrix, centred on the centroid of the rotated body-frame point sums.
#pragma once
#include "common.cuh"

namespace amlp {
namespace direct {

constexpr int NR = 11, NA = 11, LM = 10, D = NR + NA * LM;  // 121
constexpr int kWarps = 4;  // warps (pairs in flight) per block (static shared memory <= 48 KB)
constexpr int kMaxNd = 64;

// Per-warp scratch: the cloud's unit vectors, distances and radial basis.
struct Cloud {
    float ux[kMaxNd], uy[kMaxNd], uz[kMaxNd], d[kMaxNd];
    float rx[kMaxNd], ry[kMaxNd], rz[kMaxNd];
    float f[kMaxNd][NR], df[kMaxNd][NR];
};

// f_n and df_n/dd with the cutoff cosine from the hardware sine/cosine, the same
// arithmetic in the forward and the backward pass.
__device__ __forceinline__ void radial(float dist, float inv_rc, float *f, float *df) {
    const float u = dist * inv_rc, um1 = u - 1.0f;
    const float x = fmaf(2.0f * um1, um1, -1.0f);
    float s, c;
    __sincosf(3.14159265358979f * u, &s, &c);
    const float hfc = fmaf(0.25f, c, 0.25f);
    const float hdfc = -0.25f * 3.14159265358979f * s * inv_rc;
    const float hdxfc = 4.0f * um1 * inv_rc * hfc;
    float tm1 = 1.0f, t = x, dtm1 = 0.0f, dt = 1.0f;
    f[0] = 2.0f * hfc;
    df[0] = 2.0f * hdfc;
    f[1] = fmaf(hfc, x, hfc);
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
}

// P_l(c), l = 1..LM, and (when DER) P_l'(c), by the three-term recurrences.
template <bool DER>
__device__ __forceinline__ void legendre(float c, float *P, float *dP) {
    float pm1 = 1.0f, p = c, dpm1 = 0.0f, dp = 1.0f;
    P[0] = p;
    if (DER) dP[0] = dp;
#pragma unroll
    for (int l = 1; l < LM; ++l) {
        const float pn = ((float)(2 * l + 1) * c * p - (float)l * pm1) * (1.0f / (float)(l + 1));
        if (DER) {
            const float dpn = fmaf((float)(2 * l + 1), p, dpm1);
            dpm1 = dp;
            dp = dpn;
            dP[l] = dpn;
        }
        pm1 = p;
        p = pn;
        P[l] = pn;
    }
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

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The pair's cloud into C (all lanes of the warp take part). Returns the
// translation t = pos_j - pos_i and the centroid c (same in every lane), and
// the rotation matrices of both bodies.
__device__ __forceinline__ void build_cloud(Cloud &C, const float *pos, const float *quat, float L, int i, int j,
                                            const float *pts, int npts, float inv_rc, float3 &t, float3 &cen,
                                            float *mi, float *mj) {
    const int lane = threadIdx.x & 31, nd = 2 * npts;
    float dd;
    t = min_image(pos, i, j, L, &dd);
    quat_matrix(load_quat(quat, i), mi);
    quat_matrix(load_quat(quat, j), mj);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int a = lane; a < npts; a += 32) sx += pts[3 * a], sy += pts[3 * a + 1], sz += pts[3 * a + 2];
    sx = warp_sum(sx), sy = warp_sum(sy), sz = warp_sum(sz);
    const float3 si = mat_apply(mi, sx, sy, sz), sj = mat_apply(mj, sx, sy, sz);
    const float inv = 1.0f / (float)nd, n = (float)npts;
    cen = make_float3(fmaf(n, t.x, si.x + sj.x) * inv, fmaf(n, t.y, si.y + sj.y) * inv,
                      fmaf(n, t.z, si.z + sj.z) * inv);
    for (int a = lane; a < nd; a += 32) {
        const int b = a < npts ? a : a - npts;
        const float px = pts[3 * b], py = pts[3 * b + 1], pz = pts[3 * b + 2];
        float3 r = a < npts ? mat_apply(mi, px, py, pz) : mat_apply(mj, px, py, pz);
        if (a >= npts) r.x += t.x, r.y += t.y, r.z += t.z;
        r.x -= cen.x, r.y -= cen.y, r.z -= cen.z;
        const float d2 = fmaf(r.x, r.x, fmaf(r.y, r.y, r.z * r.z));
        const float inv_d = rsqrtf(d2), dist = d2 * inv_d;
        C.rx[a] = r.x, C.ry[a] = r.y, C.rz[a] = r.z;
        C.ux[a] = r.x * inv_d, C.uy[a] = r.y * inv_d, C.uz[a] = r.z * inv_d, C.d[a] = dist;
        radial(dist, inv_rc, C.f[a], C.df[a]);
    }
    __syncwarp();
}


// Forward: row q of g (121 values, then zeros up to g_ld) for every filtered pair.
__global__ void __launch_bounds__(32 * kWarps) k_desc_direct_fwd(const float *pos, const float *quat, float L,
                                                                   const int *pairs, const long long *d_np,
                                                                   long long cap, const float *pts, int npts,
                                                                   float inv_rc, float *g_rows, int g_ld) {
    __shared__ Cloud clouds[kWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    Cloud &C = clouds[wib];
    const int nd = 2 * npts;
    const long long P = min(*d_np, cap);
    for (long long q = (long long)blockIdx.x * kWarps + wib; q < P; q += (long long)gridDim.x * kWarps) {
        const int i = pairs[2 * q], j = pairs[2 * q + 1];
        float3 t, cen;
        float mi[9], mj[9];
        build_cloud(C, pos, quat, L, i, j, pts, npts, inv_rc, t, cen, mi, mj);
        float acc[NA][LM], rad[NR];
#pragma unroll
        for (int n = 0; n < NA; ++n)
#pragma unroll
            for (int l = 0; l < LM; ++l) acc[n][l] = 0.f;
#pragma unroll
        for (int n = 0; n < NR; ++n) rad[n] = 0.f;
        for (int a = lane; a < nd; a += 32)
#pragma unroll
            for (int n = 0; n < NR; ++n) rad[n] += C.f[a][n];
        // the point pairs (a, b) spread over the lanes: every lane busy even for 8-point clouds
        for (int ab = lane; ab < nd * nd; ab += 32) {
            const int a = ab / nd, b = ab - a * nd;
            float Pl[LM];
            legendre<false>(fmaf(C.ux[a], C.ux[b], fmaf(C.uy[a], C.uy[b], C.uz[a] * C.uz[b])), Pl, nullptr);
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                const float ff = C.f[a][n] * C.f[b][n];
#pragma unroll
                for (int l = 0; l < LM; ++l) acc[n][l] = fmaf(ff, Pl[l], acc[n][l]);
            }
        }
        // warp sums; lane k writes columns k, k + 32, ...
        float *row = g_rows + q * g_ld;
#pragma unroll
        for (int n = 0; n < NR; ++n) {
            const float v = warp_sum(rad[n]);
            if (lane == n) row[n] = v;
        }
#pragma unroll
        for (int n = 0; n < NA; ++n)
#pragma unroll
            for (int l = 0; l < LM; ++l) {
                const float v = warp_sum(acc[n][l]);
                const int col = NR + n * LM + l;
                if (lane == (col & 31)) row[col] = v;
            }
        for (int col = D + lane; col < g_ld; col += 32) row[col] = 0.f;
        __syncwarp();
    }
}

// Backward: dE/dg rows (stride gp) and net outputs y in; forces, torques and
// pair energies out (the scaling, clip and scatter of ForceEvaluator.py:119-142).
// wt (may be null) weights pair q's dE/dg by wt[q]; clip = 0 leaves out the clip.
__global__ void __launch_bounds__(32 * kWarps) k_desc_direct_bwd(const float *pos, const float *quat, float L,
                                                                   const int *pairs, const long long *d_np,
                                                                   long long cap, const float *pts, int npts,
                                                                   float inv_rc, float en_min, float en_range,
                                                                   const float *dg_rows, int gp, const float *y_rows,
                                                                   const float *wt, int clip, float *F, float *T,
                                                                   double *pe) {
    __shared__ Cloud clouds[kWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    Cloud &C = clouds[wib];
    const int nd = 2 * npts;
    const long long P = min(*d_np, cap);
    double pe_acc = 0.0;
    for (long long q = (long long)blockIdx.x * kWarps + wib; q < P; q += (long long)gridDim.x * kWarps) {
        const int i = pairs[2 * q], j = pairs[2 * q + 1];
        float3 t, cen;
        float mi[9], mj[9];
        build_cloud(C, pos, quat, L, i, j, pts, npts, inv_rc, t, cen, mi, mj);
        const float w = wt ? wt[q] : 1.0f;
        const float *dg = dg_rows + q * gp;
        float G[NA][LM], R[NR];
#pragma unroll
        for (int n = 0; n < NR; ++n) R[n] = w * dg[n];
#pragma unroll
        for (int n = 0; n < NA; ++n)
#pragma unroll
            for (int l = 0; l < LM; ++l) G[n][l] = w * dg[NR + n * LM + l];
        // per-lane partial sums over its points: sum_{a in i} G_a, sum_a G_a,
        // sum_{a in i} r_a x G_a, sum_{a in j} r_a x G_a (centred r_a)
        float Si[3] = {0, 0, 0}, Sa[3] = {0, 0, 0}, Xi[3] = {0, 0, 0}, Xj[3] = {0, 0, 0};
        // the gradient dE/dr_a is linear in its terms, and so are the sums over a below: the
        // point pairs (a, b) spread over the lanes, each lane adding the terms of its pairs
        auto add_grad = [&](int a, float Gx, float Gy, float Gz) {
            const float rx = C.rx[a], ry = C.ry[a], rz = C.rz[a];
            const float cx = ry * Gz - rz * Gy, cy = rz * Gx - rx * Gz, cz = rx * Gy - ry * Gx;
            Sa[0] += Gx, Sa[1] += Gy, Sa[2] += Gz;
            if (a < npts) {
                Si[0] += Gx, Si[1] += Gy, Si[2] += Gz;
                Xi[0] += cx, Xi[1] += cy, Xi[2] += cz;
            } else {
                Xj[0] += cx, Xj[1] += cy, Xj[2] += cz;
            }
        };
        for (int a = lane; a < nd; a += 32) {  // radial part: (sum_n R_n f_n'(a)) rhat_a
            float ga = 0.f;
#pragma unroll
            for (int n = 0; n < NR; ++n) ga = fmaf(R[n], C.df[a][n], ga);
            add_grad(a, ga * C.ux[a], ga * C.uy[a], ga * C.uz[a]);
        }
        for (int ab = lane; ab < nd * nd; ab += 32) {
            const int a = ab / nd, b = ab - a * nd;
            const float ax = C.ux[a], ay = C.uy[a], az = C.uz[a];
            const float bx = C.ux[b], by = C.uy[b], bz = C.uz[b];
            const float c = fmaf(ax, bx, fmaf(ay, by, az * bz));
            float Pl[LM], dPl[LM];
            legendre<true>(c, Pl, dPl);
            float al = 0.f, be = 0.f;
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                const float fb = C.f[b][n];
                float sp = 0.f, sd = 0.f;
#pragma unroll
                for (int l = 0; l < LM; ++l) {
                    sp = fmaf(G[n][l], Pl[l], sp);
                    sd = fmaf(G[n][l], dPl[l], sd);
                }
                al = fmaf(fb * C.df[a][n], sp, al);
                be = fmaf(fb * C.f[a][n], sd, be);
            }
            // 2 alpha_ab rhat_a + 2 beta_ab (rhat_b - c_ab rhat_a) / d_a (no beta term for b = a)
            const float wb = b != a ? 2.0f * be / C.d[a] : 0.f;
            const float cu = fmaf(-wb, c, 2.0f * al);
            add_grad(a, fmaf(cu, ax, wb * bx), fmaf(cu, ay, wb * by), fmaf(cu, az, wb * bz));
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Si[k] = warp_sum(Si[k]), Sa[k] = warp_sum(Sa[k]), Xi[k] = warp_sum(Xi[k]), Xj[k] = warp_sum(Xj[k]);
        }
        if (lane == 0) {
            // torques about the body origins, then the centroid moving with every point
            const float c3[3] = {cen.x, cen.y, cen.z}, e3[3] = {cen.x - t.x, cen.y - t.y, cen.z - t.z};
            const float Sj[3] = {Sa[0] - Si[0], Sa[1] - Si[1], Sa[2] - Si[2]};
            Xi[0] += c3[1] * Si[2] - c3[2] * Si[1], Xi[1] += c3[2] * Si[0] - c3[0] * Si[2];
            Xi[2] += c3[0] * Si[1] - c3[1] * Si[0];
            Xj[0] += e3[1] * Sj[2] - e3[2] * Sj[1], Xj[1] += e3[2] * Sj[0] - e3[0] * Sj[2];
            Xj[2] += e3[0] * Sj[1] - e3[1] * Sj[0];
            float sx = 0.f, sy = 0.f, sz = 0.f;
            for (int a = 0; a < npts; ++a) sx += pts[3 * a], sy += pts[3 * a + 1], sz += pts[3 * a + 2];
            const float3 pi3 = mat_apply(mi, sx, sy, sz), qj3 = mat_apply(mj, sx, sy, sz);
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
        __syncwarp();
    }
    if (pe && lane == 0 && pe_acc != 0.0) atomicAdd(pe, pe_acc);
}

}  // namespace direct
}  // namespace amlp
