// NEP-style pair descriptor on the device.
//
// For a cloud of Nd points p_a (the points of both bodies of a pair), centred
// on their centroid (r_a = p_a - mean p), the reference computes
// (NepDescriptorKernels.py:3-144, DescriptorGenerator.py:296-442)
//   f_n(a)     = (1 + T_n(x_a)) / 2 * fc(u_a),  u = |r_a| / r_c, x = 2 (u-1)^2 - 1,
//                fc = (1 + cos(pi u)) / 2  (no clamp for u > 1), n = 0..nrad
//   g_rad[n]   = sum_a f_n(a)
//   g_ang[n,l] = sum_{a,b} f_n(a) f_n(b) P_l(rhat_a . rhat_b),  n <= nang, l = 1..lmax
// The O(Nd^2) angular double sum is evaluated through the Legendre addition
// theorem, sum_{a,b} f_a f_b P_l(rhat_a.rhat_b) = sum_m (sum_a f_a Y_lm(rhat_a))^2
// with real harmonics scaled so that sum_m Y_lm(u) Y_lm(v) = P_l(u.v); the
// result is the same number with O(Nd) work instead of O(Nd^2).
//
// Harmonic order inside each l (offset l*l - 1): m = 0, then (cos m, sin m) for
// m = 1..l. Y_l0 = P_l(z); Y_lm = N_lm Q_l^m(z) {Re, Im}(x + i y)^m with
// Q_l^m = d^m P_l / dz^m and N_lm = sqrt(2 (l-m)! / (l+m)!).
#pragma once
#include "common.cuh"

namespace amlp {

// N_lm = sqrt(2 (l-m)!/(l+m)!) for m >= 1, 1 for m = 0; l, m <= 10.
__constant__ float c_shnorm[11][11] = {
  {1.000000000e+00f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 1.000000000e+00f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 5.773502692e-01f, 2.886751346e-01f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 4.082482905e-01f, 1.290994449e-01f, 5.270462767e-02f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 3.162277660e-01f, 7.453559925e-02f, 1.992047682e-02f, 7.042952123e-03f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 2.581988897e-01f, 4.879500365e-02f, 9.960238411e-03f, 2.347650708e-03f, 7.423923386e-04f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 2.182178902e-01f, 3.450327797e-02f, 5.750546328e-03f, 1.049901314e-03f, 2.238397122e-04f, 6.461695906e-05f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 1.889822365e-01f, 2.571722499e-02f, 3.636964837e-03f, 5.482930791e-04f, 9.138217986e-05f, 1.792151993e-05f, 4.789727674e-06f, 0.0f, 0.0f, 0.0f},
  {1.000000000e+00f, 1.666666667e-01f, 1.992047682e-02f, 2.452041193e-03f, 3.165571568e-04f, 4.389857925e-05f, 6.773697837e-06f, 1.236702368e-06f, 3.091755919e-07f, 0.0f, 0.0f},
  {1.000000000e+00f, 1.490711985e-01f, 1.589104315e-02f, 1.733854955e-03f, 1.963204147e-04f, 2.346477762e-05f, 3.029289765e-06f, 4.372403153e-07f, 7.498609544e-08f, 1.767439219e-08f, 0.0f},
  {1.000000000e+00f, 1.348399725e-01f, 1.297498240e-02f, 1.272301701e-03f, 1.285218801e-04f, 1.354739567e-05f, 1.514644882e-06f, 1.836776716e-07f, 2.499536515e-08f, 4.054783656e-09f, 9.066771888e-10f}};

__host__ __device__ constexpr int dfact_odd(int m) {  // (2m-1)!!
    int r = 1;
    for (int k = 1; k < 2 * m; k += 2) r *= k;
    return r;
}

template <int NRAD_, int NANG_, int LMAX_, int KC_>
struct NepCfg {
    static constexpr int NRAD = NRAD_, NANG = NANG_, LMAX = LMAX_;
    static constexpr int NR = NRAD + 1;            // radial functions
    static constexpr int NA = NANG + 1;            // radial functions used in the angular part
    static constexpr int K = LMAX * (LMAX + 2);    // harmonics, l = 1..LMAX
    static constexpr int D = NR + NA * LMAX;       // descriptor length
    static constexpr int KC = KC_;                 // harmonics accumulated per pass
    static constexpr int NPASS = (K + KC - 1) / KC;
};

__host__ __device__ constexpr int sh_l_of(int k) {  // l of harmonic index k
    int l = 1;
    while ((l + 1) * (l + 1) - 1 <= k) ++l;
    return l;
}

// All K scaled real harmonics of the unit vector (x, y, z).
template <int LMAX>
__device__ __forceinline__ void sh_eval(float x, float y, float z, float *Y) {
    float C[LMAX + 1], S[LMAX + 1];
    C[0] = 1.0f;
    S[0] = 0.0f;
#pragma unroll
    for (int m = 1; m <= LMAX; ++m) {
        C[m] = fmaf(x, C[m - 1], -y * S[m - 1]);
        S[m] = fmaf(x, S[m - 1], y * C[m - 1]);
    }
#pragma unroll
    for (int m = 0; m <= LMAX; ++m) {
        float q2 = 0.0f, q1 = 0.0f;
#pragma unroll
        for (int l = m; l <= LMAX; ++l) {
            float q;
            if (l == m) q = (float)dfact_odd(m);
            else if (l == m + 1) q = (float)(2 * m + 1) * z * q1;
            else q = ((float)(2 * l - 1) * z * q1 - (float)(l + m - 1) * q2) * (1.0f / (float)(l - m));
            q2 = q1;
            q1 = q;
            if (l >= 1) {
                int base = l * l - 1;
                if (m == 0) {
                    Y[base] = q;
                } else {
                    float nq = c_shnorm[l][m] * q;
                    Y[base + 2 * m - 1] = nq * C[m];
                    Y[base + 2 * m] = nq * S[m];
                }
            }
        }
    }
}

// Radial basis f_n, n = 0..NR-1, of a point at distance d. The cutoff cosine
// comes from the hardware cosine (__cosf: an absolute error of a few 1e-7 for
// the arguments here, smooth in u, so that it cancels in the finite
// differences of neighbouring clouds); cospif costs about twenty more
// instructions per point and finite-difference variant.
template <int NR>
__device__ __forceinline__ void radial_basis(float d, float inv_rc, float *f) {
    float u = d * inv_rc;
    float x = fmaf(2.0f * (u - 1.0f), (u - 1.0f), -1.0f);
    float fc = 0.5f * (1.0f + __cosf(3.14159265358979f * u));
    float hfc = 0.5f * fc;
    float tm1 = 1.0f, t = x;
    f[0] = fc;
    if (NR > 1) f[1] = fmaf(hfc, x, hfc);
#pragma unroll
    for (int n = 2; n < NR; ++n) {
        float tn = fmaf(2.0f * x, t, -tm1);
        tm1 = t;
        t = tn;
        f[n] = fmaf(hfc, tn, hfc);
    }
}

// Descriptor of one point cloud. `pt(a)` returns point a (a < Nd) and
// `pt.point_sum()` the sum of all Nd points. The D values are written to
// g[d * gstride] (a column of a transposed tile). Only the harmonic passes in
// pass_mask run (bit p: harmonics p KC .. p KC + KC - 1); the radial sums are
// written with pass 0, and the angular entries hold the sums of the passes run
// (zero where they have no harmonic), so that a descriptor split over threads
// by passes is the sum of their outputs.
template <class Cfg, class PointFn>
__device__ __forceinline__ void nep_descriptor(const PointFn &pt, int Nd, float inv_rc, float *g, int gstride,
                                               unsigned pass_mask = (1u << Cfg::NPASS) - 1u) {
    const float3 ps = pt.point_sum();
    float inv_nd = 1.0f / (float)Nd;
    const float cx = ps.x * inv_nd, cy = ps.y * inv_nd, cz = ps.z * inv_nd;
    // the angular entries start at zero in g and every pass adds its sums of
    // squares there, so that no register holds them across a pass
#pragma unroll
    for (int i = 0; i < Cfg::NA * Cfg::LMAX; ++i) g[(Cfg::NR + i) * gstride] = 0.f;
#pragma unroll
    for (int pass = 0; pass < Cfg::NPASS; ++pass) {
        if (!((pass_mask >> pass) & 1u)) continue;  // uniform over the warp
        constexpr int KC = Cfg::KC;
        const int k0 = pass * KC;
        float A[Cfg::NA][KC];
        float R[Cfg::NR];
#pragma unroll
        for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
            for (int kk = 0; kk < KC; ++kk) A[n][kk] = 0.f;
#pragma unroll
        for (int n = 0; n < Cfg::NR; ++n) R[n] = 0.f;
        for (int a = 0; a < Nd; ++a) {
            float3 p = pt(a);
            float rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
            float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
            float inv_d = rsqrtf(d2);
            float d = d2 * inv_d;
            float f[Cfg::NR];
            radial_basis<Cfg::NR>(d, inv_rc, f);
            if (pass == 0) {
#pragma unroll
                for (int n = 0; n < Cfg::NR; ++n) R[n] += f[n];
            }
            float Y[Cfg::K];
            sh_eval<Cfg::LMAX>(rx * inv_d, ry * inv_d, rz * inv_d, Y);
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n)
#pragma unroll
                for (int kk = 0; kk < KC; ++kk)
                    if (k0 + kk < Cfg::K) A[n][kk] = fmaf(f[n], Y[k0 + kk], A[n][kk]);
        }
        if (pass == 0) {
#pragma unroll
            for (int n = 0; n < Cfg::NR; ++n) g[n * gstride] = R[n];
        }
        // the l of the pass's harmonics (every index is a constant once the
        // pass loop is unrolled)
#pragma unroll
        for (int l = 1; l <= Cfg::LMAX; ++l) {
            if (l < sh_l_of(k0) || l > sh_l_of(min(k0 + KC, Cfg::K) - 1)) continue;
#pragma unroll
            for (int n = 0; n < Cfg::NA; ++n) {
                float *e = g + (Cfg::NR + n * Cfg::LMAX + l - 1) * gstride;
                float s = *e;
#pragma unroll
                for (int kk = 0; kk < KC; ++kk)
                    if (k0 + kk < Cfg::K && sh_l_of(k0 + kk) == l) s = fmaf(A[n][kk], A[n][kk], s);
                *e = s;
            }
        }
    }
}

// Points of finite-difference variant v of a pair from the rotated body points
// Ri, Rj (body frames rotated into the lab frame, at the origin) and the
// minimum-image translation t = pos_j - pos_i:
//   v = 0..6 use cloud 1 = [Ri, Rj + t], v = 7..9 cloud 2 = [Rj, Ri - t]
//   (PosToPtsKernels.py:3-150), and change the first half of the points:
//   v = 1..3: + dx along x/y/z; v = 4..6 and 7..9: rotation by dteta about x/y/z
//   (PosToPtsKernels.py:153-446).
struct VariantPoints {
    const float *Ri, *Rj;  // npts x 3 (stride 3)
    float tx, ty, tz;
    int h;                 // npts
    int v;
    float dx;
    float4 q;              // rotation of variants 4..9 (identity otherwise)
    // Sum of the variant's points. The rotated half enters as the rotation of its
    // point sum (one rotation instead of one per point; the same sum up to
    // rounding, as the order of a float sum is not the reference's either).
    __device__ __forceinline__ float3 point_sum() const {
        const bool c2 = v >= 7;
        const float *A = c2 ? Rj : Ri, *B = c2 ? Ri : Rj;
        float ax = 0.f, ay = 0.f, az = 0.f, bx = 0.f, by = 0.f, bz = 0.f;
        for (int a = 0; a < h; ++a) {
            ax += A[3 * a], ay += A[3 * a + 1], az += A[3 * a + 2];
            bx += B[3 * a], by += B[3 * a + 1], bz += B[3 * a + 2];
        }
        float3 sa = make_float3(ax, ay, az);
        if (v >= 4) sa = rotate_ref(q, sa);
        const float n = (float)h;
        if (v == 1) sa.x = fmaf(n, dx, sa.x);
        if (v == 2) sa.y = fmaf(n, dx, sa.y);
        if (v == 3) sa.z = fmaf(n, dx, sa.z);
        const float s = c2 ? -1.0f : 1.0f;  // the second half is translated by +t (cloud 1) or -t (cloud 2)
        return make_float3(sa.x + fmaf(s * n, tx, bx), sa.y + fmaf(s * n, ty, by), sa.z + fmaf(s * n, tz, bz));
    }
    __device__ __forceinline__ float3 operator()(int a) const {
        const bool c2 = v >= 7;
        if (a < h) {
            const float *B = c2 ? Rj : Ri;
            float3 p = make_float3(B[3 * a], B[3 * a + 1], B[3 * a + 2]);
            if (v >= 4) return rotate_ref(q, p);
            if (v == 1) p.x = __fadd_rn(p.x, dx);
            if (v == 2) p.y = __fadd_rn(p.y, dx);
            if (v == 3) p.z = __fadd_rn(p.z, dx);
            return p;
        }
        const float *B = c2 ? Ri : Rj;
        int b = a - h;
        float3 p = make_float3(B[3 * b], B[3 * b + 1], B[3 * b + 2]);
        if (c2) return make_float3(__fsub_rn(p.x, tx), __fsub_rn(p.y, ty), __fsub_rn(p.z, tz));
        return make_float3(__fadd_rn(p.x, tx), __fadd_rn(p.y, ty), __fadd_rn(p.z, tz));
    }
};

// Rotation quaternion of variant v (cos(dteta/2), sin(dteta/2) e_axis) with
// the reference's FP32 arguments (PosToPtsKernels.py:225-228).
__device__ __forceinline__ float4 variant_quat(int v, float dteta) {
    float4 q = make_float4(1.f, 0.f, 0.f, 0.f);
    if (v >= 4) {
        float h = __fmul_rn(dteta, 0.5f);
        float c = cosf(h), s = sinf(h);
        int ax = (v - 4) % 3;
        q.x = c;
        if (ax == 0) q.y = s;
        if (ax == 1) q.z = s;
        if (ax == 2) q.w = s;
    }
    return q;
}

}  // namespace amlp
