// Two-half MTK Nose-Hoover NVT integrator for rigid bodies (NVT.py:12-129,
// IntegrateStepOneKernels.py, IntegrateStepTwoKernels.py), one thread per body
// for any N (the reference's fixed grids cover N <= 1706).
//
// Per-body arithmetic keeps the reference kernels' FP32 operation order, with
// the double promotions the CUDA C source implies (a `2.0` or `0.5` literal).
// The kinetic-energy sums are FP64: per-block partial sums, reduced by the last
// block to finish (deterministic order), read by the next thermostat update.
#include "common.cuh"

namespace amlp {
namespace {

constexpr int kIntThreads = 256;

// update_variables (IntegrateStepTwoKernels.py:74-130) of one thermostat.
__device__ __forceinline__ void thermo_update(float ts, float tau, float kT, float n_dof, float rn_dof, int nve,
                                              amlp_thermostat *th) {
    if (nve) {
        th->thermo_fac = 1.0f;
        return;
    }
    const float c = __fdiv_rn(__fdiv_rn(ts, tau), tau);
    const float trans_temp = __fmul_rn(__fdiv_rn(2.0f, n_dof), (float)th->ke_t);
    const float gt = __fsub_rn(__fdiv_rn(trans_temp, kT), 1.0f);
    const float xi_p = __fadd_rn(th->xi, __fmul_rn(__fmul_rn(0.5f, c), gt));
    const float xi_new = __fadd_rn(xi_p, __fmul_rn(__fmul_rn(0.5f, c), gt));
    th->eta = __fadd_rn(th->eta, __fmul_rn(xi_p, ts));
    th->thermo_fac = expf(__fmul_rn(__fmul_rn(-0.5f, xi_new), ts));
    th->xi = xi_new;
    const float rot_temp = __fdiv_rn(__fmul_rn(2.0f, (float)th->ke_r), rn_dof);
    const float gr = __fsub_rn(__fdiv_rn(rot_temp, kT), 1.0f);
    const float xr_p = __fadd_rn(th->xi_rot, __fmul_rn(__fmul_rn(0.5f, c), gr));
    th->xi_rot = __fadd_rn(xr_p, __fmul_rn(__fmul_rn(0.5f, c), gr));
    th->eta_rot = __fadd_rn(th->eta_rot, __fmul_rn(xr_p, ts));
}

__global__ void k_thermo_update(amlp_nvt p, amlp_thermostat *th) {
    if (threadIdx.x != 0) return;
    thermo_update(p.dt, p.tau, p.kT, p.n_dof, p.rn_dof, p.nve, th);
}

// NVT.py:42-62 for body i: accel = F/m, v <- v f + (dt/2) accel, and
// step_two_rotation (IntegrateStepTwoKernels.py:2-71): torque into the body
// frame, dp, angular-momentum kick. f and xi_rot come from the body's thermostat.
__device__ __forceinline__ void step_two_body(int i, float *vel, float *accel, const float *F, const float *mass,
                                              const float *quat, const float *T, float *angmom, float *dp, float ts,
                                              float f, float xi_rot) {
    const float m = mass[i], hdt = __fmul_rn(0.5f, ts);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float a = __fdiv_rn(F[3 * i + k], m);
        accel[3 * i + k] = a;
        vel[3 * i + k] = __fadd_rn(__fmul_rn(vel[3 * i + k], f), __fmul_rn(hdt, a));
    }
    float4 q = load_quat(quat, i);
    const float c0 = q.x, c1 = -q.y, c2 = -q.z, c3 = -q.w;
    const float t1 = T[3 * i], t2 = T[3 * i + 1], t3 = T[3 * i + 2];
    const float coef1 = __fsub_rn(__fmul_rn(c0, c0), __fadd_rn(__fadd_rn(__fmul_rn(c1, c1), __fmul_rn(c2, c2)), __fmul_rn(c3, c3)));
    const float t2x = __fmul_rn(__fmul_rn(2.0f, c0), __fsub_rn(__fmul_rn(c2, t3), __fmul_rn(c3, t2)));
    const float t2y = __fmul_rn(__fmul_rn(2.0f, c0), __fsub_rn(__fmul_rn(c3, t1), __fmul_rn(c1, t3)));
    const float t2z = __fmul_rn(__fmul_rn(2.0f, c0), __fsub_rn(__fmul_rn(c1, t2), __fmul_rn(c2, t1)));
    const float ss = __fadd_rn(__fadd_rn(__fmul_rn(c1, t1), __fmul_rn(c2, t2)), __fmul_rn(c3, t3));
    const float tx = __fadd_rn(__fadd_rn(__fmul_rn(t1, coef1), t2x), __fmul_rn(__fmul_rn(2.0f, ss), c1));
    const float ty = __fadd_rn(__fadd_rn(__fmul_rn(t2, coef1), t2y), __fmul_rn(__fmul_rn(2.0f, ss), c2));
    const float tz = __fadd_rn(__fadd_rn(__fmul_rn(t3, coef1), t2z), __fmul_rn(__fmul_rn(2.0f, ss), c3));
    float d[4];
    d[0] = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(c1, tx), __fmul_rn(c2, ty)), __fmul_rn(c3, tz)), ts);
    d[1] = __fmul_rn(__fadd_rn(__fsub_rn(-__fmul_rn(c2, tz), -__fmul_rn(c3, ty)), __fmul_rn(c0, tx)), ts);
    d[2] = __fmul_rn(__fadd_rn(__fsub_rn(-__fmul_rn(c3, tx), -__fmul_rn(c1, tz)), __fmul_rn(c0, ty)), ts);
    d[3] = __fmul_rn(__fadd_rn(__fsub_rn(-__fmul_rn(c1, ty), -__fmul_rn(c2, tx)), __fmul_rn(c0, tz)), ts);
    // expf((-dt/2.0) * xi_rot) with the product in double (IntegrateStepTwoKernels.py:62)
    const float ef = expf((float)(((double)(-ts) / 2.0) * (double)xi_rot));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        dp[4 * i + k] = d[k];
        angmom[4 * i + k] = __fadd_rn(__fmul_rn(angmom[4 * i + k], ef), d[k]);
    }
}

__global__ void k_step_two(float *vel, float *accel, const float *F, const float *mass, const float *quat,
                           const float *T, float *angmom, float *dp, int n, amlp_nvt p, const amlp_thermostat *th) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    step_two_body(i, vel, accel, F, mass, quat, T, angmom, dp, p.dt, th->thermo_fac, th->xi_rot);
}

struct Q4 {
    float a[4];
};

// One free-rotor sub-rotation of step_one_rotation (IntegrateStepOneKernels.py:43-171).
__device__ __forceinline__ void perm_rotate(Q4 &ang, Q4 &ori, int which, float moi_k, float scale_dt) {
    Q4 an, on;
    if (which == 1) {
        an = {{-ang.a[3], ang.a[2], -ang.a[1], ang.a[0]}};
        on = {{-ori.a[3], ori.a[2], -ori.a[1], ori.a[0]}};
    } else if (which == 2) {
        an = {{-ang.a[2], -ang.a[3], ang.a[0], ang.a[1]}};
        on = {{-ori.a[2], -ori.a[3], ori.a[0], ori.a[1]}};
    } else {
        an = {{-ang.a[1], ang.a[0], ang.a[3], -ang.a[2]}};
        on = {{-ori.a[1], ori.a[0], ori.a[3], -ori.a[2]}};
    }
    float dot = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(ang.a[0], on.a[0]), __fmul_rn(ang.a[1], on.a[1])),
                                    __fmul_rn(ang.a[2], on.a[2])), __fmul_rn(ang.a[3], on.a[3]));
    float phi = __fmul_rn(__fdiv_rn(0.25f, moi_k), dot);
    float arg = __fmul_rn(scale_dt, phi);
    float cp = cosf(arg), sp = sinf(arg);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float na = __fadd_rn(__fmul_rn(cp, ang.a[k]), __fmul_rn(sp, an.a[k]));
        float no = __fadd_rn(__fmul_rn(cp, ori.a[k]), __fmul_rn(sp, on.a[k]));
        ang.a[k] = na;
        ori.a[k] = no;
    }
}

// rotational_kinetic_energy (IntegrateStepOneKernels.py:213-251) of one body.
__device__ __forceinline__ float rot_ke(float4 q, const float *p, const float *moi) {
    const float c0 = q.x, c1 = -q.y, c2 = -q.z, c3 = -q.w;
    const float a0 = p[0], a1 = p[1], a2 = p[2], a3 = p[3];
    float sx = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(c0, a1), __fmul_rn(a0, c1)), __fsub_rn(__fmul_rn(c2, a3), __fmul_rn(c3, a2))), 0.5f);
    float sy = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(c0, a2), __fmul_rn(a0, c2)), __fsub_rn(__fmul_rn(c3, a1), __fmul_rn(c1, a3))), 0.5f);
    float sz = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(c0, a3), __fmul_rn(a0, c3)), __fsub_rn(__fmul_rn(c1, a2), __fmul_rn(c2, a1))), 0.5f);
    float e = __fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(sx, sx), moi[0]), __fdiv_rn(__fmul_rn(sy, sy), moi[1])),
                        __fdiv_rn(__fmul_rn(sz, sz), moi[2]));
    return __fmul_rn(e, 0.5f);
}

__device__ __forceinline__ float trans_ke(const float *v, float m) {
    float s = __fadd_rn(__fadd_rn(__fmul_rn(v[0], v[0]), __fmul_rn(v[1], v[1])), __fmul_rn(v[2], v[2]));
    return __fmul_rn(__fmul_rn(0.5f, m), s);
}

// Block sums of (ke_t, ke_r) in FP64 into part[2*block]; the last block to
// finish adds the partials in block order and stores them in th.
__device__ void reduce_ke(double kt, double kr, double *part, unsigned int *done, amlp_thermostat *th) {
    __shared__ double sh[2][kIntThreads / 32];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kt += __shfl_xor_sync(0xffffffffu, kt, o);
        kr += __shfl_xor_sync(0xffffffffu, kr, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = kt;
        sh[1][threadIdx.x >> 5] = kr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kIntThreads / 32; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
        __threadfence();
        unsigned int prev = atomicAdd(done, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        // the last block adds the partials: thread t takes blocks t, t + 256, ... in
        // order, then a fixed tree over the threads (the same order in every run)
        __threadfence();
        double a = 0.0, b = 0.0;
        for (unsigned int k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
            a += ((volatile double *)part)[2 * k];
            b += ((volatile double *)part)[2 * k + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        __syncthreads();  // sh is reused
        if ((threadIdx.x & 31) == 0) {
            sh[0][threadIdx.x >> 5] = a;
            sh[1][threadIdx.x >> 5] = b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double ta = 0.0, tb = 0.0;
            for (int w = 0; w < kIntThreads / 32; ++w) {
                ta += sh[0][w];
                tb += sh[1][w];
            }
            th->ke_t = ta;
            th->ke_r = tb;
            *done = 0;  // ready for the next launch
        }
    }
}

// step_one_translation + step_one_rotation of body i (IntegrateStepOneKernels.py:3-210,
// NVT.py:67-106); returns its translational and rotational kinetic energies.
__device__ __forceinline__ void step_one_body(int i, float *pos, float *vel, const float *accel, float *quat,
                                              float *angmom, const float *dp, const float *mass, float ts, float f,
                                              float xi_rot, float L, const float *moi, double *kt, double *kr) {
    float v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float nv = __fmul_rn(__fadd_rn(vel[3 * i + k], __fmul_rn(__fmul_rn(accel[3 * i + k], 0.5f), ts)), f);
        vel[3 * i + k] = nv;
        v[k] = nv;
        float np = __fadd_rn(pos[3 * i + k], __fmul_rn(nv, ts));
        np = np > 0.5f * L ? __fsub_rn(np, L) : np;
        np = np < -0.5f * L ? __fadd_rn(np, L) : np;
        pos[3 * i + k] = np;
    }
    // rotation: exp factor with the FP32 literal 2.0f (IntegrateStepOneKernels.py:19)
    const float ef = expf(__fmul_rn(__fdiv_rn(-ts, 2.0f), xi_rot));
    Q4 ang, ori;
    float4 q = load_quat(quat, i);
    ori = {{q.x, q.y, q.z, q.w}};
#pragma unroll
    for (int k = 0; k < 4; ++k) ang.a[k] = __fmul_rn(__fadd_rn(angmom[4 * i + k], dp[4 * i + k]), ef);
    const float hts = __fmul_rn(0.5f, ts);
    perm_rotate(ang, ori, 1, moi[2], hts);
    perm_rotate(ang, ori, 2, moi[1], hts);
    perm_rotate(ang, ori, 3, moi[0], ts);
    perm_rotate(ang, ori, 2, moi[1], hts);
    perm_rotate(ang, ori, 1, moi[2], hts);
    float nrm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(ori.a[0], ori.a[0]), __fmul_rn(ori.a[1], ori.a[1])),
                                               __fmul_rn(ori.a[2], ori.a[2])), __fmul_rn(ori.a[3], ori.a[3])));
    float4 qn = make_float4(__fdiv_rn(ori.a[0], nrm), __fdiv_rn(ori.a[1], nrm), __fdiv_rn(ori.a[2], nrm),
                            __fdiv_rn(ori.a[3], nrm));
    reinterpret_cast<float4 *>(quat)[i] = qn;
#pragma unroll
    for (int k = 0; k < 4; ++k) angmom[4 * i + k] = ang.a[k];
    *kt = (double)trans_ke(v, mass[i]);
    *kr = (double)rot_ke(qn, ang.a, moi);
}

// Step one of all bodies plus the kinetic-energy sums (NVT.py:67-129).
__global__ void __launch_bounds__(kIntThreads) k_step_one(float *pos, float *vel, const float *accel, float *quat,
                                                          float *angmom, const float *dp, const float *mass, int n,
                                                          amlp_nvt p, amlp_thermostat *th, double *part,
                                                          unsigned int *done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double kt = 0.0, kr = 0.0;
    if (i < n) step_one_body(i, pos, vel, accel, quat, angmom, dp, mass, p.dt, th->thermo_fac, th->xi_rot, p.box,
                             p.moi, &kt, &kr);
    reduce_ke(kt, kr, part, done, th);
}

// Kinetic energies before the first step (Sim.py:157-158, :171-180).
__global__ void __launch_bounds__(kIntThreads) k_nvt_init(const float *vel, const float *quat, const float *angmom,
                                                          const float *mass, int n, amlp_nvt p, int quirk,
                                                          amlp_thermostat *th, double *part, unsigned int *done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double kt = 0.0, kr = 0.0;
    if (i < n) {
        float v[3] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
        float a[4] = {angmom[4 * i], angmom[4 * i + 1], angmom[4 * i + 2], angmom[4 * i + 3]};
        float e = trans_ke(v, mass[i]);
        kt = (quirk && i != 0) ? 0.0 : (double)e;
        kr = (double)rot_ke(load_quat(quat, i), a, p.moi);
    }
    reduce_ke(kt, kr, part, done, th);
}

int blocks_for(int n) { return (n + kIntThreads - 1) / kIntThreads; }

// ---------------------------------------------------------------- many systems
// Segmented (by system) sum of (kt, kr) over the lanes of a warp whose keys form
// contiguous runs; one FP64 atomic per run into the system's thermostat.
__device__ __forceinline__ void add_ke_by_system(int key, double kt, double kr, amlp_thermostat *th) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ko = __shfl_up_sync(0xffffffffu, key, o);
        double a = __shfl_up_sync(0xffffffffu, kt, o), b = __shfl_up_sync(0xffffffffu, kr, o);
        if (lane >= o && ko == key) {
            kt += a;
            kr += b;
        }
    }
    int kn = __shfl_down_sync(0xffffffffu, key, 1);
    if (key >= 0 && (lane == 31 || kn != key)) {
        atomicAdd(&th[key].ke_t, kt);
        atomicAdd(&th[key].ke_r, kr);
    }
}

__global__ void k_multi_zero_ke(int nrep, amlp_thermostat *th) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep) {
        th[r].ke_t = 0.0;
        th[r].ke_r = 0.0;
    }
}

__global__ void k_multi_nvt_init(const float *vel, const float *quat, const float *angmom, const float *mass,
                                 const int *rep, int n, amlp_nvt p, amlp_thermostat *th) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double kt = 0.0, kr = 0.0;
    int key = -1 - (int)(threadIdx.x & 31);
    if (i < n && rep[i] >= 0) {  // rep < 0: a free body slot
        float v[3] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
        float a[4] = {angmom[4 * i], angmom[4 * i + 1], angmom[4 * i + 2], angmom[4 * i + 3]};
        kt = (double)trans_ke(v, mass[i]);
        kr = (double)rot_ke(load_quat(quat, i), a, p.moi);
        key = rep[i];
    }
    add_ke_by_system(key, kt, kr, th);
}

// Thermostat update of every system; clears its kinetic-energy sums for the
// step one that follows.
__global__ void k_multi_thermo_update(int nrep, const amlp_replica *rp, amlp_nvt p, amlp_thermostat *th) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    const amlp_replica q = rp[r];
    if (!(q.n_dof > 0.f)) return;  // a free system slot
    thermo_update(p.dt, p.tau, q.kT, q.n_dof, q.rn_dof, q.nve, th + r);
    th[r].ke_t = 0.0;
    th[r].ke_r = 0.0;
}

__global__ void k_multi_step_two(float *vel, float *accel, const float *F, const float *mass, const float *quat,
                                 const float *T, float *angmom, float *dp, const int *rep, int n, amlp_nvt p,
                                 const amlp_thermostat *th) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || rep[i] < 0) return;  // rep < 0: a free body slot
    const amlp_thermostat *t = th + rep[i];
    step_two_body(i, vel, accel, F, mass, quat, T, angmom, dp, p.dt, t->thermo_fac, t->xi_rot);
}

__global__ void __launch_bounds__(kIntThreads) k_multi_step_one(float *pos, float *vel, const float *accel,
                                                                float *quat, float *angmom, const float *dp,
                                                                const float *mass, const int *rep, int n,
                                                                const amlp_replica *rp, amlp_nvt p,
                                                                amlp_thermostat *th) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double kt = 0.0, kr = 0.0;
    int key = -1 - (int)(threadIdx.x & 31);
    if (i < n && rep[i] >= 0) {  // rep < 0: a free body slot
        key = rep[i];
        const amlp_thermostat *t = th + key;
        step_one_body(i, pos, vel, accel, quat, angmom, dp, mass, p.dt, t->thermo_fac, t->xi_rot, rp[key].box, p.moi,
                      &kt, &kr);
    }
    add_ke_by_system(key, kt, kr, th);
}

}  // namespace
}  // namespace amlp

using namespace amlp;

extern "C" amlp_status amlp_nvt_workspace_bytes(int n, size_t *bytes) {
    if (n <= 0 || !bytes) return AMLP_ERR_INVALID_ARG;
    *bytes = align_up(sizeof(unsigned int)) + align_up(2 * sizeof(double) * blocks_for(n));
    return AMLP_OK;
}

static amlp_status nvt_ws(void *d_ws, size_t ws_bytes, int n, double **part, unsigned int **done) {
    size_t need;
    amlp_nvt_workspace_bytes(n, &need);
    if (!d_ws || ws_bytes < need) return AMLP_ERR_WORKSPACE;
    *done = static_cast<unsigned int *>(d_ws);
    *part = reinterpret_cast<double *>(static_cast<char *>(d_ws) + align_up(sizeof(unsigned int)));
    return AMLP_OK;
}

extern "C" amlp_status amlp_nvt_init(const float *d_vel, const float *d_quat, const float *d_angmom,
                                     const float *d_mass, int n, const amlp_nvt *prm, int initial_ke_quirk,
                                     amlp_thermostat *d_th, void *d_ws, size_t ws_bytes, void *stream) {
    if (n <= 0 || !prm || !d_vel || !d_quat || !d_angmom || !d_mass || !d_th) return AMLP_ERR_INVALID_ARG;
    double *part;
    unsigned int *done;
    amlp_status st = nvt_ws(d_ws, ws_bytes, n, &part, &done);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    AMLP_CHECK_CUDA(cudaMemsetAsync(done, 0, sizeof(unsigned int), s));
    k_nvt_init<<<blocks_for(n), kIntThreads, 0, s>>>(d_vel, d_quat, d_angmom, d_mass, n, *prm, initial_ke_quirk,
                                                     d_th, part, done);
    return check_launch();
}

extern "C" amlp_status amlp_nvt_step_two(float *d_vel, float *d_accel, const float *d_F, const float *d_mass,
                                         const float *d_quat, const float *d_T, float *d_angmom, float *d_dp, int n,
                                         const amlp_nvt *prm, amlp_thermostat *d_th, void *stream) {
    if (n <= 0 || !prm || !d_vel || !d_accel || !d_F || !d_mass || !d_quat || !d_T || !d_angmom || !d_dp || !d_th)
        return AMLP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    k_thermo_update<<<1, 32, 0, s>>>(*prm, d_th);
    k_step_two<<<blocks_for(n), kIntThreads, 0, s>>>(d_vel, d_accel, d_F, d_mass, d_quat, d_T, d_angmom, d_dp, n, *prm,
                                                     d_th);
    return check_launch();
}

extern "C" amlp_status amlp_nvt_step_one(float *d_pos, float *d_vel, const float *d_accel, float *d_quat,
                                         float *d_angmom, const float *d_dp, const float *d_mass, int n,
                                         const amlp_nvt *prm, amlp_thermostat *d_th, void *d_ws, size_t ws_bytes,
                                         void *stream) {
    if (n <= 0 || !prm || !d_pos || !d_vel || !d_accel || !d_quat || !d_angmom || !d_dp || !d_mass || !d_th)
        return AMLP_ERR_INVALID_ARG;
    double *part;
    unsigned int *done;
    amlp_status st = nvt_ws(d_ws, ws_bytes, n, &part, &done);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    AMLP_CHECK_CUDA(cudaMemsetAsync(done, 0, sizeof(unsigned int), s));
    k_step_one<<<blocks_for(n), kIntThreads, 0, s>>>(d_pos, d_vel, d_accel, d_quat, d_angmom, d_dp,
                                                                     d_mass, n, *prm, d_th, part, done);
    return check_launch();
}

extern "C" amlp_status amlp_multi_nvt_init(const float *d_vel, const float *d_quat, const float *d_angmom,
                                           const float *d_mass, const int *d_rep, int n, int nrep,
                                           const amlp_nvt *prm, amlp_thermostat *d_th, void *stream) {
    if (n <= 0 || nrep <= 0 || !prm || !d_vel || !d_quat || !d_angmom || !d_mass || !d_rep || !d_th)
        return AMLP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    k_multi_zero_ke<<<(nrep + 127) / 128, 128, 0, s>>>(nrep, d_th);
    k_multi_nvt_init<<<blocks_for(n), kIntThreads, 0, s>>>(d_vel, d_quat, d_angmom, d_mass, d_rep, n, *prm, d_th);
    return check_launch();
}

extern "C" amlp_status amlp_multi_nvt_step_two(float *d_vel, float *d_accel, const float *d_F, const float *d_mass,
                                               const float *d_quat, const float *d_T, float *d_angmom, float *d_dp,
                                               const int *d_rep, int n, int nrep, const amlp_replica *d_rp,
                                               const amlp_nvt *prm, amlp_thermostat *d_th, void *stream) {
    if (n <= 0 || nrep <= 0 || !prm || !d_vel || !d_accel || !d_F || !d_mass || !d_quat || !d_T || !d_angmom ||
        !d_dp || !d_rep || !d_rp || !d_th)
        return AMLP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    k_multi_thermo_update<<<(nrep + 127) / 128, 128, 0, s>>>(nrep, d_rp, *prm, d_th);
    k_multi_step_two<<<blocks_for(n), kIntThreads, 0, s>>>(d_vel, d_accel, d_F, d_mass, d_quat, d_T, d_angmom, d_dp,
                                                           d_rep, n, *prm, d_th);
    return check_launch();
}

extern "C" amlp_status amlp_multi_nvt_step_one(float *d_pos, float *d_vel, const float *d_accel, float *d_quat,
                                               float *d_angmom, const float *d_dp, const float *d_mass,
                                               const int *d_rep, int n, const amlp_replica *d_rp,
                                               const amlp_nvt *prm, amlp_thermostat *d_th, void *stream) {
    if (n <= 0 || !prm || !d_pos || !d_vel || !d_accel || !d_quat || !d_angmom || !d_dp || !d_mass || !d_rep ||
        !d_rp || !d_th)
        return AMLP_ERR_INVALID_ARG;
    k_multi_step_one<<<blocks_for(n), kIntThreads, 0, as_stream(stream)>>>(d_pos, d_vel, d_accel, d_quat, d_angmom,
                                                                          d_dp, d_mass, d_rep, n, d_rp, *prm, d_th);
    return check_launch();
}
