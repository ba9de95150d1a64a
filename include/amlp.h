/*
 * amlp.h -- C ABI of libamlp.so, the B200 (sm_100a) implementation of the
 * per-step force evaluation and NVT rigid-body integration of the reference's
 * nep_simulator (baho-cb/anisotropic-ML).
 *
 * Conventions
 *   - Every pointer argument named d_* is device memory owned by the caller.
 *     The library allocates nothing except where a function says so; scratch
 *     memory is a caller-provided workspace whose size a *_workspace_bytes()
 *     query returns.
 *   - Every function returns an amlp_status (0 = success) and never exits the
 *     process. Kernel launches are asynchronous on the given stream; launch
 *     errors are reported by the call, device-side errors at the next
 *     synchronisation.
 *   - Layouts follow the reference: positions (N,3) f32, orientations and
 *     angular momenta (N,4) f32 as (w,x,y,z) quaternions (HOOMD convention),
 *     forces/torques (N,3) f32, pair lists (P,2) with i < j. Pair indices are
 *     int32 here (the reference keeps int64 from scipy). Filtered pair lists
 *     may come in any order; the lists amlp_pair_filter writes are sorted by
 *     (i, j), which lets the force kernels merge a warp's atomics per body.
 *   - The stateless calls take every buffer from the caller; calls on one
 *     stream are ordered, calls on different streams that share output
 *     buffers race. The handles at the end of this file (amlp_sim,
 *     amlp_pool) own their buffers and sequence those calls.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   amlp_nlist_build      Sim.setNeighborList / Sim.refreshNList   Sim.py:85-92, :192-198
 *   amlp_nlist_build_gated, amlp_nlist_check_displacement
 *                         the rebuild schedule of Sim.run (every 100 steps, Sim.py:218-221)
 *                         replaced by a displacement criterion (opt-in)
 *   amlp_pair_filter      DescriptorGenerator.pos_to_pts (filter)  DescriptorGenerator.py:168-182
 *   amlp_descriptors      DescriptorGenerator.generate_nep_descriptors  DescriptorGenerator.py:136-161
 *                         (pos_to_pts :163-218, apply_dx_dteta :220-255, pts_to_nep_descriptors :296-442)
 *   amlp_mlp_energy       ForceEvaluator.evaluate_gradients (net forward)  ForceEvaluator.py:80-83
 *   amlp_mlp_loss_grad    FFNN.train_step loss.backward (MSE on normalised energies)  05/FFNN.py:95-106
 *   amlp_fd_scatter       ForceEvaluator.evaluate_gradients (differences) + evaluate_forces_torques
 *                         ForceEvaluator.py:86-146
 *   amlp_forces_fd        Sim.step lines 261-266 (descriptors + evaluate_interactions), fused
 *   amlp_forces_adjoint   same call with analytic forces/torques (no reference counterpart)
 *   amlp_nvt_step_two     NVT.integrate_step_two  NVT.py:17-64
 *   amlp_nvt_step_one     NVT.integrate_step_one  NVT.py:12-15, :67-129
 *   amlp_nvt_init         Sim.move_data_to_device kinetic energies  Sim.py:157-158, :171-180
 *   amlp_device_error     (no reference counterpart: error flags of bounded device waits)
 */
#ifndef AMLP_H
#define AMLP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int amlp_status;
#define AMLP_OK 0
#define AMLP_ERR_INVALID_ARG 1     /* bad size, null pointer or unsupported parameter */
#define AMLP_ERR_UNSUPPORTED 2     /* hypers / widths without a compiled kernel */
#define AMLP_ERR_WORKSPACE 3       /* workspace smaller than the query returned */
#define AMLP_ERR_CUDA 4            /* a CUDA call failed (see amlp_last_cuda_error) */
#define AMLP_ERR_CAPACITY 5        /* output capacity too small (count still written) */
#define AMLP_ERR_TOO_LARGE 6       /* size beyond the fixed scratch of an allocation-free entry point */
#define AMLP_ERR_DEVICE_WAIT 7     /* a bounded device-side wait gave up (amlp_device_error; clear it there) */

#define AMLP_ACT_RELU 0
#define AMLP_ACT_TANH 1
#define AMLP_ACT_SILU 2
#define AMLP_MAX_LAYERS 8
#define AMLP_MAX_PTS 64            /* points per body; a pair cloud holds 2x */

/* Pair-energy descriptor and shape, DescriptorGenerator.setHyperParameters /
 * setShape (DescriptorGenerator.py:37-43, :58-125). D = (nrad+1) + (nang+1)*lmax. */
typedef struct amlp_nep {
    int nrad, nang, lmax;
    int npts;                 /* points per body, <= AMLP_MAX_PTS */
    const float *d_pts;       /* (npts,3) body-frame points */
    double cutoff;            /* pair filter: centre distance < cutoff (compared in FP64) */
    float nep_cutoff;         /* descriptor radius r_c */
    float en_min, en_max;     /* net output y maps to E = en_min + (en_max-en_min) y */
    float dx, dteta;          /* finite-difference steps (Sim.py:49-50) */
} amlp_nep;

/* FFNN, TheEnergyNet (ForceEvaluator.py:6-26) with a selectable activation.
 * Layer k maps dims[k] -> dims[k+1]; dims[0] = D, dims[n_layers] = 1.
 * d_w: all layers packed in FP32, per layer W (dims[k+1] x dims[k], row-major as
 * torch.nn.Linear.weight) followed by b (dims[k+1]). */
typedef struct amlp_mlp {
    int n_layers;
    int dims[AMLP_MAX_LAYERS + 1];
    int act;
    const float *d_w;
} amlp_mlp;

/* Device-resident NVT thermostat state (Sim.setkT, Sim.py:99-111), updated in place. */
typedef struct amlp_thermostat {
    float xi, eta;            /* integrator_vars0, integrator_vars1 */
    float xi_rot, eta_rot;    /* integrator_vars2, integrator_vars3 */
    float thermo_fac;         /* m_exp_thermo_fac */
    float pad[3];
    double ke_t, ke_r;        /* kinetic energies read by the next step two */
    double pe;                /* sum of pair energies of the last force pass */
} amlp_thermostat;

typedef struct amlp_nvt {
    float dt, tau, kT;        /* tau = 100 dt in the reference (Sim.py:115) */
    float n_dof, rn_dof;      /* (N-1)*3 and 3N (Sim.py:35-36) */
    float moi[3];             /* principal moments shared by all bodies */
    float box;                /* cubic box edge L */
    int nve;                  /* 1: no thermostat (thermo_fac = 1, xi_rot = 0) */
} amlp_nvt;

/* One system of a multi-system launch (serving): systems own contiguous body
 * ranges; the per-body int32 array `rep` gives each body's system. A body with
 * rep < 0 is a free slot that every multi-system kernel skips, and a system
 * with n_dof = 0 is a free system slot (its thermostat is left alone), so that
 * buffers of a fixed capacity (and CUDA graphs over them) can serve a changing
 * set of systems. */
typedef struct amlp_replica {
    float kT, n_dof, rn_dof, box;
    int nve;
    int pad[3];
} amlp_replica;

/* --------------------------------------------------------------- library */
int amlp_version(void);
const char *amlp_status_string(amlp_status s);
const char *amlp_last_cuda_error(void);
/* Measurement utility (no reference counterpart): launches a kernel of
 * independent FP32 multiply-add chains on every SM and returns in *flops the
 * floating-point operations it performs (2 per multiply-add), for timing with
 * events around it on the same stream: the measured FP32 peak that the FP32
 * roofline of the force kernels divides by. d_out: one float, never written in
 * practice. */
amlp_status amlp_fp32_fma_probe(float *d_out, int iters, double *flops, void *stream);

/* --------------------------------------------------------------- Verlet list
 * All pairs i < j with |x_i - x_j|_periodic <= r, computed exactly as scipy's
 * cKDTree.query_pairs does for the reference: FP64 distances of
 * float32(pos + L/2) in a periodic box of edge float32(L + 1e-4), folded once
 * per axis, squared components summed x, y, z, compared inclusively with r*r.
 * Output sorted by (i, j). *d_count receives the number of pairs even when it
 * exceeds cap; nothing past cap is written, so a caller that finds
 * *d_count > cap grows the buffer and calls again. */
amlp_status amlp_nlist_workspace_bytes(int n, float box, double r, size_t *bytes);
amlp_status amlp_nlist_build(const float *d_pos, int n, float box, double r,
                             int *d_pairs, long long cap, long long *d_count,
                             void *d_ws, size_t ws_bytes, void *stream);

/* Same list, for callers that cannot allocate device memory at all (not even a
 * workspace), e.g. plug-ins of a host program that owns every GPU buffer under
 * a fixed memory budget. No reference counterpart. Scratch is a fixed array
 * inside the library (13 MiB per GPU, held until exit); n is limited to
 * 262,144 bodies (AMLP_ERR_TOO_LARGE beyond). The first call on a device looks
 * up the array's device address and should come before any stream capture.
 * The address is kept for the life of the process: it assumes the device's
 * one primary context throughout, so after cudaDeviceReset this entry point
 * must not be called again. Calls share the array, so calls that overlap on
 * the GPU race. */
amlp_status amlp_nlist_build_noalloc(const float *d_pos, int n, float box, double r,
                                     int *d_pairs, long long cap, long long *d_count, void *stream);

/* Displacement-triggered rebuilds (no reference counterpart: the reference
 * rebuilds every 100 steps, Sim.py:87, :218-221).
 *   amlp_nlist_check_displacement: d_gate[0] = 1 when some body has moved
 *     farther than max_disp (minimum image in the box) from d_ref, else 0.
 *     With max_disp = skin / 2 no pair within the cutoff can be missing from
 *     a list built with radius cutoff + skin.
 *   amlp_nlist_build_gated: amlp_nlist_build when d_gate[0] != 0 (it then also
 *     copies d_pos to d_ref, adds 1 to d_gate[1] and sets d_gate[2] = 1 if the
 *     list had more than cap pairs); nothing otherwise. Both take the same
 *     launches whatever the flag, so a CUDA graph can hold them in every step.
 *     d_gate: three ints in device memory; d_gate[1] and d_gate[2] are only
 *     ever raised by the library (the caller clears them). */
amlp_status amlp_nlist_check_displacement(const float *d_pos, const float *d_ref, int n, float box,
                                          float max_disp, int *d_gate, void *stream);
amlp_status amlp_nlist_build_gated(const float *d_pos, int n, float box, double r, int *d_pairs,
                                   long long cap, long long *d_count, void *d_ws, size_t ws_bytes,
                                   int *d_gate, float *d_ref, void *stream);

/* --------------------------------------------------------------- pair filter
 * Minimum image (FP32, box L) and |t| < cutoff on the Verlet pairs, kept in
 * Verlet order. The count is read from d_nverlet on the device. */
amlp_status amlp_filter_workspace_bytes(long long cap_verlet, size_t *bytes);
amlp_status amlp_pair_filter(const float *d_pos, float box, double cutoff,
                             const int *d_vpairs, const long long *d_nverlet, long long cap_verlet,
                             int *d_pairs, long long *d_npairs,
                             void *d_ws, size_t ws_bytes, void *stream);

/* --------------------------------------------------------------- descriptors
 * g_all of the reference: row v*P + p holds the D descriptors of
 * finite-difference variant v (0..9) of filtered pair p (P pairs, host value). */
amlp_status amlp_descriptors(const float *d_pos, const float *d_quat, float box,
                             const int *d_pairs, long long P, const amlp_nep *nep,
                             float *d_g, void *stream);

/* Net energies of `rows` descriptor rows: d_e[r] = net(d_g[r]) (the net output
 * y, before the en_min/en_max map). FP32 throughout. */
amlp_status amlp_mlp_energy(const float *d_g, long long rows, const amlp_mlp *mlp,
                            float *d_e, void *stream);

/* Gradient of the training loss L = (1/rows) sum_r (net(d_g[r]) - d_y[r])^2
 * (torch.nn.MSELoss of 05/FFNN.py:95-106; d_y holds the normalised energies of
 * 05/FFNN.py:59-63) with respect to every weight and bias of the net, in the
 * packed layout of amlp_mlp.d_w (per layer W (out x in) then b). d_grad is
 * accumulated into (zero it first); d_loss (may be NULL) accumulates L in FP64.
 * FP32, layer widths up to 256. */
amlp_status amlp_mlp_loss_grad(const float *d_g, const float *d_y, long long rows, const amlp_mlp *mlp,
                               float *d_grad, double *d_loss, void *stream);

/* Finite differences, scaling, clip to [-100,100] and scatter of
 * ForceEvaluator.py:86-146. d_F, d_T (N,3) are accumulated into (zero them
 * first). d_pe (may be NULL) accumulates sum_p (en_min + (en_max-en_min) e0_p). */
amlp_status amlp_fd_scatter(const float *d_e, long long P, const int *d_pairs, const amlp_nep *nep,
                            float *d_F, float *d_T, double *d_pe, void *stream);

/* --------------------------------------------------------------- fused force passes
 * Plain path: per filtered pair the 10 finite-difference variants, descriptors,
 * FP32 net, differences, clip and scatter in one kernel; g_all never reaches
 * HBM. The pair count is read on the device (d_npairs). Nets wider than 64
 * return AMLP_ERR_UNSUPPORTED (use the three calls above). */
amlp_status amlp_forces_fd(const float *d_pos, const float *d_quat, float box,
                           const int *d_pairs, const long long *d_npairs, long long cap,
                           const amlp_nep *nep, const amlp_mlp *mlp,
                           float *d_F, float *d_T, double *d_pe, void *stream);

/* amlp_forces_fd that also writes the net output of every finite-difference
 * variant, d_e[v * P + p] for variant v = 0..9 of filtered pair p
 * (P = min(*d_npairs, cap); d_e holds 10 cap floats): the e_all of
 * ForceEvaluator.evaluate_gradients (ForceEvaluator.py:80-96), for checking
 * the fused kernel's energies row by row. */
amlp_status amlp_forces_fd_energies(const float *d_pos, const float *d_quat, float box,
                                    const int *d_pairs, const long long *d_npairs, long long cap,
                                    const amlp_nep *nep, const amlp_mlp *mlp,
                                    float *d_F, float *d_T, double *d_pe, float *d_e, void *stream);

/* Adjoint path: one descriptor evaluation per pair and the exact derivative of
 * the pair energy with respect to the translation of body i and the rotations
 * of bodies i and j; the same scaling, clip and scatter as the plain path. */
amlp_status amlp_forces_adjoint(const float *d_pos, const float *d_quat, float box,
                                const int *d_pairs, const long long *d_npairs, long long cap,
                                const amlp_nep *nep, const amlp_mlp *mlp,
                                float *d_F, float *d_T, double *d_pe, void *stream);

/* Same forces for nets with hidden widths up to 128 (amlp_forces_adjoint takes
 * widths up to 64): the descriptor forward, the net forward/backward on the
 * tensor cores (weights staged layer by layer) and the descriptor backward run
 * as three kernels that pass g, dE/dg and the net output through a workspace
 * of amlp_adjoint_workspace_bytes(cap). */
amlp_status amlp_adjoint_workspace_bytes(long long cap, size_t *bytes);
amlp_status amlp_forces_adjoint_wide(const float *d_pos, const float *d_quat, float box,
                                     const int *d_pairs, const long long *d_npairs, long long cap,
                                     const amlp_nep *nep, const amlp_mlp *mlp,
                                     float *d_F, float *d_T, double *d_pe, void *d_ws, size_t ws_bytes, void *stream);

/* ------------------------------------------------- differentiation (no reference counterpart)
 * The pieces of a torch.autograd.Function over the pair energies
 * E_p = en_min + (en_max - en_min) net(g_p):
 *   amlp_pair_descriptors  g_p of the unperturbed pair (row p at d_g + p*ld_g,
 *                          ld_g >= D, columns D..ld_g-1 set to zero);
 *   amlp_pair_energy_vjp   F = -sum_p w_p dE_p/dx, T = -sum_p w_p dE_p/dtheta
 *                          (world-frame rotation about each body's centre),
 *                          accumulated into d_F, d_T; w_p = d_wt[p] (NULL: 1);
 *                          clip = 1 clips each pair's terms to [-100,100] as the
 *                          force path does, clip = 0 gives the exact product.
 *                          Same kernels and workspace as amlp_forces_adjoint_wide;
 *   amlp_mlp_backward      d_grad += sum_r d_dy[r] d net(d_g[r]) / d theta over
 *                          every weight and bias (packed like amlp_mlp.d_w). */
amlp_status amlp_pair_descriptors(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                  const long long *d_npairs, long long cap, const amlp_nep *nep,
                                  float *d_g, int ld_g, void *stream);
amlp_status amlp_pair_energy_vjp(const float *d_pos, const float *d_quat, float box, const int *d_pairs,
                                 const long long *d_npairs, long long cap, const amlp_nep *nep,
                                 const amlp_mlp *mlp, const float *d_wt, int clip, float *d_F, float *d_T,
                                 double *d_pe, void *d_ws, size_t ws_bytes, void *stream);
amlp_status amlp_mlp_backward(const float *d_g, const float *d_dy, long long rows, const amlp_mlp *mlp,
                              float *d_grad, void *stream);

/* Sticky error bits raised by device code since the last clear (1 = a bounded
 * wait for tensor-core completion gave up; the kernel then stops early). */
amlp_status amlp_device_error(unsigned int *flags, int clear);

/* Test hook (no reference counterpart): the number of polls allowed to the
 * first tensor-core completion wait of every CTA of amlp_forces_adjoint's
 * kernel, so that a test can make that wait give up without a fault: with 0 it
 * gives up at once, the kernel raises bit 1 of amlp_device_error, issues no
 * further MMA, drains the one in flight (normal limit) and frees its tensor
 * memory. -1 restores the normal limit. It applies to later launches. */
amlp_status amlp_test_first_wait_limit(int polls);

/* Stage timing (no reference counterpart): with enable = 1, every later
 * amlp_forces_adjoint_wide / amlp_pair_energy_vjp call records CUDA events on
 * its stream around its three stages: descriptor forward, net forward and
 * backward (k_mlp_grad, with the weight split), descriptor backward. Not for
 * calls captured into a CUDA graph. amlp_stage_times waits for the last such
 * call's events and writes the three durations in milliseconds. */
amlp_status amlp_stage_timing(int enable);
amlp_status amlp_stage_times(float *h_ms3);

/* --------------------------------------------------------------- NVT integrator
 * d_th: one amlp_thermostat in device memory.
 * init: kinetic energies before the first step. With initial_ke_quirk = 1 the
 * translational value is body 0's kinetic energy only, as the reference passes
 * its per-body array to update_variables (Sim.py:157, IntegrateStepTwoKernels.py:245). */
amlp_status amlp_nvt_init(const float *d_vel, const float *d_quat, const float *d_angmom,
                          const float *d_mass, int n, const amlp_nvt *prm, int initial_ke_quirk,
                          amlp_thermostat *d_th, void *d_ws, size_t ws_bytes, void *stream);
amlp_status amlp_nvt_workspace_bytes(int n, size_t *bytes);
/* Step two: thermostat update, v <- v f + dt/2 F/m, angular-momentum kick.
 * Writes d_accel (N,3) and d_dp (N,4) for step one. */
amlp_status amlp_nvt_step_two(float *d_vel, float *d_accel, const float *d_F, const float *d_mass,
                              const float *d_quat, const float *d_T, float *d_angmom, float *d_dp,
                              int n, const amlp_nvt *prm, amlp_thermostat *d_th, void *stream);
/* Step one: translation (kick, drift, one periodic wrap), rotation (kick +
 * free-rotor splitting + renormalisation) and the FP64 kinetic-energy sums. */
amlp_status amlp_nvt_step_one(float *d_pos, float *d_vel, const float *d_accel,
                              float *d_quat, float *d_angmom, const float *d_dp, const float *d_mass,
                              int n, const amlp_nvt *prm, amlp_thermostat *d_th,
                              void *d_ws, size_t ws_bytes, void *stream);

/* --------------------------------------------------------------- many systems in one launch
 * Serving path: the bodies of independent systems (different sizes, boxes,
 * temperatures; one shape and one net per call) are concatenated, pair lists
 * hold global body indices, and every kernel looks up the body's system.
 * No reference counterpart (the reference runs one system per process).
 * d_rp: nrep amlp_replica; d_th: nrep amlp_thermostat; d_pe: nrep doubles. */
amlp_status amlp_multi_pair_filter(const float *d_pos, const int *d_rep, const amlp_replica *d_rp, double cutoff,
                                   const int *d_vpairs, const long long *d_nverlet, long long cap_verlet,
                                   int *d_pairs, long long *d_npairs, void *d_ws, size_t ws_bytes, void *stream);
amlp_status amlp_multi_forces_adjoint(const float *d_pos, const float *d_quat, const int *d_rep,
                                      const amlp_replica *d_rp, const int *d_pairs, const long long *d_npairs,
                                      long long cap, const amlp_nep *nep, const amlp_mlp *mlp,
                                      float *d_F, float *d_T, double *d_pe, void *stream);
amlp_status amlp_multi_forces_adjoint_wide(const float *d_pos, const float *d_quat, const int *d_rep,
                                           const amlp_replica *d_rp, const int *d_pairs, const long long *d_npairs,
                                           long long cap, const amlp_nep *nep, const amlp_mlp *mlp,
                                           float *d_F, float *d_T, double *d_pe, void *d_ws, size_t ws_bytes,
                                           void *stream);
/* prm supplies dt, tau and moi shared by the systems; the rest is per system. */
amlp_status amlp_multi_nvt_init(const float *d_vel, const float *d_quat, const float *d_angmom, const float *d_mass,
                                const int *d_rep, int n, int nrep, const amlp_nvt *prm, amlp_thermostat *d_th,
                                void *stream);
amlp_status amlp_multi_nvt_step_two(float *d_vel, float *d_accel, const float *d_F, const float *d_mass,
                                    const float *d_quat, const float *d_T, float *d_angmom, float *d_dp,
                                    const int *d_rep, int n, int nrep, const amlp_replica *d_rp, const amlp_nvt *prm,
                                    amlp_thermostat *d_th, void *stream);
amlp_status amlp_multi_nvt_step_one(float *d_pos, float *d_vel, const float *d_accel, float *d_quat,
                                    float *d_angmom, const float *d_dp, const float *d_mass, const int *d_rep, int n,
                                    const amlp_replica *d_rp, const amlp_nvt *prm, amlp_thermostat *d_th,
                                    void *stream);

/* --------------------------------------------------------------- simulation handles
 * A handle owns one system's device state and buffers and runs the reference's
 * step (Sim.step, Sim.py:257-285) through the calls above. It rebuilds the
 * Verlet list every nlist_every steps (Sim.py:87, :218-221) and replays the
 * steps in between as one CUDA graph. Reference interfaces replaced:
 *   amlp_create / amlp_destroy   Sim.__init__ + setDevice + setNepDescriptors + setkT + setdt
 *                                Sim.py:14-25, :67-74, :99-116
 *   amlp_set_state               initializeSystem + move_data_to_device   Sim.py:27-51, :147-169
 *   amlp_set_shape               setShape   Sim.py:76-83, DescriptorGenerator.py:58-125
 *   amlp_set_model               setEvaluator (weights already on the device)   Sim.py:53-65
 *   amlp_build_nlist             setNeighborList / refreshNList   Sim.py:85-92, :192-198
 *   amlp_sim_descriptors         DescriptorGenerator.generate_nep_descriptors   DescriptorGenerator.py:136-161
 *                                (named apart from the stateless amlp_descriptors above)
 *   amlp_forces                  descriptors + ForceEvaluator.evaluate_interactions   Sim.py:261-266
 *   amlp_step                    Sim.run   Sim.py:207-255
 *   amlp_get_state, amlp_get_thermostat   the arrays and integrator variables Sim.dumpConfig writes
 *                                Sim.py:117-145
 * Order: create, then set_shape, set_model and set_state (any order), then
 * the rest. set_state resets the time step to 0 and computes the initial
 * kinetic energies (amlp_nvt_init). A handle is used from one host thread at a
 * time; its work is ordered on the stream each call gets, and calls that read
 * a count back (build_nlist, sim_descriptors, step when it rebuilds)
 * synchronise that stream. d_* arguments are device memory, copied in or out. */
typedef struct amlp_sim amlp_sim;

typedef struct amlp_sim_config {
    int n;                    /* bodies */
    int nrad, nang, lmax;     /* descriptor hypers (setNepDescriptors) */
    float kT, dt;             /* setkT, setdt */
    float tau;                /* thermostat time constant; <= 0: float(100 dt) as Sim.py:115 */
    int nve;                  /* 1: no thermostat */
    int initial_ke_quirk;     /* 1: the reference's first-step kinetic energy (amlp_nvt_init) */
    int nlist_every;          /* Verlet rebuild period; <= 0: 100 */
    double skin;              /* Verlet radius = cutoff + skin; <= 0: 2.0 (Sim.py:86) */
    float dx, dteta;          /* finite-difference steps; <= 0: 1e-5 (Sim.py:49-50) */
} amlp_sim_config;

#define AMLP_FORCES_FD 0          /* the reference's finite differences (amlp_forces_fd) */
#define AMLP_FORCES_ADJOINT 1     /* analytic forces (amlp_forces_adjoint / _wide by net width) */

amlp_status amlp_create(const amlp_sim_config *cfg, amlp_sim **out);
void amlp_destroy(amlp_sim *h);
/* h_pts: host (npts,3) body-frame points. */
amlp_status amlp_set_shape(amlp_sim *h, const float *h_pts, int npts, float en_min, float en_max,
                           double cutoff, float nep_cutoff);
/* mlp->d_w (device) is copied; dims[0] must equal the descriptor length. */
amlp_status amlp_set_model(amlp_sim *h, const amlp_mlp *mlp, void *stream);
/* h_moi: host, 3 principal moments shared by the bodies. */
amlp_status amlp_set_state(amlp_sim *h, const float *d_pos, const float *d_quat, const float *d_vel,
                           const float *d_angmom, const float *d_mass, const float *h_moi, float box,
                           void *stream);
amlp_status amlp_build_nlist(amlp_sim *h, void *stream);
/* Filters the pairs and writes g_all (10 P rows of D, amlp_descriptors'
 * layout) to d_g and the filtered pairs to d_pairs (P x 2 int32); *h_P gets P.
 * With P > cap nothing is written and AMLP_ERR_CAPACITY is returned. */
amlp_status amlp_sim_descriptors(amlp_sim *h, float *d_g, int *d_pairs, long long cap, long long *h_P,
                                 void *stream);
/* One force pass (filter, forces, torques, pair-energy sum) on the current
 * state; d_F, d_T (N,3) receive copies when not NULL. */
amlp_status amlp_forces(amlp_sim *h, float *d_F, float *d_T, int mode, void *stream);
/* Returns AMLP_ERR_DEVICE_WAIT when, at one of its synchronisations (the
 * Verlet rebuilds), a bounded device-side wait has given up since the flags
 * were last cleared with amlp_device_error. */
amlp_status amlp_step(amlp_sim *h, int nsteps, int mode, void *stream);
/* Any of the outputs may be NULL. */
amlp_status amlp_get_state(amlp_sim *h, float *d_pos, float *d_quat, float *d_vel, float *d_angmom,
                           void *stream);
amlp_status amlp_get_thermostat(amlp_sim *h, amlp_thermostat *h_th, void *stream);
long long amlp_timestep(const amlp_sim *h);
/* Message of the last failed call on h ("" when none). */
const char *amlp_last_error(const amlp_sim *h);

/* --------------------------------------------------------------- serving pool
 * Many independent systems of one shape and one net, resident on one GPU and
 * advanced together. Each pool step runs one launch per stage over every
 * system (amlp_multi_*). No reference counterpart: the reference runs one
 * system per process. Admitted systems join, and evicted ones leave, between
 * segments. A segment rebuilds every system's Verlet list and then replays its
 * steps as one CUDA graph. The status is kept per system. */
typedef struct amlp_pool amlp_pool;

typedef struct amlp_pool_config {
    int nrad, nang, lmax;
    float dt, tau;            /* tau <= 0: float(100 dt) */
    const float *h_pts;       /* host (npts,3) */
    int npts;
    float en_min, en_max;
    double cutoff;
    float nep_cutoff;
    double skin;              /* <= 0: 2.0 */
    const float *h_moi;       /* host, 3 */
    const amlp_mlp *mlp;      /* d_w (device) is copied */
} amlp_pool_config;

typedef struct amlp_pool_system {
    int n;
    float box, kT;
    int nve;
    long long verlet_cap;     /* capacity of its Verlet list; <= 0: 1.5 x the ideal-gas pair
                                 count at radius cutoff + skin, plus 4 n + 1024 */
    /* host arrays, copied: (n,3), (n,4), (n,3), (n,4), (n) */
    const float *h_pos, *h_quat, *h_vel, *h_angmom, *h_mass;
} amlp_pool_system;

/* Per-system status (amlp_pool_system_status). A system whose Verlet list
 * outgrows its capacity gets a larger one at the next segment. */
#define AMLP_POOL_ACTIVE 0          /* packed and stepping */
#define AMLP_POOL_PENDING 1         /* admitted; joins at the next segment */

amlp_status amlp_pool_create(const amlp_pool_config *cfg, amlp_pool **out);
void amlp_pool_destroy(amlp_pool *p);
/* Adds a system (thermostat at the reference's seeds); *id identifies it. */
amlp_status amlp_pool_admit(amlp_pool *p, const amlp_pool_system *sys, int *id);
/* Removes a system, copying its state to the host arrays given (any may be
 * NULL) and its thermostat to *h_th (may be NULL). */
amlp_status amlp_pool_evict(amlp_pool *p, int id, float *h_pos, float *h_quat, float *h_vel, float *h_angmom,
                            amlp_thermostat *h_th);
/* nsteps steps of every active system (adjoint forces). Synchronises the stream;
 * AMLP_ERR_DEVICE_WAIT as for amlp_step. */
amlp_status amlp_pool_step_segment(amlp_pool *p, int nsteps, void *stream);
amlp_status amlp_pool_system_status(amlp_pool *p, int id, int *status, long long *steps_done,
                                    amlp_thermostat *h_th);
int amlp_pool_size(const amlp_pool *p);
const char *amlp_pool_last_error(const amlp_pool *p);

#ifdef __cplusplus
}
#endif
#endif /* AMLP_H */
