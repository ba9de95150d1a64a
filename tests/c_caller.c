/* A plain C caller of libamlp's simulation handle (include/amlp.h): the
 * integration a host program written in C would do. Used by
 * tests/test_c_caller.py.
 *
 *   c_caller <in.bin> <out.bin> <nsteps> <mode>
 *
 * in.bin (little-endian): int32 n, npts, n_layers; float32 box, kT, dt,
 * en_min, en_max, cutoff, nep_cutoff, moi[3]; int32 dims[n_layers + 1], act;
 * float32 pts[npts*3], pos[n*3], quat[n*4], vel[n*3], angmom[n*4], mass[n],
 * weights (packed as amlp_mlp.d_w).
 * out.bin: float32 pos[n*3], quat[n*4], vel[n*3], angmom[n*4]; float64 xi,
 * eta, pe (the thermostat after the run). Exit status 0 on success.
 */
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "amlp.h"

static int rd(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes ? 0 : -1; }

static void *dev_copy(const void *h, size_t bytes) {
    void *d = NULL;
    if (cudaMalloc(&d, bytes) != cudaSuccess) return NULL;
    if (cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return NULL;
    return d;
}

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s in.bin out.bin nsteps mode\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int n, npts, nl;
    float box, kT, dt, en_min, en_max, cutoff, nep_cutoff, moi[3];
    if (rd(f, &n, 4) || rd(f, &npts, 4) || rd(f, &nl, 4) || rd(f, &box, 4) || rd(f, &kT, 4) || rd(f, &dt, 4) ||
        rd(f, &en_min, 4) || rd(f, &en_max, 4) || rd(f, &cutoff, 4) || rd(f, &nep_cutoff, 4) || rd(f, moi, 12))
        return 3;
    amlp_mlp mlp = {0};
    mlp.n_layers = nl;
    if (nl < 1 || nl > AMLP_MAX_LAYERS || rd(f, mlp.dims, 4 * (nl + 1)) || rd(f, &mlp.act, 4)) return 3;
    long long nw = 0;
    for (int k = 0; k < nl; ++k) nw += (long long)mlp.dims[k + 1] * (mlp.dims[k] + 1);
    size_t sz[7] = {(size_t)npts * 3, (size_t)n * 3, (size_t)n * 4, (size_t)n * 3, (size_t)n * 4, (size_t)n,
                    (size_t)nw};
    float *h[7];
    for (int k = 0; k < 7; ++k) {
        h[k] = (float *)malloc(sz[k] * 4);
        if (!h[k] || rd(f, h[k], sz[k] * 4)) return 3;
    }
    fclose(f);
    float *d_pos = dev_copy(h[1], sz[1] * 4), *d_quat = dev_copy(h[2], sz[2] * 4);
    float *d_vel = dev_copy(h[3], sz[3] * 4), *d_ang = dev_copy(h[4], sz[4] * 4);
    float *d_mass = dev_copy(h[5], sz[5] * 4), *d_w = dev_copy(h[6], sz[6] * 4);
    if (!d_pos || !d_quat || !d_vel || !d_ang || !d_mass || !d_w) return 4;
    mlp.d_w = d_w;

    amlp_sim_config cfg = {0};
    cfg.n = n;
    cfg.nrad = 10;
    cfg.nang = 8;
    cfg.lmax = 4;
    cfg.kT = kT;
    cfg.dt = dt;
    amlp_sim *sim = NULL;
    amlp_status st = amlp_create(&cfg, &sim);
    if (st == AMLP_OK) st = amlp_set_shape(sim, h[0], npts, en_min, en_max, cutoff, nep_cutoff);
    if (st == AMLP_OK) st = amlp_set_model(sim, &mlp, NULL);
    if (st == AMLP_OK) st = amlp_set_state(sim, d_pos, d_quat, d_vel, d_ang, d_mass, moi, box, NULL);
    if (st == AMLP_OK) st = amlp_step(sim, atoi(argv[3]), atoi(argv[4]), NULL);
    if (st == AMLP_OK) st = amlp_get_state(sim, d_pos, d_quat, d_vel, d_ang, NULL);
    amlp_thermostat th;
    if (st == AMLP_OK) st = amlp_get_thermostat(sim, &th, NULL);
    if (st != AMLP_OK) {
        fprintf(stderr, "amlp: %s (%s)\n", amlp_status_string(st), sim ? amlp_last_error(sim) : "");
        return 5;
    }
    FILE *o = fopen(argv[2], "wb");
    if (!o) return 6;
    float *dsrc[4] = {d_pos, d_quat, d_vel, d_ang};
    for (int k = 0; k < 4; ++k) {
        if (cudaMemcpy(h[1 + k], dsrc[k], sz[1 + k] * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 6;
        fwrite(h[1 + k], 4, sz[1 + k], o);
    }
    double tv[3] = {th.xi, th.eta, th.pe};
    fwrite(tv, 8, 3, o);
    fclose(o);
    printf("ok %lld steps\n", amlp_timestep(sim));
    amlp_destroy(sim);
    return 0;
}
