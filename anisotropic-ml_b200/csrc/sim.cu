// Simulation handles (amlp_sim) and the serving pool (amlp_pool): host-side
// runtimes that own device buffers and sequence the stateless entry points of
// this library into the reference's time step (Sim.step, Sim.py:257-285):
// pair filter, force pass, NVT step two, NVT step one, with the Verlet list
// rebuilt every nlist_every steps (Sim.py:87, :218-221). The steps between two
// rebuilds are captured once as a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

using namespace amlp;

// Thermostat seeds of Sim.setkT (Sim.py:101-105).
constexpr float kSeedXi = -0.0317711f, kSeedEta = 0.108609f, kSeedXiRot = 0.00814227f, kSeedEtaRot = -0.014238f,
                kSeedFac = 1.00011f;

// One owning device allocation, grown on demand (contents are not kept).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t b) {
        if (b == 0) b = 16;
        if (b <= bytes) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

amlp_thermostat seeded_thermostat(int nve) {
    amlp_thermostat t;
    std::memset(&t, 0, sizeof(t));
    if (nve) {
        t.thermo_fac = 1.0f;
    } else {
        t.xi = kSeedXi;
        t.eta = kSeedEta;
        t.xi_rot = kSeedXiRot;
        t.eta_rot = kSeedEtaRot;
        t.thermo_fac = kSeedFac;
    }
    return t;
}

int descriptor_length(int nrad, int nang, int lmax) { return (nrad + 1) + (nang + 1) * lmax; }

long long packed_weight_count(const amlp_mlp &m) {
    long long c = 0;
    for (int k = 0; k < m.n_layers; ++k) c += (long long)m.dims[k + 1] * (m.dims[k] + 1);
    return c;
}

int max_hidden_width(const amlp_mlp &m) {
    int w = 0;
    for (int k = 1; k < m.n_layers; ++k) w = m.dims[k] > w ? m.dims[k] : w;
    return w;
}

// A graph of `seg` steps, valid while the buffers it captured stay in place.
struct StepGraph {
    int mode = -1, seg = 0;
    long long cap = -1;
    cudaGraphExec_t exec = nullptr;
};

void destroy_graphs(std::vector<StepGraph> &gs) {
    for (auto &g : gs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    gs.clear();
}

// Captures `seg` calls of enqueue(stream) on a private stream. The library's
// launches set their kernel attributes on the first call, so the caller runs
// one step eagerly (on a snapshot) before the first capture.
template <class F>
cudaError_t capture_steps(cudaStream_t cs, int seg, F &&enqueue, amlp_status &st, cudaGraphExec_t *exec) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    st = AMLP_OK;
    for (int k = 0; k < seg && st == AMLP_OK; ++k) st = enqueue(cs);
    e = cudaStreamEndCapture(cs, &graph);
    if (st != AMLP_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return e;
    }
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    return e;
}

// Pairs of one system's Verlet list (local body indices) appended to the
// pool's list with the system's first body added.
__global__ void k_offset_pairs(const int *src, int *dst, long long count, int first) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < 2 * count;
         k += (long long)gridDim.x * blockDim.x)
        dst[k] = src[k] + first;
}

}  // namespace

// ------------------------------------------------------------------ amlp_sim

struct amlp_sim {
    amlp_sim_config cfg{};
    int n = 0, D = 0;
    DevBuf pos, quat, vel, angmom, mass, accel, dp, F, T, th, nvt_ws, nl_ws, pts, w, nv, nf, vpairs, fpairs, f_ws,
        adj_ws, snap;
    bool have_state = false, have_shape = false, have_model = false, list_valid = false;
    amlp_nep nep{};
    amlp_mlp mlp{};
    amlp_nvt nvt{};
    double r_verlet = 0.0;
    long long cap = 0, timestep = 0;
    cudaStream_t cs = nullptr;  // capture stream
    std::vector<StepGraph> graphs;
    std::string err;

    amlp_status fail(amlp_status s, const std::string &msg) {
        err = msg;
        return s;
    }
    amlp_status cuda(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return AMLP_OK;
        set_cuda_error(e);
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return AMLP_ERR_CUDA;
    }
    amlp_status lib(amlp_status s, const char *what) {
        if (s != AMLP_OK) err = std::string(what) + ": " + amlp_status_string(s);
        return s;
    }
    amlp_status ready() {
        if (!have_shape) return fail(AMLP_ERR_INVALID_ARG, "no shape (amlp_set_shape)");
        if (!have_model) return fail(AMLP_ERR_INVALID_ARG, "no model (amlp_set_model)");
        if (!have_state) return fail(AMLP_ERR_INVALID_ARG, "no state (amlp_set_state)");
        return AMLP_OK;
    }
    double *pe() { return reinterpret_cast<double *>(th.as<char>() + offsetof(amlp_thermostat, pe)); }

    amlp_status alloc_pairs(long long c) {
        destroy_graphs(graphs);
        cap = c;
        size_t fb = 0, ab = 0;
        amlp_filter_workspace_bytes(cap, &fb);
        amlp_status s;
        if ((s = cuda(vpairs.ensure((size_t)cap * 2 * sizeof(int)), "pair list"))) return s;
        if ((s = cuda(fpairs.ensure((size_t)cap * 2 * sizeof(int)), "filtered pairs"))) return s;
        if ((s = cuda(f_ws.ensure(fb), "filter workspace"))) return s;
        if (max_hidden_width(mlp) > 64) {
            amlp_adjoint_workspace_bytes(cap, &ab);
            if ((s = cuda(adj_ws.ensure(ab), "adjoint workspace"))) return s;
        }
        return AMLP_OK;
    }

    amlp_status build_nlist(cudaStream_t st) {
        size_t wb = 0;
        amlp_status s = lib(amlp_nlist_workspace_bytes(n, nvt.box, r_verlet, &wb), "amlp_nlist_workspace_bytes");
        if (s) return s;
        if ((s = cuda(nl_ws.ensure(wb), "Verlet workspace"))) return s;
        if (cap == 0 && (s = alloc_pairs(1024))) return s;
        for (;;) {
            s = amlp_nlist_build(pos.as<float>(), n, nvt.box, r_verlet, vpairs.as<int>(), cap, nv.as<long long>(),
                                 nl_ws.p, nl_ws.bytes, st);
            if (s) return lib(s, "amlp_nlist_build");
            long long count = 0;
            if ((s = cuda(cudaMemcpyAsync(&count, nv.p, sizeof(count), cudaMemcpyDeviceToHost, st), "pair count")))
                return s;
            if ((s = cuda(cudaStreamSynchronize(st), "pair count"))) return s;
            if (count <= cap) break;
            if ((s = alloc_pairs(count + count / 4 + 1024))) return s;
        }
        list_valid = true;
        return AMLP_OK;
    }

    amlp_status enqueue_forces(int mode, cudaStream_t st) {
        amlp_status s;
        if ((s = cuda(cudaMemsetAsync(F.p, 0, (size_t)n * 3 * sizeof(float), st), "zero F"))) return s;
        if ((s = cuda(cudaMemsetAsync(T.p, 0, (size_t)n * 3 * sizeof(float), st), "zero T"))) return s;
        if ((s = cuda(cudaMemsetAsync(pe(), 0, sizeof(double), st), "zero pe"))) return s;
        s = amlp_pair_filter(pos.as<float>(), nvt.box, nep.cutoff, vpairs.as<int>(), nv.as<long long>(), cap,
                             fpairs.as<int>(), nf.as<long long>(), f_ws.p, f_ws.bytes, st);
        if (s) return lib(s, "amlp_pair_filter");
        if (mode == AMLP_FORCES_FD) {
            s = amlp_forces_fd(pos.as<float>(), quat.as<float>(), nvt.box, fpairs.as<int>(), nf.as<long long>(), cap,
                               &nep, &mlp, F.as<float>(), T.as<float>(), pe(), st);
            return lib(s, "amlp_forces_fd");
        }
        if (mode != AMLP_FORCES_ADJOINT) return fail(AMLP_ERR_INVALID_ARG, "unknown force mode");
        if (max_hidden_width(mlp) > 64)
            s = amlp_forces_adjoint_wide(pos.as<float>(), quat.as<float>(), nvt.box, fpairs.as<int>(),
                                         nf.as<long long>(), cap, &nep, &mlp, F.as<float>(), T.as<float>(), pe(),
                                         adj_ws.p, adj_ws.bytes, st);
        else
            s = amlp_forces_adjoint(pos.as<float>(), quat.as<float>(), nvt.box, fpairs.as<int>(), nf.as<long long>(),
                                    cap, &nep, &mlp, F.as<float>(), T.as<float>(), pe(), st);
        return lib(s, "amlp_forces_adjoint");
    }

    amlp_status enqueue_step(int mode, cudaStream_t st) {
        amlp_status s = enqueue_forces(mode, st);
        if (s) return s;
        s = amlp_nvt_step_two(vel.as<float>(), accel.as<float>(), F.as<float>(), mass.as<float>(), quat.as<float>(),
                              T.as<float>(), angmom.as<float>(), dp.as<float>(), n, &nvt, th.as<amlp_thermostat>(), st);
        if (s) return lib(s, "amlp_nvt_step_two");
        s = amlp_nvt_step_one(pos.as<float>(), vel.as<float>(), accel.as<float>(), quat.as<float>(),
                              angmom.as<float>(), dp.as<float>(), mass.as<float>(), n, &nvt, th.as<amlp_thermostat>(),
                              nvt_ws.p, nvt_ws.bytes, st);
        return lib(s, "amlp_nvt_step_one");
    }

    // The state a step changes, saved and restored around the eager warm-up step.
    struct Piece {
        DevBuf *b;
        size_t bytes;
    };
    std::vector<Piece> pieces() {
        return {{&pos, (size_t)n * 12}, {&quat, (size_t)n * 16}, {&vel, (size_t)n * 12}, {&angmom, (size_t)n * 16},
                {&accel, (size_t)n * 12}, {&dp, (size_t)n * 16}, {&th, sizeof(amlp_thermostat)}};
    }
    amlp_status save_restore(bool save, cudaStream_t st) {
        size_t total = 0;
        for (auto &pc : pieces()) total += align_up(pc.bytes);
        amlp_status s;
        if (save && (s = cuda(snap.ensure(total), "snapshot"))) return s;
        size_t off = 0;
        for (auto &pc : pieces()) {
            char *sp = snap.as<char>() + off;
            cudaError_t e = save ? cudaMemcpyAsync(sp, pc.b->p, pc.bytes, cudaMemcpyDeviceToDevice, st)
                                 : cudaMemcpyAsync(pc.b->p, sp, pc.bytes, cudaMemcpyDeviceToDevice, st);
            if ((s = cuda(e, "snapshot copy"))) return s;
            off += align_up(pc.bytes);
        }
        return AMLP_OK;
    }

    amlp_status run_segment(int mode, int seg, cudaStream_t st) {
        StepGraph *g = nullptr;
        for (auto &x : graphs)
            if (x.mode == mode && x.seg == seg && x.cap == cap) g = &x;
        amlp_status s;
        if (!g) {
            if ((s = save_restore(true, st)) || (s = enqueue_step(mode, st)) || (s = save_restore(false, st))) return s;
            if ((s = cuda(cudaStreamSynchronize(st), "warm-up step"))) return s;
            StepGraph ng;
            ng.mode = mode;
            ng.seg = seg;
            ng.cap = cap;
            amlp_status es = AMLP_OK;
            cudaError_t e = capture_steps(cs, seg, [&](cudaStream_t c) { return enqueue_step(mode, c); }, es,
                                          &ng.exec);
            if (es) return es;
            if ((s = cuda(e, "graph capture"))) return s;
            graphs.push_back(ng);
            g = &graphs.back();
        }
        return cuda(cudaGraphLaunch(g->exec, st), "graph launch");
    }
};

extern "C" amlp_status amlp_create(const amlp_sim_config *cfg, amlp_sim **out) {
    if (!cfg || !out) return AMLP_ERR_INVALID_ARG;
    *out = nullptr;
    if (cfg->n <= 0 || cfg->dt <= 0.f || cfg->nrad < 0 || cfg->nang < 0 || cfg->lmax < 1)
        return AMLP_ERR_INVALID_ARG;
    amlp_sim *h = new amlp_sim();
    h->cfg = *cfg;
    if (h->cfg.nlist_every <= 0) h->cfg.nlist_every = 100;
    if (h->cfg.skin <= 0.0) h->cfg.skin = 2.0;
    if (h->cfg.dx <= 0.f) h->cfg.dx = 1e-5f;
    if (h->cfg.dteta <= 0.f) h->cfg.dteta = 1e-5f;
    h->n = cfg->n;
    h->D = descriptor_length(cfg->nrad, cfg->nang, cfg->lmax);
    const size_t n = (size_t)cfg->n;
    size_t nvt_bytes = 0;
    amlp_nvt_workspace_bytes(cfg->n, &nvt_bytes);
    amlp_status s = AMLP_OK;
    DevBuf *bufs[] = {&h->pos, &h->vel, &h->accel, &h->F, &h->T};
    for (DevBuf *b : bufs)
        if (!s) s = h->cuda(b->ensure(n * 3 * sizeof(float)), "state");
    DevBuf *bufs4[] = {&h->quat, &h->angmom, &h->dp};
    for (DevBuf *b : bufs4)
        if (!s) s = h->cuda(b->ensure(n * 4 * sizeof(float)), "state");
    if (!s) s = h->cuda(h->mass.ensure(n * sizeof(float)), "state");
    if (!s) s = h->cuda(h->th.ensure(sizeof(amlp_thermostat)), "thermostat");
    if (!s) s = h->cuda(h->nvt_ws.ensure(nvt_bytes), "integrator workspace");
    if (!s) s = h->cuda(h->nv.ensure(sizeof(long long)), "counts");
    if (!s) s = h->cuda(h->nf.ensure(sizeof(long long)), "counts");
    if (!s) s = h->cuda(cudaStreamCreateWithFlags(&h->cs, cudaStreamNonBlocking), "capture stream");
    if (!s) s = h->cuda(cudaMemset(h->accel.p, 0, n * 3 * sizeof(float)), "state");
    if (!s) s = h->cuda(cudaMemset(h->dp.p, 0, n * 4 * sizeof(float)), "state");
    if (s) {
        amlp_destroy(h);
        return s;
    }
    h->nep.nrad = cfg->nrad;
    h->nep.nang = cfg->nang;
    h->nep.lmax = cfg->lmax;
    h->nep.dx = h->cfg.dx;
    h->nep.dteta = h->cfg.dteta;
    h->nvt.dt = cfg->dt;
    h->nvt.tau = cfg->tau > 0.f ? cfg->tau : (float)(100.0 * (double)cfg->dt);
    h->nvt.kT = cfg->kT;
    h->nvt.n_dof = (float)((cfg->n - 1) * 3);
    h->nvt.rn_dof = (float)(cfg->n * 3);
    h->nvt.nve = cfg->nve ? 1 : 0;
    *out = h;
    return AMLP_OK;
}

extern "C" void amlp_destroy(amlp_sim *h) {
    if (!h) return;
    destroy_graphs(h->graphs);
    DevBuf *all[] = {&h->pos, &h->quat, &h->vel, &h->angmom, &h->mass, &h->accel, &h->dp, &h->F, &h->T, &h->th,
                     &h->nvt_ws, &h->nl_ws, &h->pts, &h->w, &h->nv, &h->nf, &h->vpairs, &h->fpairs, &h->f_ws,
                     &h->adj_ws, &h->snap};
    for (DevBuf *b : all) b->release();
    if (h->cs) cudaStreamDestroy(h->cs);
    delete h;
}

extern "C" amlp_status amlp_set_shape(amlp_sim *h, const float *h_pts, int npts, float en_min, float en_max,
                                      double cutoff, float nep_cutoff) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    if (!h_pts || npts <= 0 || npts > AMLP_MAX_PTS) return h->fail(AMLP_ERR_INVALID_ARG, "npts out of range");
    if (!(cutoff > 0.0) || !(nep_cutoff > 0.f) || !(en_max > en_min))
        return h->fail(AMLP_ERR_INVALID_ARG, "cutoff, nep_cutoff or energy range invalid");
    amlp_status s = h->cuda(h->pts.ensure((size_t)npts * 3 * sizeof(float)), "shape points");
    if (!s) s = h->cuda(cudaMemcpy(h->pts.p, h_pts, (size_t)npts * 3 * sizeof(float), cudaMemcpyHostToDevice),
                        "shape points");
    if (s) return s;
    h->nep.npts = npts;
    h->nep.d_pts = h->pts.as<float>();
    h->nep.cutoff = cutoff;
    h->nep.nep_cutoff = nep_cutoff;
    h->nep.en_min = en_min;
    h->nep.en_max = en_max;
    h->r_verlet = cutoff + h->cfg.skin;
    h->have_shape = true;
    h->list_valid = false;
    destroy_graphs(h->graphs);
    return AMLP_OK;
}

extern "C" amlp_status amlp_set_model(amlp_sim *h, const amlp_mlp *mlp, void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    if (!mlp || !mlp->d_w || mlp->n_layers < 1 || mlp->n_layers > AMLP_MAX_LAYERS)
        return h->fail(AMLP_ERR_INVALID_ARG, "net: bad layer count or no weights");
    if (mlp->dims[0] != h->D || mlp->dims[mlp->n_layers] != 1)
        return h->fail(AMLP_ERR_INVALID_ARG, "net must map the descriptor length to one energy");
    for (int k = 1; k < mlp->n_layers; ++k)
        if (mlp->dims[k] <= 0) return h->fail(AMLP_ERR_INVALID_ARG, "net: empty layer");
    const size_t bytes = (size_t)packed_weight_count(*mlp) * sizeof(float);
    cudaStream_t st = as_stream(stream);
    amlp_status s = h->cuda(h->w.ensure(bytes), "weights");
    if (!s) s = h->cuda(cudaMemcpyAsync(h->w.p, mlp->d_w, bytes, cudaMemcpyDeviceToDevice, st), "weights");
    if (s) return s;
    const bool was_wide = h->have_model && max_hidden_width(h->mlp) > 64;
    h->mlp = *mlp;
    h->mlp.d_w = h->w.as<float>();
    h->have_model = true;
    destroy_graphs(h->graphs);
    if (h->cap > 0 && (max_hidden_width(h->mlp) > 64) != was_wide) return h->alloc_pairs(h->cap);
    return AMLP_OK;
}

extern "C" amlp_status amlp_set_state(amlp_sim *h, const float *d_pos, const float *d_quat, const float *d_vel,
                                      const float *d_angmom, const float *d_mass, const float *h_moi, float box,
                                      void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    if (!d_pos || !d_quat || !d_vel || !d_angmom || !d_mass || !h_moi || !(box > 0.f))
        return h->fail(AMLP_ERR_INVALID_ARG, "null state array, moments or box <= 0");
    cudaStream_t st = as_stream(stream);
    const size_t n = (size_t)h->n;
    struct {
        DevBuf *dst;
        const float *src;
        size_t bytes;
    } cp[] = {{&h->pos, d_pos, n * 12}, {&h->quat, d_quat, n * 16}, {&h->vel, d_vel, n * 12},
              {&h->angmom, d_angmom, n * 16}, {&h->mass, d_mass, n * 4}};
    amlp_status s;
    for (auto &c : cp)
        if ((s = h->cuda(cudaMemcpyAsync(c.dst->p, c.src, c.bytes, cudaMemcpyDeviceToDevice, st), "state copy")))
            return s;
    for (int k = 0; k < 3; ++k) h->nvt.moi[k] = h_moi[k];
    h->nvt.box = box;
    amlp_thermostat t = seeded_thermostat(h->nvt.nve);
    if ((s = h->cuda(cudaMemcpyAsync(h->th.p, &t, sizeof(t), cudaMemcpyHostToDevice, st), "thermostat"))) return s;
    // the host struct t must outlive the copy
    if ((s = h->cuda(cudaStreamSynchronize(st), "thermostat"))) return s;
    s = amlp_nvt_init(h->vel.as<float>(), h->quat.as<float>(), h->angmom.as<float>(), h->mass.as<float>(), h->n,
                      &h->nvt, h->cfg.initial_ke_quirk, h->th.as<amlp_thermostat>(), h->nvt_ws.p, h->nvt_ws.bytes, st);
    if (s) return h->lib(s, "amlp_nvt_init");
    h->have_state = true;
    h->list_valid = false;
    h->timestep = 0;
    destroy_graphs(h->graphs);
    return AMLP_OK;
}

extern "C" amlp_status amlp_build_nlist(amlp_sim *h, void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    amlp_status s = h->ready();
    return s ? s : h->build_nlist(as_stream(stream));
}

extern "C" amlp_status amlp_sim_descriptors(amlp_sim *h, float *d_g, int *d_pairs, long long cap, long long *h_P,
                                            void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    amlp_status s = h->ready();
    if (s) return s;
    if (!d_g || !d_pairs || !h_P || cap < 0) return h->fail(AMLP_ERR_INVALID_ARG, "null output or cap < 0");
    cudaStream_t st = as_stream(stream);
    if (!h->list_valid && (s = h->build_nlist(st))) return s;
    s = amlp_pair_filter(h->pos.as<float>(), h->nvt.box, h->nep.cutoff, h->vpairs.as<int>(), h->nv.as<long long>(),
                         h->cap, h->fpairs.as<int>(), h->nf.as<long long>(), h->f_ws.p, h->f_ws.bytes, st);
    if (s) return h->lib(s, "amlp_pair_filter");
    long long P = 0;
    if ((s = h->cuda(cudaMemcpyAsync(&P, h->nf.p, sizeof(P), cudaMemcpyDeviceToHost, st), "pair count"))) return s;
    if ((s = h->cuda(cudaStreamSynchronize(st), "pair count"))) return s;
    *h_P = P;
    if (P > cap) return h->fail(AMLP_ERR_CAPACITY, "more filtered pairs than cap");
    if (P == 0) return AMLP_OK;
    s = amlp_descriptors(h->pos.as<float>(), h->quat.as<float>(), h->nvt.box, h->fpairs.as<int>(), P, &h->nep, d_g,
                         st);
    if (s) return h->lib(s, "amlp_descriptors");
    return h->cuda(cudaMemcpyAsync(d_pairs, h->fpairs.p, (size_t)P * 2 * sizeof(int), cudaMemcpyDeviceToDevice, st),
                   "pairs copy");
}

extern "C" amlp_status amlp_forces(amlp_sim *h, float *d_F, float *d_T, int mode, void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    amlp_status s = h->ready();
    if (s) return s;
    cudaStream_t st = as_stream(stream);
    if (!h->list_valid && (s = h->build_nlist(st))) return s;
    if ((s = h->enqueue_forces(mode, st))) return s;
    const size_t b = (size_t)h->n * 3 * sizeof(float);
    if (d_F && (s = h->cuda(cudaMemcpyAsync(d_F, h->F.p, b, cudaMemcpyDeviceToDevice, st), "F copy"))) return s;
    if (d_T && (s = h->cuda(cudaMemcpyAsync(d_T, h->T.p, b, cudaMemcpyDeviceToDevice, st), "T copy"))) return s;
    return AMLP_OK;
}

extern "C" amlp_status amlp_step(amlp_sim *h, int nsteps, int mode, void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    amlp_status s = h->ready();
    if (s) return s;
    if (nsteps < 0) return h->fail(AMLP_ERR_INVALID_ARG, "nsteps < 0");
    if (mode != AMLP_FORCES_FD && mode != AMLP_FORCES_ADJOINT) return h->fail(AMLP_ERR_INVALID_ARG, "unknown mode");
    cudaStream_t st = as_stream(stream);
    if (!h->list_valid && (s = h->build_nlist(st))) return s;
    const long long every = h->cfg.nlist_every, end = h->timestep + nsteps;
    while (h->timestep < end) {
        if (h->timestep % every == 0 && h->timestep > 0) {
            if ((s = h->build_nlist(st))) return s;
            if ((s = device_wait_status())) return h->fail(s, "a bounded device-side wait gave up");
        }
        const int seg = (int)std::min(end - h->timestep, every - h->timestep % every);
        if ((s = h->run_segment(mode, seg, st))) return s;
        h->timestep += seg;
    }
    return AMLP_OK;
}

extern "C" amlp_status amlp_get_state(amlp_sim *h, float *d_pos, float *d_quat, float *d_vel, float *d_angmom,
                                      void *stream) {
    if (!h) return AMLP_ERR_INVALID_ARG;
    if (!h->have_state) return h->fail(AMLP_ERR_INVALID_ARG, "no state (amlp_set_state)");
    cudaStream_t st = as_stream(stream);
    const size_t n = (size_t)h->n;
    struct {
        float *dst;
        const DevBuf *src;
        size_t bytes;
    } cp[] = {{d_pos, &h->pos, n * 12}, {d_quat, &h->quat, n * 16}, {d_vel, &h->vel, n * 12},
              {d_angmom, &h->angmom, n * 16}};
    for (auto &c : cp) {
        if (!c.dst) continue;
        amlp_status s =
            h->cuda(cudaMemcpyAsync(c.dst, c.src->p, c.bytes, cudaMemcpyDeviceToDevice, st), "state copy");
        if (s) return s;
    }
    return AMLP_OK;
}

extern "C" amlp_status amlp_get_thermostat(amlp_sim *h, amlp_thermostat *h_th, void *stream) {
    if (!h || !h_th) return AMLP_ERR_INVALID_ARG;
    if (!h->have_state) return h->fail(AMLP_ERR_INVALID_ARG, "no state (amlp_set_state)");
    cudaStream_t st = as_stream(stream);
    amlp_status s =
        h->cuda(cudaMemcpyAsync(h_th, h->th.p, sizeof(amlp_thermostat), cudaMemcpyDeviceToHost, st), "thermostat");
    return s ? s : h->cuda(cudaStreamSynchronize(st), "thermostat");
}

extern "C" long long amlp_timestep(const amlp_sim *h) { return h ? h->timestep : -1; }

extern "C" const char *amlp_last_error(const amlp_sim *h) { return h ? h->err.c_str() : "null handle"; }

// ------------------------------------------------------------------ amlp_pool

namespace {

struct PoolSys {
    int id = -1, n = 0, nve = 0;
    float box = 0.f, kT = 0.f;
    long long cap = 0, steps_done = 0;
    bool packed = false;
    long long first = 0;  // first body in the packed arrays (packed systems)
    std::vector<float> pos, quat, vel, angmom, mass;  // host copies until packed
};

}  // namespace

struct amlp_pool {
    amlp_nep nep{};
    amlp_mlp mlp{};
    amlp_nvt prm{};
    double r_verlet = 0.0;
    DevBuf pts, w;
    std::vector<PoolSys> sys;
    bool dirty = false;
    int next_id = 0, N = 0;
    long long cap = 0, total_pairs = 0;
    std::vector<long long> slot;  // start of each system's slot in vgap
    DevBuf pos, quat, vel, angmom, mass, rep, F, T, accel, dp, rp, th, pe, vpairs, vgap, fpairs, nv, nf, counts, nl_ws,
        f_ws, adj_ws, snap;
    cudaStream_t cs = nullptr;
    std::vector<StepGraph> graphs;
    std::string err;

    amlp_status fail(amlp_status s, const std::string &msg) {
        err = msg;
        return s;
    }
    amlp_status cuda(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return AMLP_OK;
        set_cuda_error(e);
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return AMLP_ERR_CUDA;
    }
    amlp_status lib(amlp_status s, const char *what) {
        if (s != AMLP_OK) err = std::string(what) + ": " + amlp_status_string(s);
        return s;
    }
    int find(int id) const {
        for (size_t r = 0; r < sys.size(); ++r)
            if (sys[r].id == id) return (int)r;
        return -1;
    }
    bool wide() const { return max_hidden_width(mlp) > 64; }

    // Lays the systems out contiguously: packed ones move from the current
    // arrays, new ones come from their host copies with seeded thermostats.
    amlp_status repack(cudaStream_t st) {
        destroy_graphs(graphs);
        dirty = false;
        long long n_new = 0;
        for (auto &x : sys) n_new += x.n;
        const int nrep = (int)sys.size();
        DevBuf npos, nquat, nvel, nang, nmass, nth;
        amlp_status s;
        const size_t n = (size_t)std::max<long long>(n_new, 1);
        if ((s = cuda(npos.ensure(n * 12), "pool state")) || (s = cuda(nquat.ensure(n * 16), "pool state")) ||
            (s = cuda(nvel.ensure(n * 12), "pool state")) || (s = cuda(nang.ensure(n * 16), "pool state")) ||
            (s = cuda(nmass.ensure(n * 4), "pool state")) ||
            (s = cuda(nth.ensure((size_t)std::max(nrep, 1) * sizeof(amlp_thermostat)), "pool thermostats")))
            return s;
        std::vector<amlp_thermostat> seeds(sys.size());
        long long off = 0;
        for (size_t r = 0; r < sys.size(); ++r) {
            PoolSys &x = sys[r];
            const size_t b3 = (size_t)x.n * 12, b4 = (size_t)x.n * 16, b1 = (size_t)x.n * 4;
            char *dp3[] = {npos.as<char>() + off * 12, nvel.as<char>() + off * 12};
            char *dp4[] = {nquat.as<char>() + off * 16, nang.as<char>() + off * 16};
            cudaError_t e = cudaSuccess;
            if (x.packed) {
                e = cudaMemcpyAsync(dp3[0], pos.as<char>() + x.first * 12, b3, cudaMemcpyDeviceToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp3[1], vel.as<char>() + x.first * 12, b3, cudaMemcpyDeviceToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp4[0], quat.as<char>() + x.first * 16, b4, cudaMemcpyDeviceToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp4[1], angmom.as<char>() + x.first * 16, b4, cudaMemcpyDeviceToDevice, st);
                if (!e)
                    e = cudaMemcpyAsync(nmass.as<char>() + off * 4, mass.as<char>() + x.first * 4, b1,
                                        cudaMemcpyDeviceToDevice, st);
                const int row = th_row(x.id);  // packed systems always have a row
                if (!e && row < 0) e = cudaErrorInvalidValue;
                if (!e)
                    e = cudaMemcpyAsync(nth.as<amlp_thermostat>() + r, th.as<amlp_thermostat>() + row,
                                        sizeof(amlp_thermostat), cudaMemcpyDeviceToDevice, st);
            } else {
                seeds[r] = seeded_thermostat(x.nve);
                e = cudaMemcpyAsync(dp3[0], x.pos.data(), b3, cudaMemcpyHostToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp3[1], x.vel.data(), b3, cudaMemcpyHostToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp4[0], x.quat.data(), b4, cudaMemcpyHostToDevice, st);
                if (!e) e = cudaMemcpyAsync(dp4[1], x.angmom.data(), b4, cudaMemcpyHostToDevice, st);
                if (!e) e = cudaMemcpyAsync(nmass.as<char>() + off * 4, x.mass.data(), b1, cudaMemcpyHostToDevice, st);
                if (!e)
                    e = cudaMemcpyAsync(nth.as<amlp_thermostat>() + r, &seeds[r], sizeof(amlp_thermostat),
                                        cudaMemcpyHostToDevice, st);
            }
            if ((s = cuda(e, "pool repack"))) {
                cudaStreamSynchronize(st);  // copies from host memory may still be in flight
                return s;
            }
            off += x.n;
        }
        if ((s = cuda(cudaStreamSynchronize(st), "pool repack"))) return s;  // host sources and old arrays
        std::swap(pos, npos);
        std::swap(quat, nquat);
        std::swap(vel, nvel);
        std::swap(angmom, nang);
        std::swap(mass, nmass);
        std::swap(th, nth);
        npos.release();
        nquat.release();
        nvel.release();
        nang.release();
        nmass.release();
        nth.release();
        N = (int)n_new;
        packed_ids.clear();
        off = 0;
        slot.assign(sys.size(), 0);
        cap = 0;
        std::vector<int> rep_h((size_t)N);
        std::vector<amlp_replica> rp_h(sys.size());
        size_t nl_bytes = 16;
        for (size_t r = 0; r < sys.size(); ++r) {
            PoolSys &x = sys[r];
            x.packed = true;
            x.first = off;
            std::vector<float>().swap(x.pos);
            std::vector<float>().swap(x.quat);
            std::vector<float>().swap(x.vel);
            std::vector<float>().swap(x.angmom);
            std::vector<float>().swap(x.mass);
            packed_ids.push_back(x.id);
            for (int k = 0; k < x.n; ++k) rep_h[(size_t)(off + k)] = (int)r;
            std::memset(&rp_h[r], 0, sizeof(amlp_replica));
            rp_h[r].kT = x.kT;
            rp_h[r].n_dof = (float)((x.n - 1) * 3);
            rp_h[r].rn_dof = (float)(x.n * 3);
            rp_h[r].box = x.box;
            rp_h[r].nve = x.nve;
            slot[r] = cap;
            cap += x.cap;
            size_t wb = 0;
            amlp_nlist_workspace_bytes(x.n, x.box, r_verlet, &wb);
            nl_bytes = std::max(nl_bytes, wb);
            off += x.n;
        }
        if (sys.empty()) return AMLP_OK;
        size_t fb = 0, ab = 0;
        amlp_filter_workspace_bytes(cap, &fb);
        const size_t n3 = (size_t)N * 12, n4 = (size_t)N * 16;
        if ((s = cuda(rep.ensure((size_t)N * 4), "pool")) || (s = cuda(F.ensure(n3), "pool")) ||
            (s = cuda(T.ensure(n3), "pool")) || (s = cuda(accel.ensure(n3), "pool")) ||
            (s = cuda(dp.ensure(n4), "pool")) || (s = cuda(rp.ensure(rp_h.size() * sizeof(amlp_replica)), "pool")) ||
            (s = cuda(pe.ensure(sys.size() * sizeof(double)), "pool")) ||
            (s = cuda(vpairs.ensure((size_t)cap * 8), "pool")) || (s = cuda(vgap.ensure((size_t)cap * 8), "pool")) ||
            (s = cuda(fpairs.ensure((size_t)cap * 8), "pool")) || (s = cuda(nv.ensure(8), "pool")) ||
            (s = cuda(nf.ensure(8), "pool")) || (s = cuda(counts.ensure(sys.size() * 8), "pool")) ||
            (s = cuda(nl_ws.ensure(nl_bytes), "pool")) || (s = cuda(f_ws.ensure(fb), "pool")))
            return s;
        if (wide()) {
            amlp_adjoint_workspace_bytes(cap, &ab);
            if ((s = cuda(adj_ws.ensure(ab), "pool"))) return s;
        }
        if ((s = cuda(cudaMemcpyAsync(rep.p, rep_h.data(), (size_t)N * 4, cudaMemcpyHostToDevice, st), "pool")) ||
            (s = cuda(cudaMemcpyAsync(rp.p, rp_h.data(), rp_h.size() * sizeof(amlp_replica), cudaMemcpyHostToDevice,
                                      st),
                      "pool")) ||
            (s = cuda(cudaMemsetAsync(accel.p, 0, n3, st), "pool")) ||
            (s = cuda(cudaMemsetAsync(dp.p, 0, n4, st), "pool")))
            return s;
        s = amlp_multi_nvt_init(vel.as<float>(), quat.as<float>(), angmom.as<float>(), mass.as<float>(), rep.as<int>(),
                                N, (int)sys.size(), &prm, th.as<amlp_thermostat>(), st);
        if (s) return lib(s, "amlp_multi_nvt_init");
        return cuda(cudaStreamSynchronize(st), "pool repack");  // rep_h, rp_h
    }
    // ids of the systems in the current packed arrays, in row order (their thermostat rows)
    std::vector<int> packed_ids;
    int th_row(int id) const {
        for (size_t r = 0; r < packed_ids.size(); ++r)
            if (packed_ids[r] == id) return (int)r;
        return -1;
    }

    // Every system's Verlet list into its slot, then one list with global indices.
    // Returns AMLP_ERR_CAPACITY after growing the slots of systems that overflowed
    // (the caller repacks and calls again).
    amlp_status rebuild_lists(cudaStream_t st) {
        amlp_status s;
        for (size_t r = 0; r < sys.size(); ++r) {
            const PoolSys &x = sys[r];
            s = amlp_nlist_build(pos.as<float>() + x.first * 3, x.n, x.box, r_verlet, vgap.as<int>() + slot[r] * 2,
                                 x.cap, counts.as<long long>() + r, nl_ws.p, nl_ws.bytes, st);
            if (s) return lib(s, "amlp_nlist_build");
        }
        std::vector<long long> c(sys.size());
        if ((s = cuda(cudaMemcpyAsync(c.data(), counts.p, c.size() * 8, cudaMemcpyDeviceToHost, st), "pool counts")) ||
            (s = cuda(cudaStreamSynchronize(st), "pool counts")))
            return s;
        bool grown = false;
        for (size_t r = 0; r < sys.size(); ++r)
            if (c[r] > sys[r].cap) {
                sys[r].cap = c[r] + c[r] / 4 + 1024;
                grown = true;
            }
        if (grown) {
            dirty = true;
            return AMLP_ERR_CAPACITY;
        }
        total_pairs = 0;
        for (size_t r = 0; r < sys.size(); ++r) {
            if (c[r] == 0) continue;
            const int blocks = (int)std::min<long long>((2 * c[r] + 255) / 256, 4 * kNumSM);
            k_offset_pairs<<<blocks, 256, 0, st>>>(vgap.as<int>() + slot[r] * 2, vpairs.as<int>() + total_pairs * 2,
                                                   c[r], (int)sys[r].first);
            total_pairs += c[r];
        }
        if ((s = cuda(cudaGetLastError(), "pair offsets"))) return s;
        return cuda(cudaMemcpyAsync(nv.p, &total_pairs, 8, cudaMemcpyHostToDevice, st), "pair count");
    }

    amlp_status enqueue_step(cudaStream_t st) {
        const int nrep = (int)sys.size();
        amlp_status s;
        if ((s = cuda(cudaMemsetAsync(F.p, 0, (size_t)N * 12, st), "zero F")) ||
            (s = cuda(cudaMemsetAsync(T.p, 0, (size_t)N * 12, st), "zero T")) ||
            (s = cuda(cudaMemsetAsync(pe.p, 0, (size_t)nrep * 8, st), "zero pe")))
            return s;
        s = amlp_multi_pair_filter(pos.as<float>(), rep.as<int>(), rp.as<amlp_replica>(), nep.cutoff, vpairs.as<int>(),
                                   nv.as<long long>(), cap, fpairs.as<int>(), nf.as<long long>(), f_ws.p, f_ws.bytes,
                                   st);
        if (s) return lib(s, "amlp_multi_pair_filter");
        if (wide())
            s = amlp_multi_forces_adjoint_wide(pos.as<float>(), quat.as<float>(), rep.as<int>(), rp.as<amlp_replica>(),
                                               fpairs.as<int>(), nf.as<long long>(), cap, &nep, &mlp, F.as<float>(),
                                               T.as<float>(), pe.as<double>(), adj_ws.p, adj_ws.bytes, st);
        else
            s = amlp_multi_forces_adjoint(pos.as<float>(), quat.as<float>(), rep.as<int>(), rp.as<amlp_replica>(),
                                          fpairs.as<int>(), nf.as<long long>(), cap, &nep, &mlp, F.as<float>(),
                                          T.as<float>(), pe.as<double>(), st);
        if (s) return lib(s, "amlp_multi_forces_adjoint");
        s = amlp_multi_nvt_step_two(vel.as<float>(), accel.as<float>(), F.as<float>(), mass.as<float>(),
                                    quat.as<float>(), T.as<float>(), angmom.as<float>(), dp.as<float>(), rep.as<int>(),
                                    N, nrep, rp.as<amlp_replica>(), &prm, th.as<amlp_thermostat>(), st);
        if (s) return lib(s, "amlp_multi_nvt_step_two");
        s = amlp_multi_nvt_step_one(pos.as<float>(), vel.as<float>(), accel.as<float>(), quat.as<float>(),
                                    angmom.as<float>(), dp.as<float>(), mass.as<float>(), rep.as<int>(), N,
                                    rp.as<amlp_replica>(), &prm, th.as<amlp_thermostat>(), st);
        return lib(s, "amlp_multi_nvt_step_one");
    }

    amlp_status save_restore(bool save, cudaStream_t st) {
        struct Piece {
            DevBuf *b;
            size_t bytes;
        } pcs[] = {{&pos, (size_t)N * 12}, {&quat, (size_t)N * 16}, {&vel, (size_t)N * 12},
                   {&angmom, (size_t)N * 16}, {&th, sys.size() * sizeof(amlp_thermostat)}};
        size_t total = 0;
        for (auto &pc : pcs) total += align_up(pc.bytes);
        amlp_status s;
        if (save && (s = cuda(snap.ensure(total), "snapshot"))) return s;
        size_t off = 0;
        for (auto &pc : pcs) {
            char *sp = snap.as<char>() + off;
            cudaError_t e = save ? cudaMemcpyAsync(sp, pc.b->p, pc.bytes, cudaMemcpyDeviceToDevice, st)
                                 : cudaMemcpyAsync(pc.b->p, sp, pc.bytes, cudaMemcpyDeviceToDevice, st);
            if ((s = cuda(e, "snapshot copy"))) return s;
            off += align_up(pc.bytes);
        }
        return AMLP_OK;
    }
};

extern "C" amlp_status amlp_pool_create(const amlp_pool_config *cfg, amlp_pool **out) {
    if (!cfg || !out) return AMLP_ERR_INVALID_ARG;
    *out = nullptr;
    if (!cfg->h_pts || cfg->npts <= 0 || cfg->npts > AMLP_MAX_PTS || !cfg->h_moi || !cfg->mlp || !cfg->mlp->d_w ||
        !(cfg->dt > 0.f) || !(cfg->cutoff > 0.0) || !(cfg->nep_cutoff > 0.f) || !(cfg->en_max > cfg->en_min))
        return AMLP_ERR_INVALID_ARG;
    const amlp_mlp &m = *cfg->mlp;
    if (m.n_layers < 1 || m.n_layers > AMLP_MAX_LAYERS ||
        m.dims[0] != descriptor_length(cfg->nrad, cfg->nang, cfg->lmax) || m.dims[m.n_layers] != 1)
        return AMLP_ERR_INVALID_ARG;
    amlp_pool *p = new amlp_pool();
    const size_t wbytes = (size_t)packed_weight_count(m) * sizeof(float);
    amlp_status s = p->cuda(p->pts.ensure((size_t)cfg->npts * 12), "shape points");
    if (!s) s = p->cuda(cudaMemcpy(p->pts.p, cfg->h_pts, (size_t)cfg->npts * 12, cudaMemcpyHostToDevice), "shape");
    if (!s) s = p->cuda(p->w.ensure(wbytes), "weights");
    if (!s) s = p->cuda(cudaMemcpy(p->w.p, m.d_w, wbytes, cudaMemcpyDeviceToDevice), "weights");
    if (!s) s = p->cuda(cudaStreamCreateWithFlags(&p->cs, cudaStreamNonBlocking), "capture stream");
    if (s) {
        amlp_pool_destroy(p);
        return s;
    }
    p->nep.nrad = cfg->nrad;
    p->nep.nang = cfg->nang;
    p->nep.lmax = cfg->lmax;
    p->nep.npts = cfg->npts;
    p->nep.d_pts = p->pts.as<float>();
    p->nep.cutoff = cfg->cutoff;
    p->nep.nep_cutoff = cfg->nep_cutoff;
    p->nep.en_min = cfg->en_min;
    p->nep.en_max = cfg->en_max;
    p->nep.dx = p->nep.dteta = 1e-5f;
    p->mlp = m;
    p->mlp.d_w = p->w.as<float>();
    p->prm.dt = cfg->dt;
    p->prm.tau = cfg->tau > 0.f ? cfg->tau : (float)(100.0 * (double)cfg->dt);
    for (int k = 0; k < 3; ++k) p->prm.moi[k] = cfg->h_moi[k];
    p->r_verlet = cfg->cutoff + (cfg->skin > 0.0 ? cfg->skin : 2.0);
    *out = p;
    return AMLP_OK;
}

extern "C" void amlp_pool_destroy(amlp_pool *p) {
    if (!p) return;
    destroy_graphs(p->graphs);
    DevBuf *all[] = {&p->pts, &p->w, &p->pos, &p->quat, &p->vel, &p->angmom, &p->mass, &p->rep, &p->F, &p->T,
                     &p->accel, &p->dp, &p->rp, &p->th, &p->pe, &p->vpairs, &p->vgap, &p->fpairs, &p->nv, &p->nf,
                     &p->counts, &p->nl_ws, &p->f_ws, &p->adj_ws, &p->snap};
    for (DevBuf *b : all) b->release();
    if (p->cs) cudaStreamDestroy(p->cs);
    delete p;
}

extern "C" amlp_status amlp_pool_admit(amlp_pool *p, const amlp_pool_system *x, int *id) {
    if (!p) return AMLP_ERR_INVALID_ARG;
    if (!x || !id || x->n <= 0 || !(x->box > 0.f) || !x->h_pos || !x->h_quat || !x->h_vel || !x->h_angmom || !x->h_mass)
        return p->fail(AMLP_ERR_INVALID_ARG, "bad system description");
    PoolSys s;
    s.id = p->next_id++;
    s.n = x->n;
    s.box = x->box;
    s.kT = x->kT;
    s.nve = x->nve ? 1 : 0;
    if (x->verlet_cap > 0) {
        s.cap = x->verlet_cap;
    } else {
        const double rho = (double)x->n / ((double)x->box * x->box * x->box);
        const double pi = 3.14159265358979323846;
        const double est = 0.5 * x->n * rho * 4.0 / 3.0 * pi * p->r_verlet * p->r_verlet * p->r_verlet;
        s.cap = (long long)(1.5 * est) + 4LL * x->n + 1024;
    }
    const size_t n = (size_t)x->n;
    s.pos.assign(x->h_pos, x->h_pos + 3 * n);
    s.quat.assign(x->h_quat, x->h_quat + 4 * n);
    s.vel.assign(x->h_vel, x->h_vel + 3 * n);
    s.angmom.assign(x->h_angmom, x->h_angmom + 4 * n);
    s.mass.assign(x->h_mass, x->h_mass + n);
    p->sys.push_back(std::move(s));
    p->dirty = true;
    *id = p->sys.back().id;
    return AMLP_OK;
}

extern "C" amlp_status amlp_pool_evict(amlp_pool *p, int id, float *h_pos, float *h_quat, float *h_vel,
                                       float *h_angmom, amlp_thermostat *h_th) {
    if (!p) return AMLP_ERR_INVALID_ARG;
    const int r = p->find(id);
    if (r < 0) return p->fail(AMLP_ERR_INVALID_ARG, "no such system");
    PoolSys &x = p->sys[(size_t)r];
    const size_t n = (size_t)x.n;
    amlp_status s = AMLP_OK;
    if (x.packed) {
        struct {
            float *dst;
            const DevBuf *src;
            size_t w;
        } cp[] = {{h_pos, &p->pos, 3}, {h_quat, &p->quat, 4}, {h_vel, &p->vel, 3}, {h_angmom, &p->angmom, 4}};
        for (auto &c : cp)
            if (c.dst && !s)
                s = p->cuda(cudaMemcpy(c.dst, c.src->as<float>() + x.first * c.w, n * c.w * 4, cudaMemcpyDeviceToHost),
                            "evict copy");
        const int row = p->th_row(id);
        if (h_th && !s && row < 0) s = p->fail(AMLP_ERR_INVALID_ARG, "packed system without a thermostat row");
        if (h_th && !s)
            s = p->cuda(cudaMemcpy(h_th, p->th.as<amlp_thermostat>() + row, sizeof(amlp_thermostat),
                                   cudaMemcpyDeviceToHost),
                        "evict copy");
    } else {
        if (h_pos) std::memcpy(h_pos, x.pos.data(), n * 12);
        if (h_quat) std::memcpy(h_quat, x.quat.data(), n * 16);
        if (h_vel) std::memcpy(h_vel, x.vel.data(), n * 12);
        if (h_angmom) std::memcpy(h_angmom, x.angmom.data(), n * 16);
        if (h_th) *h_th = seeded_thermostat(x.nve);
    }
    if (s) return s;
    p->sys.erase(p->sys.begin() + r);
    p->dirty = true;
    return AMLP_OK;
}

extern "C" amlp_status amlp_pool_step_segment(amlp_pool *p, int nsteps, void *stream) {
    if (!p) return AMLP_ERR_INVALID_ARG;
    if (nsteps < 0) return p->fail(AMLP_ERR_INVALID_ARG, "nsteps < 0");
    cudaStream_t st = as_stream(stream);
    amlp_status s;
    for (int attempt = 0;; ++attempt) {
        if (p->dirty && (s = p->repack(st))) return s;
        if (p->sys.empty() || nsteps == 0) return AMLP_OK;
        s = p->rebuild_lists(st);
        if (s == AMLP_OK) break;
        if (s != AMLP_ERR_CAPACITY || attempt > 4) return s;
    }
    StepGraph *g = nullptr;
    for (auto &x : p->graphs)
        if (x.seg == nsteps) g = &x;
    if (!g) {
        if ((s = p->save_restore(true, st)) || (s = p->enqueue_step(st)) || (s = p->save_restore(false, st))) return s;
        if ((s = p->cuda(cudaStreamSynchronize(st), "warm-up step"))) return s;
        StepGraph ng;
        ng.seg = nsteps;
        amlp_status es = AMLP_OK;
        cudaError_t e = capture_steps(p->cs, nsteps, [&](cudaStream_t c) { return p->enqueue_step(c); }, es, &ng.exec);
        if (es) return es;
        if ((s = p->cuda(e, "graph capture"))) return s;
        p->graphs.push_back(ng);
        g = &p->graphs.back();
    }
    if ((s = p->cuda(cudaGraphLaunch(g->exec, st), "graph launch"))) return s;
    for (auto &x : p->sys) x.steps_done += nsteps;
    if ((s = p->cuda(cudaStreamSynchronize(st), "segment"))) return s;
    if ((s = device_wait_status())) return p->fail(s, "a bounded device-side wait gave up");
    return AMLP_OK;
}

extern "C" amlp_status amlp_pool_system_status(amlp_pool *p, int id, int *status, long long *steps_done,
                                               amlp_thermostat *h_th) {
    if (!p) return AMLP_ERR_INVALID_ARG;
    const int r = p->find(id);
    if (r < 0) return p->fail(AMLP_ERR_INVALID_ARG, "no such system");
    const PoolSys &x = p->sys[(size_t)r];
    if (status) *status = x.packed ? AMLP_POOL_ACTIVE : AMLP_POOL_PENDING;
    if (steps_done) *steps_done = x.steps_done;
    if (h_th) {
        if (!x.packed) {
            *h_th = seeded_thermostat(x.nve);
        } else {
            const int row = p->th_row(id);
            if (row < 0) return p->fail(AMLP_ERR_INVALID_ARG, "packed system without a thermostat row");
            amlp_status s = p->cuda(cudaMemcpy(h_th, p->th.as<amlp_thermostat>() + row, sizeof(amlp_thermostat),
                                               cudaMemcpyDeviceToHost),
                                    "thermostat");
            if (s) return s;
        }
    }
    return AMLP_OK;
}

extern "C" int amlp_pool_size(const amlp_pool *p) { return p ? (int)p->sys.size() : 0; }

extern "C" const char *amlp_pool_last_error(const amlp_pool *p) { return p ? p->err.c_str() : "null pool"; }
