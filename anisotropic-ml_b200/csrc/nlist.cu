// Verlet pair list by a counting-sort cell list, with the pair criterion of
// scipy's cKDTree.query_pairs as the reference calls it (Sim.py:85-92,
// :192-198): FP64 periodic distances of float32(pos + L/2) in a box of edge
// float32(L + 1e-4), folded once per axis, squared components summed in x, y,
// z order without FMA, compared inclusively with r*r. Pairs (i, j), i < j,
// are written sorted by i then j.
//
// Steps: (1) cell of every body (cells of edge >= r, so every pair within r
// lies in neighbouring cells), (2) count per cell, exclusive scan, (3) fill
// the cell lists, (4) one warp per body i counts the j > i within r over the
// 27 neighbouring cells, (5) scan of the counts, (6) the same traversal
// collects the j into shared memory, ranks them and writes them in order.
//
// Gated builds (displacement-triggered rebuilds): every kernel of the pass
// takes gate (null = always build); with gate[0] == 0 they return at once, so
// a CUDA graph can hold the pass in every step and only the flagged steps pay
// for it. A gated build also stores the positions it was built from, counts
// itself in gate[1] and sets gate[2] when the list did not fit its capacity.
#include <mutex>

#include "common.cuh"
#include "scan.cuh"

namespace amlp {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kSortCap = 1024;   // neighbours per body ranked in a warp's shared buffer
constexpr int kBigCap = 8192;    // up to this many: written unordered, then ranked by one block (k_sort_big)

struct Grid {
    int n, nc;        // bodies, cells per side (1 = one cell holding all bodies)
    double fb, hb;    // periodic box edge and half edge (FP64)
    double r2;        // r * r
    double inv_cs;    // nc / fb
    float halfL;      // float32(L * 0.5)
};

__global__ void k_cells(const float *pos, Grid g, double *xd, int *cell_of, int *cell_count, const int *gate,
                        float *ref) {
    if (gate && !*gate) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    if (ref) {
        ref[3 * i] = pos[3 * i];
        ref[3 * i + 1] = pos[3 * i + 1];
        ref[3 * i + 2] = pos[3 * i + 2];
    }
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double x = (double)__fadd_rn(pos[3 * i + k], g.halfL);
        xd[3 * i + k] = x;
        int ci = (int)(x * g.inv_cs);
        c[k] = ci < 0 ? 0 : (ci >= g.nc ? g.nc - 1 : ci);
    }
    int cid = (c[0] * g.nc + c[1]) * g.nc + c[2];
    cell_of[i] = cid;
    atomicAdd(&cell_count[cid], 1);
}

__global__ void k_fill(int n, const int *cell_of, const long long *cell_start, int *cell_fill, int *cell_list,
                       const int *gate) {
    if (gate && !*gate) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cid = cell_of[i];
    int slot = atomicAdd(&cell_fill[cid], 1);
    cell_list[cell_start[cid] + slot] = i;
}

__device__ __forceinline__ bool within(const double *xd, int i, int j, const Grid &g) {
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double d = __dsub_rn(xd[3 * i + k], xd[3 * j + k]);
        if (d < -g.hb) d = __dadd_rn(g.fb, d);
        else if (d > g.hb) d = __dsub_rn(d, g.fb);
        r = __dadd_rn(r, __dmul_rn(d, d));
    }
    return r <= g.r2;
}

// Calls f(j) for every j > i within r, lane-strided over the neighbouring cells.
// All lanes of the warp call it with the same i; f is called by the lane that
// tested j, with `ok` telling whether j qualifies (every lane calls f once per
// round so that warp collectives inside f are safe).
template <class F>
__device__ __forceinline__ void for_candidates(int i, const Grid &g, const double *xd, const int *cell_of,
                                               const long long *cell_start, const int *cell_list, F &&f) {
    const int lane = threadIdx.x & 31;
    int cid = cell_of[i];
    int cz = cid % g.nc, cy = (cid / g.nc) % g.nc, cx = cid / (g.nc * g.nc);
    const int span = g.nc >= 3 ? 1 : 0;
    for (int dx = -span; dx <= span; ++dx)
        for (int dy = -span; dy <= span; ++dy)
            for (int dz = -span; dz <= span; ++dz) {
                int x = (cx + dx + g.nc) % g.nc, y = (cy + dy + g.nc) % g.nc, z = (cz + dz + g.nc) % g.nc;
                int c = (x * g.nc + y) * g.nc + z;
                long long s = cell_start[c], e = cell_start[c + 1];
                for (long long base = s; base < e; base += 32) {
                    long long idx = base + lane;
                    int j = idx < e ? cell_list[idx] : -1;
                    bool ok = j > i && within(xd, i, j, g);
                    f(j, ok);
                }
            }
}

__global__ void k_count(Grid g, const double *xd, const int *cell_of, const long long *cell_start,
                        const int *cell_list, long long *counts, const int *gate) {
    if (gate && !*gate) return;
    int i = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (i >= g.n) return;
    int cnt = 0;
    for_candidates(i, g, xd, cell_of, cell_start, cell_list, [&](int, bool ok) { cnt += ok; });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) counts[i] = cnt;
}

__global__ void k_write(Grid g, const double *xd, const int *cell_of, const long long *cell_start,
                        const int *cell_list, const long long *offsets, int *pairs, long long cap, const int *gate) {
    if (gate && !*gate) return;
    __shared__ int buf[kWarpsPerBlock][kSortCap];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int i = blockIdx.x * kWarpsPerBlock + w;
    if (i >= g.n) return;
    long long off = offsets[i];
    int cnt = (int)(offsets[i + 1] - off);
    if (cnt == 0 || off >= cap) return;  // nothing of this body's list fits
    int *b = buf[w];
    if (cnt <= kSortCap) {
        int fill = 0;
        for_candidates(i, g, xd, cell_of, cell_start, cell_list, [&](int j, bool ok) {
            unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) b[fill + __popc(m & ((1u << lane) - 1u))] = j;
            fill += __popc(m);
        });
        __syncwarp();
        for (int e = lane; e < cnt; e += 32) {
            int j = b[e], rank = 0;
            for (int k = 0; k < cnt; ++k) rank += b[k] < j;
            long long o = off + rank;
            if (o < cap) {
                pairs[2 * o] = i;
                pairs[2 * o + 1] = j;
            }
        }
        return;
    }
    if (cnt <= kBigCap && off + cnt > cap) return;  // crossing cap: k_sort_big writes the part that fits
    if (cnt <= kBigCap) {
        // written in candidate order here; k_sort_big ranks the segment afterwards
        int fill = 0;
        for_candidates(i, g, xd, cell_of, cell_start, cell_list, [&](int j, bool ok) {
            unsigned m = __ballot_sync(0xffffffffu, ok);
            long long o = off + fill + __popc(m & ((1u << lane) - 1u));
            if (ok && o < cap) pairs[2 * o + 1] = j;
            fill += __popc(m);
        });
        return;
    }
    // More neighbours than one block ranks: emit them in increasing order by
    // repeated warp-wide minimum (slow, only for pathological inputs).
    int prev = i;
    for (int k = 0; k < cnt; ++k) {
        int best = 0x7fffffff;
        for_candidates(i, g, xd, cell_of, cell_start, cell_list, [&](int j, bool ok) {
            if (ok && j > prev && j < best) best = j;
        });
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0 && off + k < cap) {
            pairs[2 * (off + k)] = i;
            pairs[2 * (off + k) + 1] = best;
        }
        prev = best;
    }
}

// Sorts the segments of bodies with kSortCap < count <= kBigCap: one block per
// body, every j ranked by counting the smaller ones (the j of a body are
// distinct), written back with i. k_write left such a segment in candidate
// order when it fits below cap; the one segment that crosses cap is gathered
// here (warp 0 walks the neighbouring cells) and only its first cap - off
// pairs are written, so the pairs that fit are always the head of the list.
__global__ void __launch_bounds__(256) k_sort_big(Grid g, const double *xd, const int *cell_of,
                                                  const long long *cell_start, const int *cell_list,
                                                  const long long *offsets, int *pairs, long long cap,
                                                  const int *gate) {
    if (gate && !*gate) return;
    __shared__ int buf[kBigCap];
    for (int i = blockIdx.x; i < g.n; i += gridDim.x) {
        const long long off = offsets[i];
        const int cnt = (int)(offsets[i + 1] - off);
        if (cnt <= kSortCap || cnt > kBigCap || off >= cap) continue;
        const bool crossing = off + cnt > cap;
        if (!crossing) {
            for (int e = threadIdx.x; e < cnt; e += blockDim.x) buf[e] = pairs[2 * (off + e) + 1];
        } else if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int fill = 0;
            for_candidates(i, g, xd, cell_of, cell_start, cell_list, [&](int j, bool ok) {
                unsigned m = __ballot_sync(0xffffffffu, ok);
                if (ok) buf[fill + __popc(m & ((1u << lane) - 1u))] = j;
                fill += __popc(m);
            });
        }
        __syncthreads();
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
            const int j = buf[e];
            int rank = 0;
            for (int k = 0; k < cnt; ++k) rank += buf[k] < j;
            if (off + rank < cap) {
                pairs[2 * (off + rank)] = i;
                pairs[2 * (off + rank) + 1] = j;
            }
        }
        __syncthreads();
    }
}

__global__ void k_total(const long long *offsets, int n, long long *d_count, int *gate, long long cap) {
    if (gate && !gate[0]) return;
    *d_count = offsets[n];
    if (gate) {
        gate[1] += 1;
        if (offsets[n] > cap) gate[2] = 1;
    }
}

// gate[0] = 1 when some body has moved more than sqrt(max_d2) from ref
// (minimum image in the cubic box), else 0 (gate[0] is cleared before).
__global__ void k_displacement(const float *pos, const float *ref, int n, float box, float max_d2, int *gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float d2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float d = pos[3 * i + k] - ref[3 * i + k];
        d -= box * rintf(d / box);
        d2 = fmaf(d, d, d2);
    }
    if (d2 > max_d2) gate[0] = 1;
}

Grid make_grid(int n, float box, double r) {
    Grid g;
    g.n = n;
    float bs = box + 0.0001f;  // float32(L + 1e-4), as numpy evaluates Lx + 0.0001
    g.fb = (double)bs;
    g.hb = 0.5 * g.fb;
    g.r2 = r * r;
    g.halfL = box * 0.5f;
    long long nc = (long long)floor(g.fb / (r * (1.0 + 1e-6)));
    if (nc > 160) nc = 160;
    if (nc < 3) nc = 1;
    g.nc = (int)nc;
    g.inv_cs = (double)g.nc / g.fb;
    return g;
}

struct NlistWs {
    double *xd;
    int *cell_of, *cell_count, *cell_fill, *cell_list;
    long long *cell_start, *counts, *scan_tmp;
};

amlp_status launch_build(const float *d_pos, const Grid &g, const NlistWs &w, int *d_pairs, long long cap,
                         long long *d_count, int *gate, float *ref, cudaStream_t s);

size_t carve(Carver &c, const Grid &g, NlistWs *w) {
    size_t ncell = (size_t)g.nc * g.nc * g.nc;
    w->xd = c.take<double>(3 * (size_t)g.n);
    w->cell_of = c.take<int>(g.n);
    w->cell_count = c.take<int>(ncell);
    w->cell_fill = c.take<int>(ncell);
    w->cell_list = c.take<int>(g.n);
    w->cell_start = c.take<long long>(ncell + 1);
    w->counts = c.take<long long>((size_t)g.n + 1);
    w->scan_tmp = c.take<long long>(scan_tmp_elems(std::max<size_t>(ncell, g.n) + 1));
    return c.used;
}

}  // namespace
}  // namespace amlp

using namespace amlp;

extern "C" amlp_status amlp_nlist_workspace_bytes(int n, float box, double r, size_t *bytes) {
    if (n <= 0 || !(box > 0.f) || !(r > 0.0) || !bytes) return AMLP_ERR_INVALID_ARG;
    Grid g = make_grid(n, box, r);
    Carver c(nullptr, 0);
    NlistWs w;
    *bytes = carve(c, g, &w) + 256;
    return AMLP_OK;
}

extern "C" amlp_status amlp_nlist_build(const float *d_pos, int n, float box, double r, int *d_pairs,
                                        long long cap, long long *d_count, void *d_ws, size_t ws_bytes,
                                        void *stream) {
    if (n <= 0 || !(box > 0.f) || !(r > 0.0) || !d_pos || !d_count || cap < 0 || (cap > 0 && !d_pairs))
        return AMLP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    Grid g = make_grid(n, box, r);
    Carver c(d_ws, ws_bytes);
    NlistWs w;
    carve(c, g, &w);
    if (!d_ws || !c.ok()) return AMLP_ERR_WORKSPACE;
    return launch_build(d_pos, g, w, d_pairs, cap, d_count, nullptr, nullptr, s);
}

namespace amlp {
namespace {

amlp_status launch_build(const float *d_pos, const Grid &g, const NlistWs &w, int *d_pairs, long long cap,
                         long long *d_count, int *gate, float *ref, cudaStream_t s) {
    const int n = g.n;
    size_t ncell = (size_t)g.nc * g.nc * g.nc;
    AMLP_CHECK_CUDA(cudaMemsetAsync(w.cell_count, 0, ncell * sizeof(int), s));
    AMLP_CHECK_CUDA(cudaMemsetAsync(w.cell_fill, 0, ncell * sizeof(int), s));
    int tb = 256;
    k_cells<<<(n + tb - 1) / tb, tb, 0, s>>>(d_pos, g, w.xd, w.cell_of, w.cell_count, gate, ref);
    amlp_status st = exclusive_scan_int(w.cell_count, w.cell_start, (long long)ncell, w.scan_tmp, s, gate);
    if (st) return st;
    k_fill<<<(n + tb - 1) / tb, tb, 0, s>>>(n, w.cell_of, w.cell_start, w.cell_fill, w.cell_list, gate);
    int nb = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
    k_count<<<nb, 32 * kWarpsPerBlock, 0, s>>>(g, w.xd, w.cell_of, w.cell_start, w.cell_list, w.counts, gate);
    st = exclusive_scan_ll(w.counts, w.counts, n, w.scan_tmp, s, gate);
    if (st) return st;
    k_write<<<nb, 32 * kWarpsPerBlock, 0, s>>>(g, w.xd, w.cell_of, w.cell_start, w.cell_list, w.counts, d_pairs, cap,
                                               gate);
    k_sort_big<<<kNumSM, 256, 0, s>>>(g, w.xd, w.cell_of, w.cell_start, w.cell_list, w.counts, d_pairs, cap, gate);
    k_total<<<1, 1, 0, s>>>(w.counts, n, d_count, gate, cap);
    return check_launch();
}

}  // namespace
}  // namespace amlp

extern "C" amlp_status amlp_nlist_check_displacement(const float *d_pos, const float *d_ref, int n, float box,
                                                     float max_disp, int *d_gate, void *stream) {
    if (n <= 0 || !(box > 0.f) || !(max_disp >= 0.f) || !d_pos || !d_ref || !d_gate) return AMLP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    AMLP_CHECK_CUDA(cudaMemsetAsync(d_gate, 0, sizeof(int), s));
    k_displacement<<<(n + 255) / 256, 256, 0, s>>>(d_pos, d_ref, n, box, max_disp * max_disp, d_gate);
    return check_launch();
}

extern "C" amlp_status amlp_nlist_build_gated(const float *d_pos, int n, float box, double r, int *d_pairs,
                                              long long cap, long long *d_count, void *d_ws, size_t ws_bytes,
                                              int *d_gate, float *d_ref, void *stream) {
    if (n <= 0 || !(box > 0.f) || !(r > 0.0) || !d_pos || !d_count || !d_gate || !d_ref || cap < 0 ||
        (cap > 0 && !d_pairs))
        return AMLP_ERR_INVALID_ARG;
    Grid g = make_grid(n, box, r);
    Carver c(d_ws, ws_bytes);
    NlistWs w;
    carve(c, g, &w);
    if (!d_ws || !c.ok()) return AMLP_ERR_WORKSPACE;
    return launch_build(d_pos, g, w, d_pairs, cap, d_count, d_gate, d_ref, as_stream(stream));
}

// ---------------------------------------------------------------------------
// Allocation-free variant of amlp_nlist_build.
//
// Some callers cannot allocate device memory at all, not even a workspace:
// for example a host program (an MD engine or a serving process) that hands
// this library only the buffers it owns, under a fixed GPU-memory budget, and
// does not let plug-ins call cudaMalloc or cudaFree. This entry point needs
// nothing beyond its inputs and outputs. Its scratch is the file-scope
// device array below: every GPU that loads the library holds it (13
// MiB) until the process exits.
//
// Limits: at most kNoAllocMaxBodies bodies, and at most kNoAllocMaxCells cells
// per box edge. Larger boxes simply use larger cells, which gives the same
// list. Every call shares the one array: calls that overlap on the GPU (on
// different streams, or from different host threads without ordering) race
// and must not be issued. The counters that must start at zero are cleared
// on the stream at the start of every call.
// ---------------------------------------------------------------------------
namespace amlp {
namespace {

constexpr int kNoAllocMaxBodies = 262144;
constexpr int kNoAllocMaxCells = 48;
constexpr size_t kNoAllocScratchBytes = 13u << 20;

__device__ __align__(256) unsigned char g_nlist_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the host-side name is only a stand-in, not a device address).
amlp_status noalloc_scratch(void **out) {
    int dev = 0;
    AMLP_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return AMLP_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        AMLP_CHECK_CUDA(cudaGetSymbolAddress(&p, g_nlist_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return AMLP_OK;
}

}  // namespace
}  // namespace amlp

extern "C" amlp_status amlp_nlist_build_noalloc(const float *d_pos, int n, float box, double r, int *d_pairs,
                                                long long cap, long long *d_count, void *stream) {
    if (n <= 0 || !(box > 0.f) || !(r > 0.0) || !d_pos || !d_count || cap < 0 || (cap > 0 && !d_pairs))
        return AMLP_ERR_INVALID_ARG;
    if (n > kNoAllocMaxBodies) return AMLP_ERR_TOO_LARGE;
    Grid g = make_grid(n, box, r);
    if (g.nc > kNoAllocMaxCells) {
        g.nc = kNoAllocMaxCells;
        g.inv_cs = (double)g.nc / g.fb;
    }
    Carver probe(nullptr, kNoAllocScratchBytes);
    NlistWs w;
    carve(probe, g, &w);
    if (!probe.ok()) return AMLP_ERR_TOO_LARGE;
    void *scratch = nullptr;
    amlp_status st = noalloc_scratch(&scratch);
    if (st) return st;
    Carver c(scratch, kNoAllocScratchBytes);
    carve(c, g, &w);
    return launch_build(d_pos, g, w, d_pairs, cap, d_count, nullptr, nullptr, as_stream(stream));
}
