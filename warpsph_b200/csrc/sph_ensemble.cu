// Batched ensemble of independent periodic delta-SPH boxes (no counterpart in the
// reference, which runs one simulation per process; the right-hand side per box is
// schemes/deltaSPH.py's, see sph_deltasph.cuh).
//
// All boxes share the periodic domain of SphParams but not their particles: box b has
// its own cell grid of G_b^dim cells (cell size L / G_b >= verlet_scale * max H in the
// box), and the cell keys of box b start at box_cell_base[b], so a neighbour search over
// every particle of every box in one set of launches (segment offsets into one cell
// table) never pairs particles of different boxes.
//
// One time step of every box is ONE cooperative persistent launch (k_ens_step): Heun
// RK2 with two right-hand sides, four phases separated by three bounded grid barriers:
//   A(y0) | B(y0), y1 = y0 + dt k1 | A(y1) | B(y1), y = y0 + dt/2 (k1 + k2)
// where A is the renormalised density gradient + EOS and B the delta-SPH right-hand side.
// dt is per box (box_dt).  Arrays that other blocks rewrite between phases are read
// with ld.global.cg.  The step also reduces the largest displacement since the list
// was built, so the caller can tell when the Verlet skin is used up.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include "sph_deltasph.cuh"
#include "sph_persistent.cuh"

namespace wsph {

// ---------------------------------------------------------------- neighbour search
template <int D> __device__ __forceinline__ void ens_cell(const Vec<D>& x, const DomainF& dom, int G, int* c) {
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        int k = (int)floorf(__fdiv_rn(__fsub_rn(x.v[a], dom.min[a]), dom.L[a]) * (float)G);
        c[a] = k < 0 ? 0 : (k >= G ? G - 1 : k);
    }
}
template <int D> __device__ __forceinline__ int ens_key(const int* c, int G, int base) {
    int k = c[D - 1];
    #pragma unroll
    for (int a = D - 2; a >= 0; --a) k = k * G + c[a];
    return base + k;
}

template <int D>
__global__ void k_ens_keys(int n, DomainF dom, const float* __restrict__ x, const int32_t* __restrict__ box_of,
                           const int32_t* __restrict__ box_grid, const int32_t* __restrict__ box_base, int32_t* __restrict__ keys,
                           int32_t* __restrict__ slot, int32_t* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = box_of[i];
    int c[D];
    ens_cell<D>(load_vec<D>(x, i), dom, box_grid[b], c);
    const int key = ens_key<D>(c, box_grid[b], box_base[b]);
    keys[i] = key;
    slot[i] = atomicAdd(counts + key, 1);
}

__global__ void k_ens_scatter(int n, const int32_t* __restrict__ keys, const int32_t* __restrict__ slot,
                              const int32_t* __restrict__ start, int32_t* __restrict__ sorted) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sorted[start[keys[i]] + slot[i]] = i;
}

// Ascending particle index inside each cell (deterministic rows).
__global__ void k_ens_sort_cells(int64_t ncells, const int32_t* __restrict__ start, const int32_t* __restrict__ counts,
                                 int32_t* __restrict__ sorted) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int32_t* s = sorted + start[c];
    const int k = counts[c];
    for (int a = 1; a < k; ++a) {
        const int v = s[a];
        int b = a - 1;
        while (b >= 0 && s[b] > v) { s[b + 1] = s[b]; --b; }
        s[b + 1] = v;
    }
}

// Count (FILL = false) or fill the Verlet rows: j in the 3^dim stencil cells of i's box
// grid (periodic wrap, x fastest), ascending index within a cell, kept when
// |x_i - x_j|^2 < (verlet_scale max(H_i, H_j))^2 with the minimum-image distance.
template <int D, int G, bool FILL>
__global__ void __launch_bounds__(128)
k_ens_verlet(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const int32_t* __restrict__ box_of,
             const int32_t* __restrict__ box_grid, const int32_t* __restrict__ box_base, const int32_t* __restrict__ start,
             const int32_t* __restrict__ counts, const int32_t* __restrict__ sorted, int32_t* __restrict__ num,
             const int32_t* __restrict__ offs, int32_t* __restrict__ list, const long long* __restrict__ nnz, int64_t cap) {
    Grp<G> g(n);
    if (FILL && *nnz > cap) return;            // uniform over the grid
    // every group (valid or not) walks the same stencil with a warp-uniform candidate
    // loop, so the ballots below always have the full warp
    const int i = g.valid ? g.i : 0;
    Vec<D> xi = vzero<D>();
    float Hi = 0.f;
    int Gb = 1, base = 0, c[D], row = 0;
    #pragma unroll
    for (int a = 0; a < D; ++a) c[a] = 0;
    if (g.valid) {
        xi = load_vec<D>(x, i);
        Hi = H[i];
        const int b = box_of[i];
        Gb = box_grid[b];
        base = box_base[b];
        ens_cell<D>(xi, P.dom, Gb, c);
        if (FILL) row = offs[i];
    }
    const unsigned int lanes = (1u << G) - 1u;
    const int gshift = threadIdx.x & 31 & ~(G - 1);
    int w = 0;
    constexpr int NS = D == 1 ? 3 : (D == 2 ? 9 : 27);
    for (int sidx = 0; sidx < NS; ++sidx) {
        int s0 = 0, cn = 0;
        if (g.valid) {
            int cc[D], t = sidx;
            #pragma unroll
            for (int a = 0; a < D; ++a) { cc[a] = (c[a] + (t % 3) - 1 + Gb) % Gb; t /= 3; }
            const int key = ens_key<D>(cc, Gb, base);
            s0 = start[key];
            cn = counts[key];
        }
        for (int q0 = 0; __any_sync(0xffffffffu, q0 < cn); q0 += G) {
            const int q = q0 + g.lane;
            bool keep = false;
            int j = 0;
            if (q < cn) {
                j = sorted[s0 + q];
                const Vec<D> d = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
                const float R = __fmul_rn(P.verlet_scale, wmax(Hi, __ldg(H + j)));
                keep = dist2_rn<D>(d) < __fmul_rn(R, R);
            }
            const unsigned int bits = (__ballot_sync(0xffffffffu, keep) >> gshift) & lanes;
            if (FILL && keep) list[row + w + __popc(bits & ((1u << g.lane) - 1u))] = j;
            w += __popc(bits);
        }
    }
    if (!FILL && g.valid && g.lane == 0) num[g.i] = w;
}

__global__ void k_ens_check(const long long* __restrict__ nnz, int64_t cap, int32_t* __restrict__ status) {
    if (*nnz > cap) atomicOr(status, SPH_STATUS_LIST_OVERFLOW);
}

struct EnsNbWs {
    int32_t *keys, *slot, *counts, *start, *sorted;
    long long* total;
    char* scan;
    int64_t bytes;
};
static int64_t al256(int64_t b) { return (b + 255) / 256 * 256; }
static EnsNbWs ens_carve(char* base, int64_t n, int64_t ncells) {
    EnsNbWs w;
    int64_t o = 0;
    w.total = reinterpret_cast<long long*>(base + o); o += 256;
    w.keys = reinterpret_cast<int32_t*>(base + o); o += al256(n * 4);
    w.slot = reinterpret_cast<int32_t*>(base + o); o += al256(n * 4);
    w.sorted = reinterpret_cast<int32_t*>(base + o); o += al256(n * 4);
    w.counts = reinterpret_cast<int32_t*>(base + o); o += al256(ncells * 4);
    w.start = reinterpret_cast<int32_t*>(base + o); o += al256(ncells * 4);
    w.scan = base + o;
    o += al256(scan_ws_bytes(ncells > n ? ncells : n));
    w.bytes = o;
    return w;
}

// ---------------------------------------------------------------- persistent step
struct EnsArgs {
    int n;
    DevParams P;
    WcDev W;
    const int32_t *box_of;
    const float *box_dt, *H, *m, *x_build;
    float *x, *v, *rho;                    // state y0 (updated in place at the end of the step)
    float *x1, *v1, *rho1, *dv1, *drho1;   // stage state and first right-hand side
    float *gL, *Pr;                        // pass-A outputs of the current stage
    const int32_t *offs, *cnt, *list;
    BarrierCtl* ctl;
    unsigned int* disp;                    // max |x - x_build| / H since the list was built (ordered float)
    int32_t* status;
};

__device__ __forceinline__ unsigned int ens_ord(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
template <int D> __device__ __forceinline__ Vec<D> wrap_pos(Vec<D> x, const DomainF& dom) {
    #pragma unroll
    for (int a = 0; a < D; ++a)
        if (dom.periodic[a]) {
            if (x.v[a] >= dom.max[a]) x.v[a] -= dom.L[a];
            else if (x.v[a] < dom.min[a]) x.v[a] += dom.L[a];
        }
    return x;
}

template <int KF, int D, int G, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_ens_step(EnsArgs a) {
    constexpr int PPB = BLOCK / G;
    const int lane = threadIdx.x & (G - 1);
    const int rounds = (a.n + (int)gridDim.x * PPB - 1) / ((int)gridDim.x * PPB);
    unsigned int dmax = 0u;
    for (int stage = 0; stage < 2; ++stage) {
        const float* xs = stage == 0 ? a.x : a.x1;
        const float* vs = stage == 0 ? a.v : a.v1;
        const float* rs = stage == 0 ? a.rho : a.rho1;
        // ---- pass A: renormalised density gradient and EOS
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = (rd * (int)gridDim.x + (int)blockIdx.x) * PPB + (int)threadIdx.x / G;
            const bool valid = i < a.n;
            Mat<D> M = mzero<D>();
            Vec<D> s = vzero<D>();
            if (valid) passA_partial<KF, D, G, true>(i, lane, a.P, xs, a.H, a.m, rs, a.offs, a.cnt, a.list, M, s);
            passA_reduce<D, G>(M, s);
            if (valid && lane == 0) {
                store_vec<D>(a.gL, i, renormalise<D>(M, s));
                a.Pr[i] = wc_eos(a.W, __ldcg(rs + i));
            }
        }
        if (!grid_barrier(a.ctl)) { if (threadIdx.x == 0) atomicOr(a.status, SPH_STATUS_TIMEOUT); return; }
        // ---- pass B: right-hand side, stage update
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = (rd * (int)gridDim.x + (int)blockIdx.x) * PPB + (int)threadIdx.x / G;
            const bool valid = i < a.n;
            float cont = 0.f, dd = 0.f;
            Vec<D> pf = vzero<D>(), visc = vzero<D>();
            if (valid) passB_partial<KF, D, G, true>(i, lane, a.P, a.W, xs, a.H, a.m, rs, vs, a.gL, a.Pr, nullptr, a.offs, a.cnt,
                                                        a.list, cont, dd, pf, visc);
            cont = gsum<G>(cont); dd = gsum<G>(dd);
            #pragma unroll
            for (int c = 0; c < D; ++c) { pf.v[c] = gsum<G>(pf.v[c]); visc.v[c] = gsum<G>(visc.v[c]); }
            if (valid && lane == 0) {
                float dr; Vec<D> dv;
                passB_finish<D>(a.W, __ldcg(rs + i), a.H[i], cont, dd, pf, visc, dr, dv);
                const float dt = a.box_dt[a.box_of[i]];
                const Vec<D> x0 = ldv<D, true>(a.x, i), v0 = ldv<D, true>(a.v, i);
                const float r0 = __ldcg(a.rho + i);
                if (stage == 0) {
                    Vec<D> xn, vn;
                    #pragma unroll
                    for (int c = 0; c < D; ++c) { xn.v[c] = x0.v[c] + dt * v0.v[c]; vn.v[c] = v0.v[c] + dt * dv.v[c]; }
                    store_vec<D>(a.x1, i, wrap_pos<D>(xn, a.P.dom));
                    store_vec<D>(a.v1, i, vn);
                    a.rho1[i] = r0 + dt * dr;
                    store_vec<D>(a.dv1, i, dv);
                    a.drho1[i] = dr;
                } else {
                    const Vec<D> v1 = ldv<D, true>(a.v1, i), k1 = ldv<D, true>(a.dv1, i);
                    const float h = 0.5f * dt;
                    Vec<D> xn, vn;
                    #pragma unroll
                    for (int c = 0; c < D; ++c) { xn.v[c] = x0.v[c] + h * (v0.v[c] + v1.v[c]); vn.v[c] = v0.v[c] + h * (k1.v[c] + dv.v[c]); }
                    xn = wrap_pos<D>(xn, a.P.dom);
                    store_vec<D>(a.x, i, xn);
                    store_vec<D>(a.v, i, vn);
                    a.rho[i] = r0 + h * (__ldcg(a.drho1 + i) + dr);
                    const Vec<D> db = dist_vec<D>(xn, load_vec<D>(a.x_build, i), a.P.dom);
                    dmax = max(dmax, ens_ord(sqrtf(dot<D>(db, db)) / a.H[i]));   // in supports
                }
            }
        }
        if (stage == 0 && !grid_barrier(a.ctl)) { if (threadIdx.x == 0) atomicOr(a.status, SPH_STATUS_TIMEOUT); return; }
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0 && dmax) atomicMax(a.disp, dmax);
}

template <int KF, int D, int G, int BLOCK>
static int launch_ens(EnsArgs& a, cudaStream_t s) {
    static std::mutex mu;
    static int cached_dev = -1, bps = 0, sms = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "ensemble step: cudaGetDevice: %s", cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_dev != dev) {
            int coop = 0;
            if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
                return set_error(SPH_ERR_UNSUPPORTED, "ensemble step: device %d has no cooperative launch", dev);
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                return set_error(SPH_ERR_CUDA, "ensemble step: SM count");
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_ens_step<KF, D, G, BLOCK>, BLOCK, 0) != cudaSuccess || bps < 1)
                return set_error(SPH_ERR_CUDA, "ensemble step: occupancy query failed");
            cached_dev = dev;
        }
    }
    const int64_t need = (a.n + BLOCK / G - 1) / (BLOCK / G);
    const int grid = (int)std::min<int64_t>(need, (int64_t)bps * sms);
    void* args[] = {&a};
    count_launch();
    e = cudaLaunchCooperativeKernel((const void*)k_ens_step<KF, D, G, BLOCK>, dim3(grid), dim3(BLOCK), args, 0, s);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "ensemble step: cooperative launch: %s", cudaGetErrorString(e));
    return SPH_OK;
}

}  // namespace wsph

using namespace wsph;

extern "C" {

int64_t sph_ensemble_neighbors_workspace_size(int64_t n, int64_t total_cells) {
    if (n < 0 || total_cells < 1) return -1;
    return ens_carve(nullptr, n, total_cells).bytes;
}

int sph_ensemble_neighbors_build(const SphParams* p, int64_t n, int32_t nbox, const int32_t* box_of, const int32_t* box_grid,
                                 const int32_t* box_cell_base, int64_t total_cells, const float* x, const float* H, void* workspace,
                                 int64_t workspace_bytes, int32_t* offs, int32_t* cnt, int32_t* list, int64_t list_capacity,
                                 int64_t* nnz_out, int32_t* status, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff || nbox < 1 || total_cells < 1 || total_cells > 0x7fffffff)
        return set_error(SPH_ERR_BAD_ARG, "sph_ensemble_neighbors_build: bad sizes");
    WSPH_CHECK_PTR(nnz_out); WSPH_CHECK_PTR(status);
    cudaStream_t s = WSPH_STREAM(stream);
    if (n == 0) { cudaMemsetAsync(nnz_out, 0, 8, s); return check_launch("sph_ensemble_neighbors_build"); }
    WSPH_CHECK_PTR(box_of); WSPH_CHECK_PTR(box_grid); WSPH_CHECK_PTR(box_cell_base); WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H);
    WSPH_CHECK_PTR(workspace); WSPH_CHECK_PTR(offs); WSPH_CHECK_PTR(cnt);
    if (list_capacity > 0) WSPH_CHECK_PTR(list);
    if (P.dim == 2 && (reinterpret_cast<uintptr_t>(x) & 7)) return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    EnsNbWs w = ens_carve(static_cast<char*>(workspace), n, total_cells);
    if (workspace_bytes < w.bytes) return set_error(SPH_ERR_WORKSPACE, "ensemble neighbour workspace %lld < %lld", (long long)workspace_bytes,
                                                    (long long)w.bytes);
    cudaMemsetAsync(w.counts, 0, total_cells * 4, s);
    count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_ens_keys<D><<<grid_for(n, 256), 256, 0, s>>>((int)n, P.dom, x, box_of, box_grid, box_cell_base, w.keys,
                                                                              w.slot, w.counts)));
    exclusive_scan_i32(w.counts, w.start, total_cells, w.scan, w.total, s);
    count_launch();
    k_ens_scatter<<<grid_for(n, 256), 256, 0, s>>>((int)n, w.keys, w.slot, w.start, w.sorted);
    count_launch();
    k_ens_sort_cells<<<grid_for(total_cells, 256), 256, 0, s>>>(total_cells, w.start, w.counts, w.sorted);
    constexpr int GE = 8;
    count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_ens_verlet<D, GE, false><<<grid_for(n * GE, 128), 128, 0, s>>>(
        (int)n, P, x, H, box_of, box_grid, box_cell_base, w.start, w.counts, w.sorted, cnt, nullptr, nullptr, nullptr, 0)));
    exclusive_scan_i32(cnt, offs, n, w.scan, reinterpret_cast<long long*>(nnz_out), s);
    count_launch();
    k_ens_check<<<1, 1, 0, s>>>(reinterpret_cast<long long*>(nnz_out), list_capacity, status);
    count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_ens_verlet<D, GE, true><<<grid_for(n * GE, 128), 128, 0, s>>>(
        (int)n, P, x, H, box_of, box_grid, box_cell_base, w.start, w.counts, w.sorted, nullptr, offs, list,
        reinterpret_cast<long long*>(nnz_out), list_capacity)));
    return check_launch("sph_ensemble_neighbors_build");
}

int64_t sph_ensemble_step_workspace_size(int64_t n, int32_t dim) {
    if (n < 0 || dim < 1 || dim > 3) return -1;
    // control block, x1 v1 dv1 gL (n*dim each), rho1 drho1 Pr (n each)
    return 256 + 4 * al256(n * dim * 4) + 3 * al256(n * 4);
}

int sph_ensemble_step(const SphParams* p, const SphWcParams* wc, int64_t n, const int32_t* box_of, const float* box_dt,
                      const float* H, const float* m, float* x, float* v, float* rho, const float* x_build, const int32_t* offs,
                      const int32_t* cnt, const int32_t* list, void* workspace, int64_t workspace_bytes, int32_t lanes,
                      int32_t block, uint32_t* disp_max, int32_t* status, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x3fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_ensemble_step: n out of range");
    if (n == 0) return SPH_OK;
    WSPH_CHECK_PTR(wc); WSPH_CHECK_PTR(box_of); WSPH_CHECK_PTR(box_dt); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(x);
    WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(x_build); WSPH_CHECK_PTR(offs); WSPH_CHECK_PTR(cnt); WSPH_CHECK_PTR(list);
    WSPH_CHECK_PTR(workspace); WSPH_CHECK_PTR(disp_max); WSPH_CHECK_PTR(status);
    WcDev W;
    if ((rc = wc_to_dev(wc, P, &W))) return rc;
    if (workspace_bytes < sph_ensemble_step_workspace_size(n, P.dim)) return set_error(SPH_ERR_WORKSPACE, "sph_ensemble_step: workspace too small");
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return set_error(SPH_ERR_BAD_ARG, "sph_ensemble_step: workspace must be 256-byte aligned");
    if (P.dim == 2 && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(v) | reinterpret_cast<uintptr_t>(x_build)) & 7))
        return set_error(SPH_ERR_BAD_ARG, "vectors must be 8-byte aligned in 2D");
    cudaStream_t s = WSPH_STREAM(stream);
    char* w = static_cast<char*>(workspace);
    EnsArgs a;
    a.n = (int)n; a.P = P; a.W = W; a.box_of = box_of; a.box_dt = box_dt; a.H = H; a.m = m; a.x_build = x_build;
    a.x = x; a.v = v; a.rho = rho;
    int64_t o = 256;
    const int64_t vb = al256(n * P.dim * 4), sb = al256(n * 4);
    a.x1 = reinterpret_cast<float*>(w + o); o += vb;
    a.v1 = reinterpret_cast<float*>(w + o); o += vb;
    a.dv1 = reinterpret_cast<float*>(w + o); o += vb;
    a.gL = reinterpret_cast<float*>(w + o); o += vb;
    a.rho1 = reinterpret_cast<float*>(w + o); o += sb;
    a.drho1 = reinterpret_cast<float*>(w + o); o += sb;
    a.Pr = reinterpret_cast<float*>(w + o); o += sb;
    a.offs = offs; a.cnt = cnt; a.list = list;
    a.ctl = reinterpret_cast<BarrierCtl*>(w);
    a.disp = disp_max; a.status = status;
    cudaError_t e = cudaMemsetAsync(a.ctl, 0, sizeof(BarrierCtl), s);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_ensemble_step: memset: %s", cudaGetErrorString(e));
    if (!(lanes == 4 || lanes == 8 || lanes == 16) || !(block == 128 || block == 256))
        return set_error(SPH_ERR_BAD_ARG, "sph_ensemble_step: lanes must be 4, 8 or 16 and block 128 or 256");
    rc = SPH_ERR_UNSUPPORTED;
#define ENS_LAUNCH(GL, BL) WSPH_DISPATCH_KD(P.kernel, P.dim, (rc = launch_ens<KF, D, GL, BL>(a, s)))
    if (lanes == 4 && block == 128) { ENS_LAUNCH(4, 128); }
    else if (lanes == 4) { ENS_LAUNCH(4, 256); }
    else if (lanes == 8 && block == 128) { ENS_LAUNCH(8, 128); }
    else if (lanes == 8) { ENS_LAUNCH(8, 256); }
    else if (block == 128) { ENS_LAUNCH(16, 128); }
    else { ENS_LAUNCH(16, 256); }
#undef ENS_LAUNCH
    return rc;
}

}  // extern "C"
