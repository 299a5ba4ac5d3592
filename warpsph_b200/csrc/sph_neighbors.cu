// Neighbour search for libwarpsph_b200 and the library's host utilities.
//
// Replaces warpSPHCore's buildVerletList (compact hash + CUB radix sort in the
// reference, called at schemes/crkSPH.py:54-58).  Design:
//   1. cell size c >= verlet_scale * max(H) (device max-reduction, no host sync);
//      dense grid of G_d = floor(L_d / c) cells per axis, keyed by the Morton code
//      of the cell coordinate so that spatially close cells are close in memory.
//   2. counting sort by key: histogram (atomics), exclusive scan -> cell_begin,
//      atomic scatter, then a per-cell insertion sort by particle index, so the
//      permutation equals a stable sort by (key, index) -- deterministic and
//      bit-identical to the CPU oracle.
//   3. Verlet list as CSR: count pass, exclusive scan, fill pass.  One warp per
//      particle (in sorted order, over position/support records gathered in sorted
//      order) visits the 3^d stencil cells in offset order with lanes over the
//      candidates, keeps j when |x_i - x_j|^2 < (verlet_scale * max(H_i, H_j))^2
//      (explicit round-to-nearest operations, so the oracle reproduces it exactly)
//      and writes each row with ballot-compacted, coalesced stores.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <cuda_runtime.h>
#include "sph_common.cuh"
#include "sph_pair_common.cuh"

namespace wsph {

// ---------------------------------------------------------------- error handling
static thread_local char g_err[512] = "no error";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// launches recorded into the rebuild bodies of graph conditionals (they run only on a rebuild)
static std::atomic<long long> g_conditional_launches{0};

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return SPH_OK;
}

double kernel_norm(int kernel, int dim) {
    const double pi = 3.14159265358979323846;
    if (kernel == SPH_KERNEL_WENDLAND2) return dim == 1 ? 1.25 : (dim == 2 ? 7.0 / pi : 21.0 / (2.0 * pi));
    if (kernel == SPH_KERNEL_WENDLAND4) return dim == 1 ? 1.5 : (dim == 2 ? 9.0 / pi : 495.0 / (32.0 * pi));
    if (kernel == SPH_KERNEL_WENDLAND6) return dim == 1 ? 1.71875 : (dim == 2 ? 78.0 / (7.0 * pi) : 1365.0 / (64.0 * pi));
    if (kernel == SPH_KERNEL_B7) return dim == 1 ? 4096.0 / 315.0 : (dim == 2 ? 589824.0 / (7435.0 * pi) : 16384.0 / (105.0 * pi));
    return 0.0;
}

// Wendland kernels: H / h with h = 2 sigma, sigma^2 = (1/d) int |x|^2 W dx (Dehnen & Aly
// 2012, Table 1).  B7: the factor the reference's CFL time step divides by, read from its
// notebooks' printed initial time steps (1D: Woodward-Colella, 2D: Gresho-Chan, where the
// step depends only on this factor, the support and the sound speed); 3D continues the
// 1D -> 2D ratio, which equals the quintic B-spline's sqrt(d I_(d-1) / I_(d+1)) ratio
// (I_n = int_0^1 k(q) q^n dq) to 7e-8, by that spline's 3D/1D ratio sqrt(15/14).
double kernel_scale(int kernel, int dim) {
    static const double t[4][3] = {
        {1.620185175, 1.897366596, 1.936491673},
        {1.936491673, 2.171240593, 2.207940217},
        {2.207940217, 2.415229458, 2.449489743},
        {3.865656972, 3.932734728, 4.001335111}};
    if (kernel < 1 || kernel > 4 || dim < 1 || dim > 3) return 0.0;
    return t[kernel - 1][dim - 1];
}

int params_to_dev(const SphParams* p, DevParams* o) {
    if (!p) return set_error(SPH_ERR_BAD_ARG, "null SphParams");
    if (p->dim < 1 || p->dim > 3) return set_error(SPH_ERR_BAD_ARG, "dim must be 1..3 (got %d)", p->dim);
    if (p->kernel < SPH_KERNEL_WENDLAND2 || p->kernel > SPH_KERNEL_B7)
        return set_error(SPH_ERR_BAD_ARG, "unsupported kernel id %d", p->kernel);
    memset(o, 0, sizeof(*o));
    o->dim = p->dim;
    o->kernel = p->kernel;
    for (int a = 0; a < 3; ++a) {
        o->dom.min[a] = (float)p->domain_min[a];
        o->dom.max[a] = (float)p->domain_max[a];
        o->dom.L[a] = (float)(p->domain_max[a] - p->domain_min[a]);
        o->dom.halfL[a] = 0.5f * o->dom.L[a];
        o->dom.periodic[a] = p->periodic[a] ? 1 : 0;
        if (a < p->dim && !(o->dom.L[a] > 0.f)) return set_error(SPH_ERR_BAD_ARG, "domain extent along axis %d must be > 0", a);
    }
    o->verlet_scale = (float)p->verlet_scale;
    if (!(o->verlet_scale >= 1.f)) return set_error(SPH_ERR_BAD_ARG, "verlet_scale must be >= 1");
    o->C_l = (float)p->C_l; o->C_q = (float)p->C_q; o->Cu_l = (float)p->Cu_l; o->Cu_q = (float)p->Cu_q; o->K = (float)p->K;
    o->viscosity_term = p->viscosity_term;
    o->monaghan_switch = p->monaghan_switch; o->correct_xi = p->correct_xi; o->scale_beta = p->scale_beta;
    o->eta_crit = (float)p->eta_crit; o->eta_fold = (float)p->eta_fold;
    o->enable_crk_limiter = p->enable_crk_limiter; o->enable_vanleer = p->enable_vanleer_limiter;
    o->force_vl_off = p->force_vanleer_off; o->force_vl_on = p->force_vanleer_on;
    o->gamma = (float)p->gamma;
    o->energy_scheme = p->energy_scheme; o->limit_xi = p->limit_xi; o->kahan = p->kahan;
    o->correct_grad_v = p->correct_velocity_gradient;
    o->alpha_min = (float)p->alpha_min; o->alpha_max = (float)p->alpha_max; o->beta_xi = (float)p->beta_xi;
    o->target_neighbors = (float)p->target_neighbors;
    o->cfl = (float)p->cfl; o->min_dt = (float)p->min_dt; o->max_dt = (float)p->max_dt; o->dt_growth = (float)p->dt_growth;
    o->c_s = (float)p->c_s;
    o->beta_c = (float)p->beta_c; o->beta_d = (float)p->beta_d;
    o->conductivity_term = p->conductivity_term;
    if (p->viscosity_term < SPH_VISC_DEFAULT || p->viscosity_term > SPH_VISC_DELTASPH)
        return set_error(SPH_ERR_BAD_ARG, "viscosity_term %d out of range", p->viscosity_term);
    if (p->conductivity_term < SPH_VISC_DEFAULT || p->conductivity_term > SPH_VISC_DELTASPH)
        return set_error(SPH_ERR_BAD_ARG, "conductivity_term %d out of range", p->conductivity_term);
    o->kscale = (float)kernel_scale(p->kernel, p->dim);
    o->kxi = o->kscale;
    return SPH_OK;
}

// ---------------------------------------------------------------- list verdict
// Ordered encoding of floats into unsigned words (atomicMax on the words is a max on the
// floats), and the validity verdict of a kept Verlet list (k_refresh_check below reduces
// the three words).
__device__ __forceinline__ unsigned int ord_enc(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_dec(unsigned int o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
__device__ __forceinline__ bool refresh_valid(const unsigned int* acc3) {
    const float dmax = ord_dec(acc3[0]), amax = ord_dec(acc3[1]), hmax = ord_dec(acc3[2]);
    return amax + 1.0002f * dmax + 1e-5f * hmax <= 0.f;   // false for NaN
}
// Gate of the device-decided list update (sph_neighbors_update): a build kernel given
// the verdict words returns at once when they say the kept list is still valid, so the
// rebuild is decided on the GPU with no host read.  A null gate always runs.
__device__ __forceinline__ bool gate_closed(const unsigned int* gate) { return gate != nullptr && refresh_valid(gate); }

// ---------------------------------------------------------------- scan
// Exclusive scan of int32 values with an int64 grand total.  Block-level scans of
// 2048 items (256 threads x 8), recursive over block sums.
static constexpr int SCAN_THREADS = 256;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* smem_warp, long long& total) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        long long w = (lane < SCAN_THREADS / 32) ? smem_warp[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) smem_warp[lane] = w;
    }
    __syncthreads();
    long long warp_off = warp > 0 ? smem_warp[warp - 1] : 0;
    total = smem_warp[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return warp_off + x - v;
}

// in -> out (exclusive, local to tile), tile totals -> sums
__global__ void k_scan_tiles(const int32_t* __restrict__ in, int64_t n, long long* __restrict__ out_ll,
                             int32_t* __restrict__ out32, long long* __restrict__ sums, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    __shared__ long long sw[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    long long vals[SCAN_ITEMS];
    long long local = 0;
    #pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t idx = base + k;
        vals[k] = idx < n ? (long long)in[idx] : 0;
        local += vals[k];
    }
    long long total;
    long long off = block_exclusive_scan(local, sw, total);
    #pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t idx = base + k;
        if (idx < n) {
            if (out_ll) out_ll[idx] = off; else out32[idx] = (int32_t)off;
        }
        off += vals[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
// in and out may alias (in-place scan of tile sums): no __restrict__ here.
__global__ void k_scan_tiles_ll(const long long* in, int64_t n, long long* out, long long* __restrict__ sums,
                                const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    __shared__ long long sw[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    long long vals[SCAN_ITEMS];
    long long local = 0;
    #pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t idx = base + k;
        vals[k] = idx < n ? in[idx] : 0;
        local += vals[k];
    }
    long long total;
    long long off = block_exclusive_scan(local, sw, total);
    #pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t idx = base + k;
        if (idx < n) out[idx] = off;
        off += vals[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void k_scan_add(long long* __restrict__ out_ll, int32_t* __restrict__ out32, int64_t n,
                           const long long* __restrict__ tile_off, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    long long o = tile_off[idx / SCAN_TILE];
    if (out_ll) out_ll[idx] += o; else out32[idx] = (int32_t)((long long)out32[idx] + o);
}

// Workspace: for each level the tile sums and their scanned offsets.
int64_t scan_ws_bytes(int64_t n) {
    int64_t bytes = 0;
    int64_t m = n;
    do {
        int64_t tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
        if (tiles < 1) tiles = 1;
        bytes += 2 * ((tiles * 8 + 255) / 256) * 256;
        m = tiles;
    } while (m > 1);
    return bytes + 256;
}

__global__ void k_copy_total(long long* __restrict__ total, const long long* __restrict__ sums, const unsigned int* __restrict__ gate) {
    if (!gate_closed(gate)) *total = *sums;
}

// The single-tile total: a device copy, or under a gate a one-thread kernel (a copy
// cannot be skipped by the GPU).
static void copy_total(long long* total, const long long* sums, const unsigned int* gate, cudaStream_t s) {
    if (gate) {
        wsph::count_launch(); k_copy_total<<<1, 1, 0, s>>>(total, sums, gate);
    } else {
        cudaMemcpyAsync(total, sums, sizeof(long long), cudaMemcpyDeviceToDevice, s);
    }
}

// Scans a level of long long values in place (exclusive) and writes the total to *total.
static void scan_ll_inplace(long long* data, int64_t n, char* ws, long long* total, cudaStream_t s, const unsigned int* gate) {
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles < 1) tiles = 1;
    long long* sums = reinterpret_cast<long long*>(ws);
    char* next = ws + ((tiles * 8 + 255) / 256) * 256 * 2;
    wsph::count_launch(); k_scan_tiles_ll<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(data, n, data, sums, gate);
    if (tiles == 1) {
        copy_total(total, sums, gate, s);
        return;
    }
    scan_ll_inplace(sums, tiles, next, total, s, gate);
    wsph::count_launch(); k_scan_add<<<grid_for(n, 256), 256, 0, s>>>(data, nullptr, n, sums, gate);
}

// Exclusive scan int32 -> int32, total (int64, device).  Under a gate every launch
// returns at once when the gate is closed, leaving out and total as they were.
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, char* ws, long long* total, cudaStream_t s,
                        const unsigned int* gate) {
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles < 1) tiles = 1;
    long long* sums = reinterpret_cast<long long*>(ws);
    char* next = ws + ((tiles * 8 + 255) / 256) * 256 * 2;
    wsph::count_launch(); k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, nullptr, out, sums, gate);
    if (tiles == 1) {
        copy_total(total, sums, gate, s);
        return;
    }
    scan_ll_inplace(sums, tiles, next, total, s, gate);
    wsph::count_launch(); k_scan_add<<<grid_for(n, 256), 256, 0, s>>>(nullptr, out, n, sums, gate);
}

// ---------------------------------------------------------------- min / max
__global__ void k_minmax_init(float* out2) { out2[0] = __int_as_float(0x7f800000); out2[1] = -__int_as_float(0x7f800000); }

__device__ __forceinline__ void atomic_min_float(float* addr, float v) {
    // ordered-int trick valid for non-NaN floats of any sign
    if (v >= 0.f) atomicMin(reinterpret_cast<int*>(addr), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_float(float* addr, float v) {
    if (v >= 0.f) atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

__global__ void k_minmax(const float* __restrict__ a, int64_t n, float* out2) {
    float lo = __int_as_float(0x7f800000), hi = -lo;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = a[i];
        lo = fminf(lo, v); hi = fmaxf(hi, v);
    }
    lo = block_reduce(lo, __int_as_float(0x7f800000), OpMinF());
    hi = block_reduce(hi, -__int_as_float(0x7f800000), OpMaxF());
    if (threadIdx.x == 0) { atomic_min_float(out2, lo); atomic_max_float(out2 + 1, hi); }
}

int launch_minmax(int64_t n, const float* a, float* out2, cudaStream_t s) {
    wsph::count_launch(); k_minmax_init<<<1, 1, 0, s>>>(out2);
    int blocks = (int)((n + 1023) / 1024);        // about four elements per thread
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (blocks < 1) blocks = 1;
    wsph::count_launch(); k_minmax<<<blocks, 256, 0, s>>>(a, n, out2);
    return check_launch("sph_minmax");
}

// ---------------------------------------------------------------- grid
struct GridDev {
    int G[3];
    int bits[3];
    float inv[3];   // G_d / L_d
    float cell;     // requested cell size (>= verlet_scale * max H)
};

__device__ __forceinline__ uint32_t spread2(uint32_t x) {  // 16 bits -> even positions
    x &= 0x0000ffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third position
    x &= 0x000003ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
template <int D> __device__ __forceinline__ uint32_t morton(const int* c) {
    if constexpr (D == 1) return (uint32_t)c[0];
    else if constexpr (D == 2) return spread2((uint32_t)c[0]) | (spread2((uint32_t)c[1]) << 1);
    else return spread3((uint32_t)c[0]) | (spread3((uint32_t)c[1]) << 1) | (spread3((uint32_t)c[2]) << 2);
}

template <int D> __device__ __forceinline__ void cell_coords(const Vec<D>& x, const GridDev& g, const DomainF& dom, int* c) {
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        float t = __fmul_rn(__fsub_rn(x.v[a], dom.min[a]), g.inv[a]);
        int ci = (int)floorf(t);
        ci = ci < 0 ? 0 : (ci >= g.G[a] ? g.G[a] - 1 : ci);
        c[a] = ci;
    }
}

__global__ void k_hmax(const float* __restrict__ H, int64_t n, float* out, int32_t* status, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    float hi = 0.f;
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float h = H[i];
        if (!(h > 0.f) || isinf(h)) bad = true; else hi = fmaxf(hi, h);
    }
    hi = block_reduce(hi, 0.f, OpMaxF());
    if (threadIdx.x == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(hi));
    if (bad) atomicOr(status, SPH_STATUS_NONFINITE);
}

// One thread: derive the grid from max H and the cell-table capacity.
template <int D>
__global__ void k_grid(const float* hmax, DevParams P, int max_bits, GridDev* g, int32_t* grid_out, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    float h = *hmax;
    float Lmax = 0.f;
    for (int a = 0; a < D; ++a) Lmax = fmaxf(Lmax, P.dom.L[a]);
    // margin keeps the 3^d stencil exact despite rounding of the cell coordinate
    float cell = __fadd_rn(__fmul_rn(__fmul_rn(P.verlet_scale, h), 1.001f), __fmul_rn(Lmax, 1e-6f));
    GridDev G;
    for (int a = 0; a < 3; ++a) { G.G[a] = 1; G.bits[a] = 0; G.inv[a] = 0.f; }
    for (int a = 0; a < D; ++a) {
        float f = floorf(P.dom.L[a] / cell);
        int gmax = 1 << max_bits;
        int gi = (f >= (float)gmax) ? gmax : (f < 1.f ? 1 : (int)f);
        int b = 0;
        while ((1 << b) < gi) ++b;
        G.G[a] = gi;
        G.bits[a] = b;
        G.inv[a] = __fdiv_rn((float)gi, P.dom.L[a]);
    }
    G.cell = cell;
    *g = G;
    for (int a = 0; a < 3; ++a) { grid_out[a] = G.G[a]; grid_out[3 + a] = G.bits[a]; }
    grid_out[6] = __float_as_int(cell);
    grid_out[7] = D;
}

template <int D>
__global__ void k_keys(const float* __restrict__ x, int n, const GridDev* __restrict__ gp, DomainF dom,
                       uint32_t* __restrict__ keys, int32_t* __restrict__ counts, const unsigned int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || gate_closed(gate)) return;
    GridDev g = *gp;
    int c[3];
    cell_coords<D>(load_vec<D>(x, i), g, dom, c);
    uint32_t key = morton<D>(c);
    keys[i] = key;
    atomicAdd(counts + key, 1);
}

__global__ void k_scatter(const uint32_t* __restrict__ keys, int n, int32_t* __restrict__ cursor, int32_t* __restrict__ sort_index,
                          const unsigned int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || gate_closed(gate)) return;
    int pos = atomicAdd(cursor + keys[i], 1);
    sort_index[pos] = i;
}

// Canonical order inside a cell: ascending particle index.  After the atomic
// scatter each cell holds its particles in arbitrary order; every particle's final
// slot is begin[cell] + (number of cell members with a smaller index).  The pass
// also writes the sorted keys and packs (x, H) into sorted float4 records that the
// Verlet walk reads contiguously.
template <int D>
__global__ void k_rank_sort(const int32_t* __restrict__ tmp, const uint32_t* __restrict__ keys,
                            const int32_t* __restrict__ begin, const int32_t* __restrict__ end, int n,
                            const float* __restrict__ x, const float* __restrict__ H,
                            int32_t* __restrict__ sort_index, uint32_t* __restrict__ sorted_keys, float4* __restrict__ recs,
                            int32_t* __restrict__ tasks, int32_t* __restrict__ ntasks, const unsigned int* __restrict__ gate) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || gate_closed(gate)) return;
    int i = tmp[k];
    uint32_t c = keys[i];
    int b = begin[c], e = end[c];
    int rank = 0;
    for (int m = b; m < e; ++m) rank += tmp[m] < i;
    int slot = b + rank;
    if (rank == 0) {   // the cell's first particle appends its work items (chunks of <= 32 sorted positions)
        int nch = (e - b + 31) >> 5;
        int t0 = atomicAdd(ntasks, nch);
        for (int q = 0; q < nch; ++q) tasks[t0 + q] = b + 32 * q;
    }
    sort_index[slot] = i;
    sorted_keys[slot] = c;
    Vec<D> xi = load_vec<D>(x, i);
    float4 r = make_float4(xi.v[0], D > 1 ? xi.v[D > 1 ? 1 : 0] : 0.f, D > 2 ? xi.v[D > 2 ? 2 : 0] : 0.f, H[i]);
    recs[slot] = r;
}

template <int D> __device__ __forceinline__ Vec<D> rec_pos(const float4& r) {
    Vec<D> v;
    v.v[0] = r.x;
    if constexpr (D > 1) v.v[1] = r.y;
    if constexpr (D > 2) v.v[2] = r.z;
    return v;
}

// Stencil of neighbour cell keys in offset order (x fastest, offsets -1, 0, +1 per
// axis), periodic axes wrapped, cells outside a non-periodic grid skipped, and a cell
// reached twice (fewer than three cells along a periodic axis) kept only once.
// shift[q*3+a] is the periodic image offset of stencil cell q along axis a (-L, 0, +L):
// with at least three cells per axis, x_i - x_j - shift is the minimum-image
// difference for every pair within one cell width, bit-identical to the per-pair test
// of dist_vec (x - 0 = x exactly).  With fewer than three cells along an axis one cell
// is reached through two images and a single shift cannot serve every pair in it; the
// walk then takes the minimum image pair by pair (see grid_needs_min_image).
template <int D>
__device__ __forceinline__ bool grid_needs_min_image(const GridDev& g, const DomainF& dom) {
    bool r = false;
    #pragma unroll
    for (int a = 0; a < D; ++a) r |= dom.periodic[a] && g.G[a] < 3;
    return r;
}

template <int D>
__device__ __forceinline__ int stencil_keys(const int* c, const GridDev& g, const DomainF& dom, uint32_t* out, float* shift) {
    int cnt = 0;
    constexpr int NS = D == 1 ? 3 : (D == 2 ? 9 : 27);
    bool dedupe = false;
    #pragma unroll
    for (int a = 0; a < D; ++a) dedupe |= g.G[a] < 3;
    #pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int o[3] = {s % 3 - 1, (s / 3) % 3 - 1, (s / 9) % 3 - 1};
        int cc[3];
        float sh[3] = {0.f, 0.f, 0.f};
        bool ok = true;
        #pragma unroll
        for (int a = 0; a < D; ++a) {
            int v = c[a] + o[a];
            if (v < 0) {
                if (dom.periodic[a]) { v += g.G[a]; sh[a] = -dom.L[a]; } else ok = false;
            } else if (v >= g.G[a]) {
                if (dom.periodic[a]) { v -= g.G[a]; sh[a] = dom.L[a]; } else ok = false;
            }
            cc[a] = v;
        }
        uint32_t k = morton<D>(cc);
        if (ok && dedupe) {
            for (int q = 0; q < cnt; ++q) ok = ok && out[q] != k;
        }
        if (ok) {
            #pragma unroll
            for (int a = 0; a < 3; ++a) shift[cnt * 3 + a] = sh[a];
            out[cnt++] = k;
        }
    }
    return cnt;
}

// Verlet list walk, one warp per work item: up to 32 particles of one cell, lane l
// owning sorted position start+l.  All lanes share the cell and hence the 3^d stencil
// and every loop bound (no divergence).  Candidate records of each stencil cell are
// staged through shared memory 32 at a time (one coalesced load, broadcast reads).
// A Verlet entry needs r^2 < (verlet_scale*max(H_i,H_j))^2.
//
// Row layout (when interacting counts are requested): the interacting entries --
// fl(sqrt(r^2))/max(H_i,H_j) < 1, exactly the pairs some support scheme gives W != 0 --
// come first, then the rest of the Verlet entries, each part in walk order (stencil
// cells in offset order, candidates by sorted position).  The pair passes walk only
// the prefix [offset, offset + interacting count): plain int32 indices, and pairwise
// outputs written contiguously at their Verlet entry.  The count pass counts both
// parts, so the fill pass knows where each row's tail starts.  Rows are staged in
// shared memory (VS entries per lane and part) and flushed by the warp cooperatively,
// so they are written with contiguous stores.
constexpr int VW_WARPS = 4;
constexpr int VW_BLOCK = 32 * VW_WARPS;
constexpr int VS = 16;
// Row pitch of the staging buffers: one word more than VS, so that the 32 lanes'
// stores of their next entry fall in 32 different banks (with a pitch of 16 words the
// even and the odd lanes would each share one bank, a 16-way conflict per store).
constexpr int VP = VS + 1;

// fl(sqrt(r2)) / Hm < 1, with the square root only inside a narrow band around r = Hm
// (outside it the comparison of r2 with Hm^2 decides the same way).  For positive finite
// a and b, fl(a / b) < 1 exactly when a < b (a < b gives a / b <= 1 - 2^-24, the float
// next below 1, so a / b never rounds up to 1), so the test is fl(sqrt(r2)) < Hm.
__device__ __forceinline__ bool interacting_pair(float r2, float Hm) {
    const float h2 = Hm * Hm;
    if (r2 < 0.9998f * h2) return true;
    if (!(r2 < 1.0002f * h2)) return false;
    return sqrtf(r2) < Hm;
}

// Writes every lane's staged entries of one part: lanes pair up per owner row (16
// entries per half warp), base_o + e for the owner's base.
__device__ __forceinline__ void verlet_flush_part(int lane, int wib, int& nb, int& written, int base,
                                                  int32_t (*buf)[32][VP], int32_t* __restrict__ list) {
    const int half = lane >> 4, e = lane & 15;
    #pragma unroll 4
    for (int r = 0; r < 32; r += 2) {
        const int owner = r + half;
        const int n_o = __shfl_sync(0xffffffffu, nb, owner);
        const int b_o = __shfl_sync(0xffffffffu, base + written, owner);
        if (e < n_o) list[b_o + e] = buf[wib][owner][e];
    }
    written += nb;
    nb = 0;
}

// One work item of the walk (32 particles of one cell against its stencil).  MI: the grid
// has fewer than three cells along a periodic axis, and every pair takes its minimum image
// (rare, tiny grids; kept out of line so the common loop stays compact).  Candidate slots
// past the end of a cell hold a record at 3e38, which no test accepts, so the unrolled
// candidate loop needs no bound check.
//
// Acceptance bits (masks non-null, not MI): the count pass reserves 64 words per candidate
// chunk of its work item from a bounded pool and stores each lane's 32 acceptance bits and 32
// interacting bits per chunk; the fill pass then walks the candidates that some lane accepted,
// in the same order, and files each into the interacting prefix or the rest from the bits,
// without distance arithmetic.  A work item that found the pool exhausted tests every
// candidate again.
template <int D, bool MI, bool SH = true>
__device__ __forceinline__ void verlet_pair(const Vec<D>& xi, float Hi, const float4& rj, const float* sh, const DomainF& dom,
                                            float vs, float& r2, float& Hm, float& R) {
    Hm = fmaxf(Hi, rj.w);
    R = __fmul_rn(vs, Hm);
    Vec<D> dv;
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        const float xj = a == 0 ? rj.x : (a == 1 ? rj.y : rj.z);
        if (MI) {
            float d = __fsub_rn(xi.v[a], xj);
            if (dom.periodic[a]) {
                if (d > dom.halfL[a]) d = __fsub_rn(d, dom.L[a]);
                else if (d < -dom.halfL[a]) d = __fadd_rn(d, dom.L[a]);
            }
            dv.v[a] = d;
        } else if (SH) {
            dv.v[a] = __fsub_rn(__fsub_rn(xi.v[a], xj), sh[a]);
        } else {
            dv.v[a] = __fsub_rn(xi.v[a], xj);     // equal to the above with sh = 0 (x - 0 = x exactly)
        }
    }
    r2 = dist2_rn<D>(dv);
}

// The count pass over one staged chunk: acceptance and interacting bits of the lane's
// particle against the (up to 32) staged candidates; padded slots never match.
template <int D, bool MI, bool SH>
__device__ __forceinline__ void verlet_count_chunk(const Vec<D>& xi, float Hi, bool active, bool part, const float4* __restrict__ sr,
                                                   const float* sh, const DomainF& dom, float vs, int mcount, uint32_t& hm,
                                                   uint32_t& im) {
    for (int u0 = 0; u0 < mcount; u0 += 8) {
        #pragma unroll
        for (int du = 0; du < 8; ++du) {
            const int u = u0 + du;
            float r2, Hm, R;
            verlet_pair<D, MI, SH>(xi, Hi, sr[u], sh, dom, vs, r2, Hm, R);
            const bool hit = active & (r2 < __fmul_rn(R, R));
            hm |= hit ? (1u << u) : 0u;
            if (part) im |= (hit && interacting_pair(r2, Hm)) ? (1u << u) : 0u;
        }
    }
}

template <int D, bool FILL, bool MI>
__device__ __forceinline__ void verlet_task(int task, int lane, int wib, const float4* __restrict__ recs,
                                            const uint32_t* __restrict__ sorted_keys, const int32_t* __restrict__ tasks,
                                            const GridDev& g, const DevParams& P, const int32_t* __restrict__ sort_index,
                                            const int32_t* __restrict__ cell_begin, const int32_t* __restrict__ cell_end,
                                            int32_t* __restrict__ counts, int32_t* __restrict__ icounts,
                                            const int32_t* __restrict__ offsets, int32_t* __restrict__ list, long long& itotal,
                                            float4 (*srec)[32], int32_t (*sidx)[32], int32_t (*sbuf)[32][VP],
                                            int32_t (*sibuf)[32][VP], uint32_t* __restrict__ masks,
                                            int32_t* __restrict__ mask_base, unsigned long long* __restrict__ mask_cursor,
                                            long long mask_words) {
    const bool part = icounts != nullptr;
    const DomainF& dom = P.dom;
    const float vs = P.verlet_scale;
    const int start = tasks[task];
    const uint32_t ckey = sorted_keys[start];
    const int stop = min(start + 32, cell_end[ckey]);
    const int t = start + lane;
    const bool active = t < stop;
    const float4 ri = recs[active ? t : start];
    const Vec<D> xi = rec_pos<D>(ri);
    const float Hi = ri.w;
    int c[3];
    cell_coords<D>(rec_pos<D>(recs[start]), g, dom, c);
    uint32_t keys[D == 1 ? 3 : (D == 2 ? 9 : 27)];
    float shifts[3 * (D == 1 ? 3 : (D == 2 ? 9 : 27))];
    const int nk = stencil_keys<D>(c, g, dom, keys, shifts);
    const int i = active ? sort_index[t] : 0;
    int cnt = 0, icnt = 0;
    int row = 0, tail = 0, nb = 0, nib = 0, written = 0, iwritten = 0;
    if (FILL && active) {
        row = offsets[i];
        tail = row + (part ? icounts[i] : 0);
    }
    // the work item's slice of the acceptance-bit pool
    int mbase = -1;
    if (!MI && masks != nullptr) {
        if (!FILL) {
            int nch = 0;
            for (int q = 0; q < nk; ++q) nch += (cell_end[keys[q]] - cell_begin[keys[q]] + 31) >> 5;
            if (lane == 0) {
                const unsigned long long need = 64ull * (unsigned long long)nch;
                const unsigned long long o = atomicAdd(mask_cursor, need);
                mbase = o + need <= (unsigned long long)mask_words ? (int)o : -1;
                mask_base[task] = mbase;
            }
            mbase = __shfl_sync(0xffffffffu, mbase, 0);
        } else {
            mbase = mask_base[task];
        }
    }
    const float4 far = make_float4(3e38f, 3e38f, 3e38f, 0.f);
    int ch = 0;
    for (int q = 0; q < nk; ++q) {
        const int b = cell_begin[keys[q]], e = cell_end[keys[q]];
        const float sh[3] = {shifts[3 * q], shifts[3 * q + 1], shifts[3 * q + 2]};
        for (int k0 = b; k0 < e; k0 += 32, ++ch) {
            if (FILL && mbase >= 0) {
                const uint32_t m = active ? masks[mbase + 64 * ch + lane] : 0u;
                const uint32_t im = active ? masks[mbase + 64 * ch + 32 + lane] : 0u;
                uint32_t U = __reduce_or_sync(0xffffffffu, m);
                if (U == 0u) continue;
                __syncwarp();
                if (k0 + lane < e) sidx[wib][lane] = sort_index[k0 + lane];
                __syncwarp();
                // the candidates some lane accepted, in candidate order; each lane files at
                // most one entry per candidate, so 8 candidates fit between two flushes
                for (int r = 0; U != 0u; ++r) {
                    if ((r & 7) == 0 && __any_sync(0xffffffffu, nb > VS - 8 || nib > VS - 8)) {
                        __syncwarp();
                        verlet_flush_part(lane, wib, nib, iwritten, row, sibuf, list);
                        verlet_flush_part(lane, wib, nb, written, tail, sbuf, list);
                        __syncwarp();
                    }
                    const int u = __ffs(U) - 1;
                    U &= U - 1u;
                    if ((m >> u) & 1u) {
                        const int j = sidx[wib][u];
                        if ((im >> u) & 1u) sibuf[wib][lane][nib++] = j;
                        else sbuf[wib][lane][nb++] = j;
                    }
                }
                continue;
            }
            __syncwarp();
            const bool real = k0 + lane < e;
            srec[wib][lane] = real ? recs[k0 + lane] : far;
            if (FILL && real) sidx[wib][lane] = sort_index[k0 + lane];
            __syncwarp();
            const int mcount = min(32, e - k0);
            if constexpr (!FILL) {
                uint32_t hm = 0, im = 0;
                if (!MI && sh[0] == 0.f && sh[1] == 0.f && sh[2] == 0.f)
                    verlet_count_chunk<D, MI, false>(xi, Hi, active, part, srec[wib], sh, dom, vs, mcount, hm, im);
                else
                    verlet_count_chunk<D, MI, true>(xi, Hi, active, part, srec[wib], sh, dom, vs, mcount, hm, im);
                cnt += __popc(hm);
                icnt += __popc(im);
                if (mbase >= 0) {
                    masks[mbase + 64 * ch + lane] = hm;
                    masks[mbase + 64 * ch + 32 + lane] = im;
                }
            } else {
            for (int u0 = 0; u0 < mcount; u0 += 8) {
                // room for the next 8 candidates in every lane's buffers
                if (FILL && __any_sync(0xffffffffu, nb > VS - 8 || nib > VS - 8)) {
                    __syncwarp();
                    verlet_flush_part(lane, wib, nib, iwritten, row, sibuf, list);
                    verlet_flush_part(lane, wib, nb, written, tail, sbuf, list);
                    __syncwarp();
                }
                #pragma unroll
                for (int du = 0; du < 8; ++du) {
                    const int u = u0 + du;
                    float r2, Hm, R;
                    verlet_pair<D, MI>(xi, Hi, srec[wib][u], sh, dom, vs, r2, Hm, R);
                    const bool hit = active & (r2 < __fmul_rn(R, R));
                    const bool inter = part && hit && interacting_pair(r2, Hm);
                    if (hit) {
                        const int j = sidx[wib][u];
                        if (inter) sibuf[wib][lane][nib++] = j;
                        else sbuf[wib][lane][nb++] = j;
                    }
                }
            }
            }
        }
    }
    if (FILL) {
        if (__any_sync(0xffffffffu, nb > 0 || nib > 0)) {
            __syncwarp();
            verlet_flush_part(lane, wib, nib, iwritten, row, sibuf, list);
            verlet_flush_part(lane, wib, nb, written, tail, sbuf, list);
            __syncwarp();
        }
    } else if (active) {
        counts[i] = cnt;
        if (part) icounts[i] = icnt;
        itotal += icnt;
    }
}

template <int D, bool FILL>
__device__ __noinline__ void verlet_task_min_image(int task, int lane, int wib, const float4* __restrict__ recs,
                                                   const uint32_t* __restrict__ sorted_keys, const int32_t* __restrict__ tasks,
                                                   const GridDev& g, const DevParams& P, const int32_t* __restrict__ sort_index,
                                                   const int32_t* __restrict__ cell_begin, const int32_t* __restrict__ cell_end,
                                                   int32_t* __restrict__ counts, int32_t* __restrict__ icounts,
                                                   const int32_t* __restrict__ offsets, int32_t* __restrict__ list, long long& itotal,
                                                   float4 (*srec)[32], int32_t (*sidx)[32], int32_t (*sbuf)[32][VP],
                                                   int32_t (*sibuf)[32][VP]) {
    verlet_task<D, FILL, true>(task, lane, wib, recs, sorted_keys, tasks, g, P, sort_index, cell_begin, cell_end, counts, icounts,
                               offsets, list, itotal, srec, sidx, sbuf, sibuf, nullptr, nullptr, nullptr, 0);
}

template <int D, bool FILL>
__global__ void __launch_bounds__(VW_BLOCK)
k_verlet(const float4* __restrict__ recs, const uint32_t* __restrict__ sorted_keys, const int32_t* __restrict__ tasks,
         const int32_t* __restrict__ ntasks, const GridDev* __restrict__ gp, DevParams P,
         const int32_t* __restrict__ sort_index, const int32_t* __restrict__ cell_begin, const int32_t* __restrict__ cell_end,
         int32_t* __restrict__ counts, int32_t* __restrict__ icounts, const int32_t* __restrict__ offsets,
         int32_t* __restrict__ list, long long* __restrict__ innz, const long long* __restrict__ nnz, long long capacity,
         uint32_t* __restrict__ masks, int32_t* __restrict__ mask_base, unsigned long long* __restrict__ mask_cursor,
         long long mask_words, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    __shared__ float4 srec[VW_WARPS][32];
    __shared__ int32_t sidx[FILL ? VW_WARPS : 1][32];
    __shared__ int32_t sbuf[FILL ? VW_WARPS : 1][32][VP];     // rest of the row
    __shared__ int32_t sibuf[FILL ? VW_WARPS : 1][32][VP];    // interacting prefix
    const bool part = icounts != nullptr;
    if (FILL && *nnz > capacity) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nt = *ntasks;
    const GridDev g = *gp;
    const bool min_image = grid_needs_min_image<D>(g, P.dom);     // uniform over the grid
    long long itotal = 0;
    for (int task = warp; task < nt; task += nwarps) {
        if (min_image)
            verlet_task_min_image<D, FILL>(task, lane, wib, recs, sorted_keys, tasks, g, P, sort_index, cell_begin, cell_end, counts,
                                           icounts, offsets, list, itotal, srec, FILL ? sidx : nullptr, FILL ? sbuf : nullptr,
                                           FILL ? sibuf : nullptr);
        else
            verlet_task<D, FILL, false>(task, lane, wib, recs, sorted_keys, tasks, g, P, sort_index, cell_begin, cell_end, counts,
                                        icounts, offsets, list, itotal, srec, FILL ? sidx : nullptr, FILL ? sbuf : nullptr,
                                        FILL ? sibuf : nullptr, masks, mask_base, mask_cursor, mask_words);
    }
    if (!FILL && part) {
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) itotal += __shfl_xor_sync(0xffffffffu, itotal, o);
        if (lane == 0 && itotal) atomicAdd(reinterpret_cast<unsigned long long*>(innz), (unsigned long long)itotal);
    }
}

__global__ void k_check_capacity(const long long* nnz, long long capacity, int32_t* status, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    if (*nnz > capacity) atomicOr(status, SPH_STATUS_LIST_OVERFLOW);
}

// After a gated rebuild that overflowed the list (the fill pass wrote nothing), each row
// is cut to the part that lies inside the list, so that every walk of the rows stays in
// bounds; the overflow bit is already in the status word for the host to read.
__global__ void k_clamp_rows(const long long* __restrict__ nnz, long long capacity, const int32_t* __restrict__ offs,
                             int32_t* __restrict__ cnt, int n, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate) || *nnz <= capacity) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long room = capacity - (long long)offs[i];
    if ((long long)cnt[i] > room) cnt[i] = room > 0 ? (int32_t)room : 0;
}

// After a gated rebuild: the positions and supports the rows were built from, kept for
// the next validity check.
template <int D>
__global__ void k_keep_state(const float* __restrict__ x, const float* __restrict__ H, float* __restrict__ x0,
                             float* __restrict__ H0, int n, const unsigned int* __restrict__ gate,
                             unsigned long long* __restrict__ rebuilds) {
    if (gate_closed(gate)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && rebuilds) *rebuilds += 1ull;
    if (i >= n) return;
    #pragma unroll
    for (int a = 0; a < D; ++a) x0[(int64_t)i * D + a] = x[(int64_t)i * D + a];
    H0[i] = H[i];
}

__global__ void k_expand(const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
                         int n, int64_t* __restrict__ iout, int64_t* __restrict__ jout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b = offs[i], c = cnt[i];
    for (int k = 0; k < c; ++k) {
        if (iout) iout[b + k] = i;
        if (jout) jout[b + k] = list[b + k];
    }
}

// workspace carve-up
struct NbWs {
    float* hmax;
    GridDev* grid;
    long long* total;
    uint32_t* keys;
    int32_t* counts;
    int32_t* tmp;
    float4* recs;
    int32_t* tasks;
    int32_t* ntasks;
    char* scan;
    uint32_t* masks;                  // acceptance bits of the count pass, 32 words per candidate chunk
    int32_t* mask_base;               // per work item: first mask word, or -1 (none kept)
    unsigned long long* mask_cursor;
    int64_t mask_words;
    int64_t bytes;
};
// Acceptance-bit budget: 128 words per particle (the 3D walk needs about 116: 27 stencil
// cells of about two 32-candidate chunks per 32 particles, two words per lane and chunk), at
// most 2^28 words (1 GiB).  Work items past the budget test their candidates again in the
// fill pass.
static int64_t mask_budget(int64_t n) {
    int64_t w = n * 128;
    return w < ((int64_t)1 << 28) ? w : ((int64_t)1 << 28);
}
static int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }
static NbWs carve(char* base, int64_t n, int64_t cap) {
    NbWs w;
    int64_t off = 0;
    w.hmax = reinterpret_cast<float*>(base + off); off += 256;
    w.grid = reinterpret_cast<GridDev*>(base + off); off += align256(sizeof(GridDev));
    w.total = reinterpret_cast<long long*>(base + off); off += 256;
    w.keys = reinterpret_cast<uint32_t*>(base + off); off += align256(n * 4);
    w.counts = reinterpret_cast<int32_t*>(base + off); off += align256(cap * 4);
    w.tmp = reinterpret_cast<int32_t*>(base + off); off += align256(n * 4);
    w.recs = reinterpret_cast<float4*>(base + off); off += align256(n * 16);
    w.tasks = reinterpret_cast<int32_t*>(base + off); off += align256(n * 4);
    w.ntasks = reinterpret_cast<int32_t*>(base + off); off += 256;
    w.scan = base + off;
    int64_t sb = scan_ws_bytes(cap > n ? cap : n);
    off += align256(sb);
    w.mask_words = mask_budget(n);
    w.masks = reinterpret_cast<uint32_t*>(base + off); off += align256(w.mask_words * 4);
    w.mask_base = reinterpret_cast<int32_t*>(base + off); off += align256(n * 4);
    w.mask_cursor = reinterpret_cast<unsigned long long*>(base + off); off += 256;
    w.bytes = off;
    return w;
}

static int max_bits_for(int dim, int64_t cap) {
    int lb = 0;
    while (((int64_t)1 << (lb + 1)) <= cap) ++lb;  // floor(log2 cap)
    int mb = lb / dim;
    int lim = dim == 1 ? 30 : (dim == 2 ? 16 : 10);
    return mb > lim ? lim : mb;
}

// ---------------------------------------------------------------- prior-list refresh
// Validity of a Verlet list built at (x0, H0): every pair with |x_i - x_j| < max(H_i, H_j)
// at (x, H) is in the list when, for every particle k,
//     H_k + |x_k - x0_k| + max_l |x_l - x0_l| <= vs H0_k
// (triangle inequality, H_i the larger current support of the pair:
//  r0 <= r + |dx_i| + |dx_j| < H_i + |dx_i| + dmax <= vs H0_i <= vs max(H0_i, H0_j)).
// k_refresh_check reduces max_k |x_k - x0_k|, max_k (H_k - vs H0_k + |x_k - x0_k|) and max_k vs H0_k into
// three ordered-encoded words; k_refilter evaluates the criterion (with a relative
// margin for rounding) and, when it holds, rebuilds the interacting sublist in place of
// a full neighbour search.

template <int D>
__global__ void k_refresh_check(const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ x0,
                                const float* __restrict__ H0, int n, DevParams P, unsigned int* __restrict__ acc3) {
    float dmax = 0.f, amax = -__int_as_float(0x7f800000), hmax = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> d = dist_vec<D>(load_vec<D>(x, i), load_vec<D>(x0, i), P.dom);
        const float disp = sqrtf(dist2_rn<D>(d));
        const float h = H[i], h0 = P.verlet_scale * H0[i];
        // a NaN anywhere makes the displacement bound infinite, which forces a rebuild
        const bool bad = isnan(disp) || isnan(h) || isnan(h0);
        dmax = bad ? __int_as_float(0x7f800000) : fmaxf(dmax, disp);
        amax = fmaxf(amax, h - h0 + disp);
        hmax = fmaxf(hmax, h0);
    }
    unsigned int e0 = ord_enc(dmax), e1 = ord_enc(amax), e2 = ord_enc(hmax);
    e0 = block_reduce(e0, 0u, OpMaxU());
    e1 = block_reduce(e1, 0u, OpMaxU());
    e2 = block_reduce(e2, 0u, OpMaxU());
    if (threadIdx.x == 0) { atomicMax(acc3 + 0, e0); atomicMax(acc3 + 1, e1); atomicMax(acc3 + 2, e2); }
}

// k_refresh_check for a recorded update: the last block to finish (acc[3] counts the blocks)
// turns the verdict into the condition of the rebuild node and zeroes acc[0..3] for the
// next replay, so the update needs neither a memset nor a separate condition kernel.
// acc holds zeros before the first launch.
template <int D>
__global__ void k_refresh_check_cond(const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ x0,
                                     const float* __restrict__ H0, int n, DevParams P, unsigned int* __restrict__ acc,
                                     cudaGraphConditionalHandle h) {
    float dmax = 0.f, amax = -__int_as_float(0x7f800000), hmax = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> d = dist_vec<D>(load_vec<D>(x, i), load_vec<D>(x0, i), P.dom);
        const float disp = sqrtf(dist2_rn<D>(d));
        const float hh = H[i], h0 = P.verlet_scale * H0[i];
        const bool bad = isnan(disp) || isnan(hh) || isnan(h0);
        dmax = bad ? __int_as_float(0x7f800000) : fmaxf(dmax, disp);
        amax = fmaxf(amax, hh - h0 + disp);
        hmax = fmaxf(hmax, h0);
    }
    unsigned int e0 = ord_enc(dmax), e1 = ord_enc(amax), e2 = ord_enc(hmax);
    e0 = block_reduce(e0, 0u, OpMaxU());
    e1 = block_reduce(e1, 0u, OpMaxU());
    e2 = block_reduce(e2, 0u, OpMaxU());
    __shared__ bool last;
    if (threadIdx.x == 0) {
        atomicMax(acc + 0, e0); atomicMax(acc + 1, e1); atomicMax(acc + 2, e2);
        __threadfence();
        last = atomicAdd(acc + 3, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        unsigned int v[3];
        #pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = atomicAdd(acc + q, 0u);     // coherent reads of the merged words
        cudaGraphSetConditional(h, refresh_valid(v) ? 0u : 1u);
        #pragma unroll
        for (int q = 0; q < 4; ++q) atomicExch(acc + q, 0u);
    }
}


// Eight lanes per row, four rows per warp: the kept Verlet row rewritten into list_out
// with the interacting entries (fl(sqrt(r^2)) / max(H_i, H_j) < 1 at the new positions,
// the test the list builder applies) first, in the kept order, and the rest after them
// in reverse kept order (filled from the row's end, so one pass suffices); a ballot
// per 8-entry chunk compacts both parts.
constexpr int RF_G = 8;

// One lane's entries of a row in the rewrite (q = b + sub, b + sub + RF_G, ... < b + c):
// the neighbour index is loaded two entries ahead and its position and support one entry
// ahead, so the gathers of an entry are in flight while the previous one is tested.  Past
// the row's end the prefetches read particle 0.
template <int D> struct RewritePipe {
    const int32_t* __restrict__ list;
    const float* __restrict__ x;
    const float* __restrict__ H;
    int q2, e, j1, j2;
    Vec<D> x1;
    float H1;
    __device__ __forceinline__ RewritePipe(const int32_t* __restrict__ l, const float* __restrict__ x_, const float* __restrict__ H_,
                                           int q0, int e_)
        : list(l), x(x_), H(H_), q2(q0 + 2 * RF_G), e(e_) {
        j1 = q0 < e_ ? l[q0] : 0;
        j2 = q0 + RF_G < e_ ? l[q0 + RF_G] : 0;
        x1 = load_vec<D>(x_, j1);
        H1 = __ldg(H_ + j1);
    }
    __device__ __forceinline__ void take(int& j, Vec<D>& xj, float& Hj) {
        j = j1; xj = x1; Hj = H1;
        j1 = j2;
        x1 = load_vec<D>(x, j1);
        H1 = __ldg(H + j1);
        j2 = q2 < e ? list[q2] : 0;
        q2 += RF_G;
    }
};
template <int D>
__global__ void k_refilter(const float* __restrict__ x, const float* __restrict__ H, int n, DevParams P,
                           const unsigned int* __restrict__ acc3, const int32_t* __restrict__ offs,
                           const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
                           int32_t* __restrict__ list_out, int32_t* __restrict__ icnt,
                           unsigned long long* __restrict__ innz, int32_t* __restrict__ status,
                           int32_t* __restrict__ offs_out, int32_t* __restrict__ cnt_out) {
    if (acc3 != nullptr && !refresh_valid(acc3)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, SPH_STATUS_LIST_STALE);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int sub = lane & (RF_G - 1);
    const int gshift = lane & ~(RF_G - 1);                 // first lane of this row's group
    const unsigned int below = (1u << sub) - 1u;
    const int64_t ii = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / RF_G;
    const bool valid = ii < n;
    const int i = valid ? (int)ii : 0;
    Vec<D> xi;
    float Hi = 1.f;
    int b = 0, c = 0;
    if (valid) { xi = load_vec<D>(x, i); Hi = H[i]; b = offs[i]; c = cnt[i]; }
    int w = 0, rw = 0;
    RewritePipe<D> pipe(list, x, H, b + sub, b + c);
    for (int base = 0; __any_sync(0xffffffffu, base < c); base += RF_G) {
        const bool in_row = base + sub < c;
        bool keep = false;
        int j;
        Vec<D> xj;
        float Hj;
        pipe.take(j, xj, Hj);
        if (in_row) {
            const Vec<D> d = dist_vec<D>(xi, xj, P.dom);
            const float Hm = fmaxf(Hi, Hj);
            keep = interacting_pair(dist2_rn<D>(d), Hm);
        }
        const unsigned int kb = (__ballot_sync(0xffffffffu, keep) >> gshift) & ((1u << RF_G) - 1u);
        const unsigned int rb = (__ballot_sync(0xffffffffu, in_row && !keep) >> gshift) & ((1u << RF_G) - 1u);
        if (keep) list_out[b + w + __popc(kb & below)] = j;
        else if (in_row) list_out[b + c - 1 - (rw + __popc(rb & below))] = j;
        w += __popc(kb);
        rw += __popc(rb);
    }
    unsigned long long t = (valid && sub == 0) ? (unsigned long long)w : 0ull;
    if (valid && sub == 0) {
        icnt[i] = w;
        if (offs_out) { offs_out[i] = b; cnt_out[i] = c; }
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0 && t) atomicAdd(innz, t);
}

// k_refilter fused with the CRK volume of the rewritten rows (modules/crk, computeCRKFactors:
// V_i = 1 / sum_j W(r_ij, H_j), the scatter support): the rewrite already gathers every
// Verlet neighbour's position and support, and W(r_ij, H_j) is zero past the interacting
// prefix (r >= max(H_i, H_j) >= H_j), so the whole row can be summed.  The sum runs in
// the row's original order, 8 lanes per row.
template <int KF, int D>
__global__ void k_refilter_volume(const float* __restrict__ x, const float* __restrict__ H, int n, DevParams P,
                                  const unsigned int* __restrict__ acc3, const int32_t* __restrict__ offs,
                                  const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
                                  int32_t* __restrict__ list_out, int32_t* __restrict__ icnt,
                                  unsigned long long* __restrict__ innz, int32_t* __restrict__ status, float* __restrict__ V,
                                  int32_t* __restrict__ offs_out, int32_t* __restrict__ cnt_out) {
    if (acc3 != nullptr && !refresh_valid(acc3)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, SPH_STATUS_LIST_STALE);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int sub = lane & (RF_G - 1);
    const int gshift = lane & ~(RF_G - 1);
    const unsigned int below = (1u << sub) - 1u;
    const int64_t ii = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / RF_G;
    const bool valid = ii < n;
    const int i = valid ? (int)ii : 0;
    Vec<D> xi;
    float Hi = 1.f;
    int b = 0, c = 0;
    if (valid) { xi = load_vec<D>(x, i); Hi = H[i]; b = offs[i]; c = cnt[i]; }
    int w = 0, rw = 0;
    float wsum = 0.f;
    RewritePipe<D> pipe(list, x, H, b + sub, b + c);
    for (int base = 0; __any_sync(0xffffffffu, base < c); base += RF_G) {
        const bool in_row = base + sub < c;
        bool keep = false;
        int j;
        Vec<D> xj;
        float Hj;
        pipe.take(j, xj, Hj);
        if (in_row) {
            const Vec<D> d = dist_vec<D>(xi, xj, P.dom);
            const float Hm = fmaxf(Hi, Hj);
            keep = interacting_pair(dist2_rn<D>(d), Hm);
            wsum += kW_inv<KF, D>(safe_sqrt(dot<D>(d, d)), 1.f / Hj);
        }
        const unsigned int kb = (__ballot_sync(0xffffffffu, keep) >> gshift) & ((1u << RF_G) - 1u);
        const unsigned int rb = (__ballot_sync(0xffffffffu, in_row && !keep) >> gshift) & ((1u << RF_G) - 1u);
        if (keep) list_out[b + w + __popc(kb & below)] = j;
        else if (in_row) list_out[b + c - 1 - (rw + __popc(rb & below))] = j;
        w += __popc(kb);
        rw += __popc(rb);
    }
    #pragma unroll
    for (int o = 1; o < RF_G; o <<= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    unsigned long long t = (valid && sub == 0) ? (unsigned long long)w : 0ull;
    if (valid && sub == 0) {
        icnt[i] = w;
        V[i] = 1.f / wsum;
        if (offs_out) { offs_out[i] = b; cnt_out[i] = c; }
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0 && t) atomicAdd(innz, t);
}

// Word fill and copy for the gated build (a memset or a copy cannot be skipped by the GPU).
__global__ void k_fill_gated(uint32_t* __restrict__ p, int64_t count, uint32_t v, const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_copy_gated(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, int64_t count,
                             const unsigned int* __restrict__ gate) {
    if (gate_closed(gate)) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) dst[i] = src[i];
}
static int word_blocks(int64_t words) {
    int64_t b = (words + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

// The list build (grid, counting sort, count pass, scan, fill pass) on the stream.  With a
// gate every launch (the clears and copies included) returns at once when the gate's verdict
// says the kept rows are still valid.
static void build_rows(const DevParams& P, int64_t n, const float* x, const float* H, const NbWs& w, int64_t cell_capacity,
                       int32_t* sort_index, uint32_t* sorted_keys, int32_t* cell_begin, int32_t* cell_end, int32_t* grid_out,
                       int32_t* neighbor_offsets, int32_t* num_neighbors, int32_t* neighbor_list, int64_t list_capacity,
                       int64_t* nnz_out, int32_t* inter_counts, int64_t* inter_nnz_out, int32_t* status,
                       const unsigned int* gate, cudaStream_t s) {
    const bool part = inter_counts != nullptr;
    int mb = max_bits_for(P.dim, cell_capacity);
    int64_t ncells = (int64_t)1 << (mb * P.dim);
    long long* innz = part ? reinterpret_cast<long long*>(inter_nnz_out) : nullptr;
    auto clear = [&](void* ptr, int64_t bytes) {          // bytes: a multiple of 4
        if (gate) {
            wsph::count_launch();
            k_fill_gated<<<word_blocks(bytes / 4), 256, 0, s>>>(reinterpret_cast<uint32_t*>(ptr), bytes / 4, 0u, gate);
        } else {
            cudaMemsetAsync(ptr, 0, bytes, s);
        }
    };

    clear(w.hmax, sizeof(float));
    int rblocks = (int)((n + 1023) / 1024);
    if (rblocks > 148 * 4) rblocks = 148 * 4;
    wsph::count_launch(); k_hmax<<<rblocks, 256, 0, s>>>(H, n, w.hmax, status, gate);
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, k_grid<D><<<1, 1, 0, s>>>(w.hmax, P, mb, w.grid, grid_out, gate));
    clear(w.counts, ncells * sizeof(int32_t));
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, k_keys<D><<<grid_for(n, 256), 256, 0, s>>>(x, (int)n, w.grid, P.dom, w.keys, w.counts, gate));
    exclusive_scan_i32(w.counts, cell_begin, ncells, w.scan, w.total, s, gate);
    if (gate) {
        wsph::count_launch();
        k_copy_gated<<<word_blocks(ncells), 256, 0, s>>>(reinterpret_cast<uint32_t*>(cell_end), reinterpret_cast<const uint32_t*>(cell_begin),
                                                          ncells, gate);
    } else {
        cudaMemcpyAsync(cell_end, cell_begin, ncells * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    }
    wsph::count_launch(); k_scatter<<<grid_for(n, 256), 256, 0, s>>>(w.keys, (int)n, cell_end, w.tmp, gate);
    clear(w.ntasks, sizeof(int32_t));
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (k_rank_sort<D><<<grid_for(n, 256), 256, 0, s>>>(w.tmp, w.keys, cell_begin, cell_end, (int)n, x, H,
                                                                                                 sort_index, sorted_keys, w.recs, w.tasks, w.ntasks,
                                                                                                 gate)));
    int vblocks = grid_for(n, VW_BLOCK);          // >= one warp per 32 particles; warps stride over the work items
    if (vblocks > 148 * 32) vblocks = 148 * 32;
    if (part) clear(inter_nnz_out, sizeof(int64_t));
    clear(w.mask_cursor, sizeof(unsigned long long));
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (k_verlet<D, false><<<vblocks, VW_BLOCK, 0, s>>>(w.recs, sorted_keys, w.tasks, w.ntasks, w.grid, P, sort_index,
                                                                                 cell_begin, cell_end, num_neighbors, inter_counts, nullptr,
                                                                                 nullptr, innz, nullptr, 0, w.masks, w.mask_base,
                                                                                 w.mask_cursor, (long long)w.mask_words, gate)));
    exclusive_scan_i32(num_neighbors, neighbor_offsets, n, w.scan, reinterpret_cast<long long*>(nnz_out), s, gate);
    wsph::count_launch(); k_check_capacity<<<1, 1, 0, s>>>(reinterpret_cast<long long*>(nnz_out), list_capacity, status, gate);
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (k_verlet<D, true><<<vblocks, VW_BLOCK, 0, s>>>(w.recs, sorted_keys, w.tasks, w.ntasks, w.grid, P, sort_index,
                                                                                cell_begin, cell_end, nullptr, inter_counts, neighbor_offsets,
                                                                                neighbor_list, nullptr, reinterpret_cast<long long*>(nnz_out),
                                                                                list_capacity, w.masks, w.mask_base, w.mask_cursor,
                                                                                (long long)w.mask_words, gate)));
}

// ---------------------------------------------------------------- rebuild as a graph conditional
// While a stream is being captured into a CUDA graph, the rebuild of sph_neighbors_update
// goes into the body of an IF conditional node: the validity check's last block turns the
// verdict into the node's condition, and a replay whose rows are kept skips the whole body instead of
// launching ~20 kernels that return at once.  The body is captured on a private stream per
// device, created by the first call made outside a capture (a call during a capture with no
// such stream yet falls back to the gated launches).

constexpr int MAX_DEVICES = 64;
static cudaStream_t g_body_stream[MAX_DEVICES] = {};
static std::atomic<int> g_body_lock{0};

static cudaStream_t body_stream(bool create) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return nullptr;
    if (g_body_stream[dev] || !create) return g_body_stream[dev];
    int expected = 0;
    while (!g_body_lock.compare_exchange_weak(expected, 1)) expected = 0;
    if (!g_body_stream[dev]) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) g_body_stream[dev] = st;
        else cudaGetLastError();
    }
    g_body_lock.store(0);
    return g_body_stream[dev];
}

#define WSPH_CK_GRAPH(call)                                                                                  \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_neighbors_update: %s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// The rebuild (the gated build of build_rows with the clamp and the build-state copy) as an
// IF node on the capturing stream s; bs: the private body stream.
static int rebuild_conditional(const DevParams& P, int64_t n, const float* x, const float* H, float* x0, float* H0, const NbWs& w,
                               int64_t cell_capacity, int32_t* sort_index, uint32_t* sorted_keys, int32_t* cell_begin,
                               int32_t* cell_end, int32_t* grid_out, int32_t* offs, int32_t* cnt, int32_t* list,
                               int64_t list_capacity, int64_t* nnz, unsigned int* verdict, int32_t* status,
                               int64_t* rebuilds, cudaStream_t s, cudaStream_t bs) {
    cudaStreamCaptureStatus st;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    WSPH_CK_GRAPH(cudaStreamGetCaptureInfo(s, &st, nullptr, &graph, &deps, &ndeps));
    cudaGraphConditionalHandle h;
    WSPH_CK_GRAPH(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
    int cblocks = (int)((n + 1023) / 1024);
    if (cblocks > 148 * 4) cblocks = 148 * 4;
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_refresh_check_cond<D><<<cblocks, 256, 0, s>>>(x, H, x0, H0, (int)n, P, verdict, h)));
    WSPH_CK_GRAPH(cudaGetLastError());
    WSPH_CK_GRAPH(cudaStreamGetCaptureInfo(s, &st, nullptr, &graph, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char np_bytes[sizeof(cudaGraphNodeParams)] = {};   // zeroed, as the API wants
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_bytes);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    WSPH_CK_GRAPH(cudaGraphAddNode(&node, graph, deps, ndeps, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    WSPH_CK_GRAPH(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    WSPH_CK_GRAPH(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const long long l0 = g_launches.load();
    // the body runs only on a rebuild: its launches are ungated
    build_rows(P, n, x, H, w, cell_capacity, sort_index, sorted_keys, cell_begin, cell_end, grid_out, offs, cnt, list, list_capacity,
               nnz, nullptr, nullptr, status, nullptr, bs);
    wsph::count_launch();
    k_clamp_rows<<<grid_for(n, 256), 256, 0, bs>>>(reinterpret_cast<const long long*>(nnz), list_capacity, offs, cnt, (int)n, nullptr);
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_keep_state<D><<<grid_for(n, 256), 256, 0, bs>>>(x, H, x0, H0, (int)n, nullptr,
                                                                                reinterpret_cast<unsigned long long*>(rebuilds))));
    g_conditional_launches.fetch_add(g_launches.load() - l0);
    cudaGraph_t captured = nullptr;
    WSPH_CK_GRAPH(cudaStreamEndCapture(bs, &captured));
    return SPH_OK;
}

}  // namespace wsph

using namespace wsph;

extern "C" {

const char* sph_version(void) { return "warpsph_b200 0.1.0 (sm_100a)"; }
const char* sph_last_error_string(void) { return g_err; }
int64_t sph_launch_count(void) { return g_launches.load(); }
int64_t sph_launch_count_conditional(void) { return g_conditional_launches.load(); }

int sph_kernel_constants(int32_t kernel, int32_t dim, double* norm_out, double* scale_out) {
    double c = kernel_norm(kernel, dim), s = kernel_scale(kernel, dim);
    if (c == 0.0 || s == 0.0) return set_error(SPH_ERR_BAD_ARG, "unknown kernel %d / dim %d", kernel, dim);
    if (norm_out) *norm_out = c;
    if (scale_out) *scale_out = s;
    return SPH_OK;
}

int sph_minmax(int64_t n, const float* a, float* out2, void* stream) {
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_minmax: n < 0");
    WSPH_CHECK_PTR(out2);
    if (n > 0) WSPH_CHECK_PTR(a);
    return launch_minmax(n, a, out2, WSPH_STREAM(stream));
}

int sph_neighbors_workspace_size(const SphParams* p, int64_t n, int64_t cell_capacity, int64_t* bytes_out) {
    WSPH_CHECK_PTR(p); WSPH_CHECK_PTR(bytes_out);
    if (n < 0 || cell_capacity < 1) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_workspace_size: bad sizes");
    NbWs w = carve(nullptr, n, cell_capacity);
    *bytes_out = w.bytes;
    return SPH_OK;
}

int sph_neighbors_build(const SphParams* p, int64_t n, const float* x, const float* H,
                        void* workspace, int64_t workspace_bytes, int64_t cell_capacity,
                        int32_t* sort_index, uint32_t* sorted_keys,
                        int32_t* cell_begin, int32_t* cell_end, int32_t* grid_out,
                        int32_t* neighbor_offsets, int32_t* num_neighbors,
                        int32_t* neighbor_list, int64_t list_capacity, int64_t* nnz_out,
                        int32_t* inter_counts, int64_t* inter_nnz_out,
                        int32_t* status, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_build: n out of range");
    if (cell_capacity < 1) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_build: cell_capacity < 1");
    WSPH_CHECK_PTR(nnz_out); WSPH_CHECK_PTR(status); WSPH_CHECK_PTR(grid_out);
    const bool part = inter_counts != nullptr;
    if (part) WSPH_CHECK_PTR(inter_nnz_out);
    cudaStream_t s = WSPH_STREAM(stream);
    if (n == 0) {
        cudaMemsetAsync(nnz_out, 0, sizeof(int64_t), s);
        if (part) cudaMemsetAsync(inter_nnz_out, 0, sizeof(int64_t), s);
        return check_launch("sph_neighbors_build");
    }
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(workspace); WSPH_CHECK_PTR(sort_index);
    WSPH_CHECK_PTR(sorted_keys); WSPH_CHECK_PTR(cell_begin); WSPH_CHECK_PTR(cell_end);
    WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors);
    if (list_capacity > 0) WSPH_CHECK_PTR(neighbor_list);
    if (P.dim == 2 && (reinterpret_cast<uintptr_t>(x) & 7)) return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    NbWs w = carve(reinterpret_cast<char*>(workspace), n, cell_capacity);
    if (workspace_bytes < w.bytes) return set_error(SPH_ERR_WORKSPACE, "neighbour workspace too small: %lld < %lld", (long long)workspace_bytes, (long long)w.bytes);
    build_rows(P, n, x, H, w, cell_capacity, sort_index, sorted_keys, cell_begin, cell_end, grid_out, neighbor_offsets, num_neighbors,
               neighbor_list, list_capacity, nnz_out, inter_counts, inter_nnz_out, status, nullptr, s);
    return check_launch("sph_neighbors_build");
}

int sph_neighbors_refresh(const SphParams* p, int64_t n, const float* x, const float* H, const float* x0, const float* H0,
                          const int32_t* neighbor_offsets, const int32_t* num_neighbors, const int32_t* neighbor_list,
                          int32_t* list_out, int32_t* inter_counts, uint32_t* scratch,
                          int64_t* inter_nnz_out, int32_t* status, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_refresh: n out of range");
    WSPH_CHECK_PTR(scratch); WSPH_CHECK_PTR(status);
    const bool filter = list_out != nullptr;
    cudaStream_t s = WSPH_STREAM(stream);
    if (filter) {
        WSPH_CHECK_PTR(inter_nnz_out);
        cudaMemsetAsync(inter_nnz_out, 0, sizeof(int64_t), s);
    }
    if (n == 0) return check_launch("sph_neighbors_refresh");
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(x0); WSPH_CHECK_PTR(H0);
    if (filter) {
        WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors); WSPH_CHECK_PTR(neighbor_list);
        WSPH_CHECK_PTR(inter_counts);
        if (list_out == neighbor_list) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_refresh: list_out must not alias neighbor_list");
    }
    if (P.dim == 2 && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(x0)) & 7))
        return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    cudaMemsetAsync(scratch, 0, 3 * sizeof(uint32_t), s);
    int cblocks = (int)((n + 1023) / 1024);
    if (cblocks > 148 * 4) cblocks = 148 * 4;
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_refresh_check<D><<<cblocks, 256, 0, s>>>(x, H, x0, H0, (int)n, P, scratch)));
    // without an output list only the verdict is written (no rows are rewritten)
    const int64_t rows = filter ? n : 0;
    const int64_t rblocks = filter ? (n * RF_G + 255) / 256 : 1;   // RF_G lanes per row, 256 threads per block
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_refilter<D><<<(int)rblocks, 256, 0, s>>>(x, H, (int)rows, P, scratch, neighbor_offsets, num_neighbors,
                                                                        neighbor_list, list_out, inter_counts,
                                                                        reinterpret_cast<unsigned long long*>(inter_nnz_out), status,
                                                                        nullptr, nullptr)));
    return check_launch("sph_neighbors_refresh");
}

int sph_neighbors_refresh_volume(const SphParams* p, int64_t n, const float* x, const float* H, const float* x0, const float* H0,
                                 const int32_t* neighbor_offsets, const int32_t* num_neighbors, const int32_t* neighbor_list,
                                 int32_t* list_out, int32_t* inter_counts, uint32_t* scratch, int64_t* inter_nnz_out,
                                 int32_t* status, float* V_out, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_refresh_volume: n out of range");
    WSPH_CHECK_PTR(scratch); WSPH_CHECK_PTR(status); WSPH_CHECK_PTR(inter_nnz_out);
    cudaStream_t s = WSPH_STREAM(stream);
    cudaMemsetAsync(inter_nnz_out, 0, sizeof(int64_t), s);
    if (n == 0) return check_launch("sph_neighbors_refresh_volume");
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(x0); WSPH_CHECK_PTR(H0); WSPH_CHECK_PTR(V_out);
    WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors); WSPH_CHECK_PTR(neighbor_list); WSPH_CHECK_PTR(list_out);
    WSPH_CHECK_PTR(inter_counts);
    if (list_out == neighbor_list) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_refresh_volume: list_out must not alias neighbor_list");
    if (P.dim == 2 && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(x0)) & 7))
        return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    cudaMemsetAsync(scratch, 0, 3 * sizeof(uint32_t), s);
    int cblocks = (int)((n + 1023) / 1024);
    if (cblocks > 148 * 4) cblocks = 148 * 4;
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_refresh_check<D><<<cblocks, 256, 0, s>>>(x, H, x0, H0, (int)n, P, scratch)));
    const int rblocks = (int)((n * RF_G + 255) / 256);
    wsph::count_launch();
    WSPH_DISPATCH_KD(P.kernel, P.dim, (k_refilter_volume<KF, D><<<rblocks, 256, 0, s>>>(x, H, (int)n, P, scratch, neighbor_offsets,
                                                                                       num_neighbors, neighbor_list, list_out,
                                                                                       inter_counts,
                                                                                       reinterpret_cast<unsigned long long*>(inter_nnz_out),
                                                                                       status, V_out, nullptr, nullptr)));
    return check_launch("sph_neighbors_refresh_volume");
}

int sph_neighbors_update(const SphParams* p, int64_t n, const float* x, const float* H, float* x0, float* H0,
                         void* workspace, int64_t workspace_bytes, int64_t cell_capacity,
                         int32_t* sort_index, uint32_t* sorted_keys, int32_t* cell_begin, int32_t* cell_end, int32_t* grid_out,
                         int32_t* neighbor_offsets, int32_t* num_neighbors, int32_t* neighbor_list, int64_t list_capacity,
                         int64_t* nnz, uint32_t* verdict, int32_t* status, int64_t* rebuilds, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_update: n out of range");
    if (cell_capacity < 1) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_update: cell_capacity < 1");
    if (list_capacity < 1) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_update: list_capacity < 1");
    WSPH_CHECK_PTR(nnz); WSPH_CHECK_PTR(verdict); WSPH_CHECK_PTR(status); WSPH_CHECK_PTR(grid_out);
    cudaStream_t s = WSPH_STREAM(stream);
    if (n == 0) {
        cudaMemsetAsync(nnz, 0, sizeof(int64_t), s);
        return check_launch("sph_neighbors_update");
    }
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(x0); WSPH_CHECK_PTR(H0); WSPH_CHECK_PTR(workspace);
    WSPH_CHECK_PTR(sort_index); WSPH_CHECK_PTR(sorted_keys); WSPH_CHECK_PTR(cell_begin); WSPH_CHECK_PTR(cell_end);
    WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors); WSPH_CHECK_PTR(neighbor_list);
    if (P.dim == 2 && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(x0)) & 7))
        return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    NbWs w = carve(reinterpret_cast<char*>(workspace), n, cell_capacity);
    if (workspace_bytes < w.bytes) return set_error(SPH_ERR_WORKSPACE, "neighbour workspace too small: %lld < %lld", (long long)workspace_bytes, (long long)w.bytes);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return check_launch("sph_neighbors_update");
    cudaStream_t bs = body_stream(cs == cudaStreamCaptureStatusNone);
    if (cs == cudaStreamCaptureStatusActive && bs != nullptr && bs != s) {
        rc = rebuild_conditional(P, n, x, H, x0, H0, w, cell_capacity, sort_index, sorted_keys, cell_begin, cell_end, grid_out,
                                 neighbor_offsets, num_neighbors, neighbor_list, list_capacity, nnz, verdict, status, rebuilds, s, bs);
        if (rc) return rc;
        return check_launch("sph_neighbors_update");
    }
    cudaMemsetAsync(verdict, 0, 3 * sizeof(uint32_t), s);
    int cblocks = (int)((n + 1023) / 1024);
    if (cblocks > 148 * 4) cblocks = 148 * 4;
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_refresh_check<D><<<cblocks, 256, 0, s>>>(x, H, x0, H0, (int)n, P, verdict)));
    build_rows(P, n, x, H, w, cell_capacity, sort_index, sorted_keys, cell_begin, cell_end, grid_out, neighbor_offsets, num_neighbors,
               neighbor_list, list_capacity, nnz, nullptr, nullptr, status, verdict, s);
    wsph::count_launch();
    k_clamp_rows<<<grid_for(n, 256), 256, 0, s>>>(reinterpret_cast<const long long*>(nnz), list_capacity, neighbor_offsets, num_neighbors,
                                                 (int)n, verdict);
    wsph::count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_keep_state<D><<<grid_for(n, 256), 256, 0, s>>>(x, H, x0, H0, (int)n, verdict,
                                                                               reinterpret_cast<unsigned long long*>(rebuilds))));
    return check_launch("sph_neighbors_update");
}

int sph_neighbors_rewrite(const SphParams* p, int64_t n, const float* x, const float* H,
                          const int32_t* neighbor_offsets, const int32_t* num_neighbors, const int32_t* neighbor_list,
                          int32_t* list_out, int32_t* offsets_out, int32_t* counts_out, int32_t* inter_counts,
                          int64_t* inter_nnz_out, float* V_out, int32_t* status, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n < 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_rewrite: n out of range");
    WSPH_CHECK_PTR(inter_nnz_out); WSPH_CHECK_PTR(status);
    cudaStream_t s = WSPH_STREAM(stream);
    cudaMemsetAsync(inter_nnz_out, 0, sizeof(int64_t), s);
    if (n == 0) return check_launch("sph_neighbors_rewrite");
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors);
    WSPH_CHECK_PTR(neighbor_list); WSPH_CHECK_PTR(list_out); WSPH_CHECK_PTR(offsets_out); WSPH_CHECK_PTR(counts_out);
    WSPH_CHECK_PTR(inter_counts);
    if (list_out == neighbor_list) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_rewrite: list_out must not alias neighbor_list");
    if (P.dim == 2 && (reinterpret_cast<uintptr_t>(x) & 7)) return set_error(SPH_ERR_BAD_ARG, "positions must be 8-byte aligned in 2D");
    const int rblocks = (int)((n * RF_G + 255) / 256);
    wsph::count_launch();
    if (V_out) {
        WSPH_DISPATCH_KD(P.kernel, P.dim, (k_refilter_volume<KF, D><<<rblocks, 256, 0, s>>>(x, H, (int)n, P, nullptr, neighbor_offsets,
                                                                                           num_neighbors, neighbor_list, list_out,
                                                                                           inter_counts,
                                                                                           reinterpret_cast<unsigned long long*>(inter_nnz_out),
                                                                                           status, V_out, offsets_out, counts_out)));
    } else {
        WSPH_DISPATCH_DIM(P.dim, (k_refilter<D><<<rblocks, 256, 0, s>>>(x, H, (int)n, P, nullptr, neighbor_offsets, num_neighbors,
                                                                         neighbor_list, list_out, inter_counts,
                                                                         reinterpret_cast<unsigned long long*>(inter_nnz_out), status,
                                                                         offsets_out, counts_out)));
    }
    return check_launch("sph_neighbors_rewrite");
}

int sph_neighbors_expand(int64_t n, const int32_t* neighbor_offsets, const int32_t* num_neighbors,
                         const int32_t* neighbor_list, int64_t nnz, int64_t* i_out, int64_t* j_out, void* stream) {
    if (n < 0 || nnz < 0) return set_error(SPH_ERR_BAD_ARG, "sph_neighbors_expand: negative size");
    if (n == 0) return SPH_OK;
    WSPH_CHECK_PTR(neighbor_offsets); WSPH_CHECK_PTR(num_neighbors); WSPH_CHECK_PTR(neighbor_list);
    wsph::count_launch(); k_expand<<<grid_for(n, 256), 256, 0, WSPH_STREAM(stream)>>>(neighbor_offsets, num_neighbors, neighbor_list, (int)n, i_out, j_out);
    return check_launch("sph_neighbors_expand");
}

}  // extern "C"
