// Incompressible (DFSPH) pressure solves of the warpSPH hot path.
//
//   sph_dfsph_alpha                modules/incompressible/wp_alpha.py:35-118, :294-313
//   sph_incompressible_divergence  modules/momentum/incompressible.py:9-34
//   sph_pressure_accel_iisph       modules/pressure/iisph.py:7-24
//   sph_pressure_shift_iisph       modules/incompressible/drift.py:38-57
//   sph_dfsph_div_solve            modules/incompressible/divergenceFree.py:23-139
//   sph_dfsph_density_solve        modules/incompressible/incompressible.py:21-143
//
// The reference runs each Jacobi iteration as two Warp launches plus torch
// reductions and reads the residual back to the host every iteration.  Here a
// whole solve is one cooperative persistent kernel: every iteration is
//   phase A  a_i = -sum_j m_j (p_i/rho_i^2 + p_j/rho_j^2) gradW_ij   (pressure gauge
//            of the previous iteration applied on the fly), writes p_i and a_i
//   barrier
//   phase B  s_i = -sum_j V_j (a_j - a_i).gradW_ij, r_i = src_i - dt_f s_i,
//            p_i += omega r_i / diag_i, block partial sums of p and of the error
//            term folded into FP64 accumulators
//   barrier
//   decide   every block reads the same sums, so all take the same branch
// with a final phase A for the returned acceleration.  The grid barrier is a
// counter + generation pair in the caller's workspace; its waits are bounded
// (SPH_STATUS_TIMEOUT after ~2 s) so a failure returns instead of hanging.
//
// Data written in one phase and read by other blocks in the next (p, a) is
// loaded with ld.global.cg (L2), never through the non-coherent L1.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include "sph_pair_common.cuh"
#include "sph_persistent.cuh"

namespace wsph {

constexpr int JAC_BLOCK = 256;
constexpr int JAC_G = 8;
constexpr int JAC_PPB = JAC_BLOCK / JAC_G;   // particles per block and round

struct JacobiCtl {
    BarrierCtl bar;            // grid barrier and SPH_STATUS_* bits
    double sum[3][2];          // [slot][0] = sum p, [slot][1] = sum of the error term
    unsigned int mm[3][2];     // [slot][0] = min p, [slot][1] = max p (ordered encoding)
};

__device__ __forceinline__ unsigned int f2o(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(unsigned int o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

template <int D> __device__ __forceinline__ Vec<D> load_vec_cg(const float* p, int i) {
    Vec<D> r;
    #pragma unroll
    for (int a = 0; a < D; ++a) r.v[a] = __ldcg(p + (size_t)i * D + a);
    return r;
}

// ---------------------------------------------------------------- per-lane partial sums
// Pressure acceleration, modules/pressure/iisph.py:7-24 with the symmetric gradient
// rho_i sum_j m_j (q_i/rho_i^2 + q_j/rho_j^2) gradW(x_ij, H_j).  p_j = praw_j - mu.
template <int KF, int D, int G, bool CG>
__device__ __forceinline__ Vec<D> accel_partial(int i, int lane, const DevParams& P, const float* __restrict__ x,
                                                const float* __restrict__ H, const float* __restrict__ m,
                                                const float* __restrict__ rho, const float* praw, float mu, float qi,
                                                const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                                                const int32_t* __restrict__ list) {
    Vec<D> s = vzero<D>();
    const Vec<D> xi = load_vec<D>(x, i);
    const int b = offs[i], e = b + cnt[i];
    for (int q = b + lane; q < e; q += G) {
        int j, k; entry(list, q, j, k);
        const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
        const float r = safe_sqrt(dot<D>(xij, xij));
        float W; Vec<D> g;
        kernelWG<KF, D>(xij, r, __ldg(H + j), W, g);
        const float rj = __ldg(rho + j);
        const float pj = (CG ? __ldcg(praw + j) : __ldg(praw + j)) - mu;
        const float c = __ldg(m + j) * (qi + pj / (rj * rj));
        #pragma unroll
        for (int a = 0; a < D; ++a) s.v[a] += c * g.v[a];
    }
    return s;
}

// Pressure shift, modules/incompressible/drift.py:38-57: -sum_j V_j (a_j - a_i).gradW(x_ij, H_j).
template <int KF, int D, int G, bool CG>
__device__ __forceinline__ float shift_partial(int i, int lane, const DevParams& P, const float* __restrict__ x,
                                               const float* __restrict__ H, const float* __restrict__ m,
                                               const float* __restrict__ rho, const float* acc, const Vec<D>& ai,
                                               const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                                               const int32_t* __restrict__ list) {
    float s = 0.f;
    const Vec<D> xi = load_vec<D>(x, i);
    const int b = offs[i], e = b + cnt[i];
    for (int q = b + lane; q < e; q += G) {
        int j, k; entry(list, q, j, k);
        const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
        const float r = safe_sqrt(dot<D>(xij, xij));
        float W; Vec<D> g;
        kernelWG<KF, D>(xij, r, __ldg(H + j), W, g);
        const Vec<D> aj = CG ? load_vec_cg<D>(acc, j) : load_vec<D>(acc, j);
        float t = 0.f;
        #pragma unroll
        for (int a = 0; a < D; ++a) t += (aj.v[a] - ai.v[a]) * g.v[a];
        s += __ldg(m + j) / __ldg(rho + j) * t;
    }
    return s;
}

// ---------------------------------------------------------------- prep: divergence, alpha, source, diagonal
// mode -1: standalone (div_out and/or alpha_out); 0: divergence-free solve; 1: density solve.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_dfsph_prep(int n, DevParams P, int mode, float rho0, const float* __restrict__ x, const float* __restrict__ H,
             const float* __restrict__ m, const float* __restrict__ rho, const float* __restrict__ v,
             const float* __restrict__ dvdt, const float* __restrict__ dtp, const int32_t* __restrict__ offs,
             const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float* __restrict__ div_out,
             float* __restrict__ alpha_out, const float* __restrict__ p_init, int init_mode, float* __restrict__ src,
             float* __restrict__ diag, float* __restrict__ p0) {
    Grp<G> g(n);
    const bool want_div = div_out || src, want_alpha = alpha_out || diag;
    const float dt = dtp ? *dtp : 0.f;
    float sdiv = 0.f, sB = 0.f;
    Vec<D> sA = vzero<D>();
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i];
        Vec<D> vi = load_vec<D>(v, i);
        if (dvdt) {
            const Vec<D> ai = load_vec<D>(dvdt, i);
            #pragma unroll
            for (int a = 0; a < D; ++a) vi.v[a] = __fadd_rn(vi.v[a], __fmul_rn(dt, ai.v[a]));
        }
        const int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            const float Hj = __ldg(H + j), mj = __ldg(m + j);
            const float Vj = mj / __ldg(rho + j);
            float W;
            Vec<D> gS, gG;
            kernelWG<KF, D>(xij, r, Hj, W, gS);
            if (Hj == Hi) gG = gS; else kernelWG<KF, D>(xij, r, Hi, W, gG);
            if (want_div) {
                Vec<D> vj = load_vec<D>(v, j);
                if (dvdt) {
                    const Vec<D> aj = load_vec<D>(dvdt, j);
                    #pragma unroll
                    for (int a = 0; a < D; ++a) vj.v[a] = __fadd_rn(vj.v[a], __fmul_rn(dt, aj.v[a]));
                }
                float t = 0.f;
                #pragma unroll
                for (int a = 0; a < D; ++a) t += (vj.v[a] - vi.v[a]) * gS.v[a];
                sdiv += Vj * t;
            }
            if (want_alpha) {
                #pragma unroll
                for (int a = 0; a < D; ++a) sA.v[a] += Vj * gG.v[a];
                sB += Vj * Vj / mj * dot<D>(gG, gG);
            }
        }
    }
    sdiv = gsum<G>(sdiv);
    sB = gsum<G>(sB);
    #pragma unroll
    for (int a = 0; a < D; ++a) sA.v[a] = gsum<G>(sA.v[a]);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float div = -rho0 * sdiv;                       // momentum/incompressible.py:22
    const float Ai = m[i] / rho[i];
    const float alpha = -(Ai / m[i] * dot<D>(sA, sA) + Ai * sB);   // wp_alpha.py:115, :313
    if (div_out) div_out[i] = div;
    if (alpha_out) alpha_out[i] = alpha;
    if (mode == 0) {                                      // divergenceFree.py:54, :62, :72
        src[i] = -div;
        diag[i] = dt * alpha;
        p0[i] = init_mode ? p_init[i] : p_init[i] * 0.75f;
    } else if (mode == 1) {                               // incompressible.py:54-79
        float rs = __fadd_rn(rho[i], __fmul_rn(dt, div));
        rs = rs < 0.9f ? 0.9f : rs;
        src[i] = rho0 - rs;
        const float a = (dt * dt) * alpha;
        diag[i] = a > -1e-6f ? -1e-6f : a;
        p0[i] = init_mode ? p_init[i] : 0.f;
    }
}

// ---------------------------------------------------------------- standalone accel / shift passes
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_iisph_accel(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
              const float* __restrict__ rho, const float* __restrict__ pr, const int32_t* __restrict__ offs,
              const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float* __restrict__ acc) {
    Grp<G> g(n);
    Vec<D> s = vzero<D>();
    float rhoi = 1.f;
    if (g.valid) {
        rhoi = rho[g.i];
        s = accel_partial<KF, D, G, false>(g.i, g.lane, P, x, H, m, rho, pr, 0.f, pr[g.i] / (rhoi * rhoi), offs, cnt, list);
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) s.v[a] = gsum<G>(s.v[a]);
    if (!g.valid || g.lane != 0) return;
    #pragma unroll
    for (int a = 0; a < D; ++a) s.v[a] = -(rhoi * s.v[a]) / rhoi;
    store_vec<D>(acc, g.i, s);
}

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_iisph_shift(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
              const float* __restrict__ rho, const float* __restrict__ acc, const int32_t* __restrict__ offs,
              const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float* __restrict__ shift) {
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) s = shift_partial<KF, D, G, false>(g.i, g.lane, P, x, H, m, rho, acc, load_vec<D>(acc, g.i), offs, cnt, list);
    s = gsum<G>(s);
    if (g.valid && g.lane == 0) shift[g.i] = -s;
}

// ---------------------------------------------------------------- persistent Jacobi solve
struct JacobiArgs {
    int n, mode, min_it, max_it;
    float omega, tol;
    DevParams P;
    const float *x, *H, *m, *rho, *src, *diag, *dtp;
    const int32_t *offs, *cnt, *list;
    float* praw;       // un-gauged pressure of the last update (p0 before the first)
    float* p_out;      // gauged pressure (the iteration's pressureA; the result at the end)
    float* acc;        // pressure acceleration [n*D]
    float* hist;       // [max_it*4]
    int32_t* iters_out;
    int32_t* status_out;
    JacobiCtl* ctl;
    unsigned long long barrier_ns;   // grid-barrier wait limit
};

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned int warp_min_u(unsigned int v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned int warp_max_u(unsigned int v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// A grid barrier ran out: the block records the timeout (block 0 also the iteration it
// had reached) and returns.  p_out and acc hold the last completed phase A.
__device__ __forceinline__ void jacobi_gave_up(const JacobiArgs& a, int it) {
    if (threadIdx.x == 0) {
        atomicOr(a.status_out, SPH_STATUS_TIMEOUT);
        if (blockIdx.x == 0) *a.iters_out = it;
    }
}

template <int KF, int D>
__global__ void __launch_bounds__(JAC_BLOCK)
k_jacobi(JacobiArgs a) {
    constexpr int G = JAC_G;
    __shared__ double sh_sum[JAC_BLOCK / 32][2];
    __shared__ unsigned int sh_mm[JAC_BLOCK / 32][2];
    const int lane = threadIdx.x & (G - 1);
    const int warp = threadIdx.x >> 5;
    const int n = a.n;
    const int rounds = (n + (int)gridDim.x * JAC_PPB - 1) / ((int)gridDim.x * JAC_PPB);
    const float dt = *a.dtp;
    const float dtf = a.mode == 0 ? dt : dt * dt;
    JacobiCtl* c = a.ctl;
    float mu = 0.f;
    int it = 0;
    bool converged = false;

    for (;;) {
        // ------------------------------------------------ phase A: pressure acceleration
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const int s1 = (it + 1) % 3;
            c->sum[s1][0] = 0.0; c->sum[s1][1] = 0.0;
            c->mm[s1][0] = 0xffffffffu; c->mm[s1][1] = 0u;
            if (it == 0) { c->sum[0][0] = 0.0; c->sum[0][1] = 0.0; c->mm[0][0] = 0xffffffffu; c->mm[0][1] = 0u; }
        }
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = (rd * (int)gridDim.x + (int)blockIdx.x) * JAC_PPB + (int)threadIdx.x / G;
            const bool valid = i < n;
            Vec<D> s = vzero<D>();
            float pi = 0.f, rhoi = 1.f;
            if (valid) {
                pi = __ldcg(a.praw + i) - mu;
                rhoi = __ldg(a.rho + i);
                s = accel_partial<KF, D, G, true>(i, lane, a.P, a.x, a.H, a.m, a.rho, a.praw, mu, pi / (rhoi * rhoi),
                                                      a.offs, a.cnt, a.list);
            }
            #pragma unroll
            for (int d = 0; d < D; ++d) s.v[d] = gsum<G>(s.v[d]);
            if (valid && lane == 0) {
                #pragma unroll
                for (int d = 0; d < D; ++d) s.v[d] = -(rhoi * s.v[d]) / rhoi;
                store_vec<D>(a.acc, i, s);
                a.p_out[i] = pi;
            }
        }
        if (converged || it >= a.max_it) break;
        if (!grid_barrier(&c->bar, a.barrier_ns)) { jacobi_gave_up(a, it); return; }

        // ------------------------------------------------ phase B: shift, residual, update
        double psum = 0.0, esum = 0.0;
        unsigned int pmin = 0xffffffffu, pmax = 0u;
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = (rd * (int)gridDim.x + (int)blockIdx.x) * JAC_PPB + (int)threadIdx.x / G;
            const bool valid = i < n;
            float s = 0.f;
            if (valid) s = shift_partial<KF, D, G, true>(i, lane, a.P, a.x, a.H, a.m, a.rho, a.acc, load_vec_cg<D>(a.acc, i),
                                                             a.offs, a.cnt, a.list);
            s = gsum<G>(s);
            if (valid && lane == 0) {
                const float r = a.src[i] - dtf * (-s);
                float pb = __ldcg(a.p_out + i) + a.omega * r / a.diag[i];
                float e;
                if (a.mode == 1) {
                    pb = pb < 0.f ? 0.f : pb;                       // incompressible.py:108
                    e = -r < -a.tol ? -a.tol : -r;                  // :111
                } else {
                    e = fabsf(r);                                   // divergenceFree.py:112
                }
                a.praw[i] = pb;
                psum += (double)pb;
                esum += (double)e;
                const unsigned int o = f2o(pb);
                pmin = min(pmin, o);
                pmax = max(pmax, o);
            }
        }
        psum = warp_sum(psum); esum = warp_sum(esum);
        pmin = warp_min_u(pmin); pmax = warp_max_u(pmax);
        if ((threadIdx.x & 31) == 0) { sh_sum[warp][0] = psum; sh_sum[warp][1] = esum; sh_mm[warp][0] = pmin; sh_mm[warp][1] = pmax; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double ps = 0.0, es = 0.0;
            unsigned int lo = 0xffffffffu, hi = 0u;
            for (int w = 0; w < JAC_BLOCK / 32; ++w) { ps += sh_sum[w][0]; es += sh_sum[w][1]; lo = min(lo, sh_mm[w][0]); hi = max(hi, sh_mm[w][1]); }
            const int sl = it % 3;
            atomicAdd(&c->sum[sl][0], ps);
            atomicAdd(&c->sum[sl][1], es);
            atomicMin(&c->mm[sl][0], lo);
            atomicMax(&c->mm[sl][1], hi);
        }
        if (!grid_barrier(&c->bar, a.barrier_ns)) { jacobi_gave_up(a, it); return; }

        // ------------------------------------------------ decide (identical in every block)
        const int sl = it % 3;
        const double ps = *(volatile double*)&c->sum[sl][0];
        const double es = *(volatile double*)&c->sum[sl][1];
        const float lo = o2f(*(volatile unsigned int*)&c->mm[sl][0]);
        const float hi = o2f(*(volatile unsigned int*)&c->mm[sl][1]);
        const double mean = ps / (double)n;
        const double err = es / (double)n;
        mu = a.mode == 0 ? (float)mean : 0.f;                       // divergenceFree.py:104
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.hist[it * 4 + 0] = (float)err;
            a.hist[it * 4 + 1] = lo - mu;
            a.hist[it * 4 + 2] = hi - mu;
            a.hist[it * 4 + 3] = (float)(mean - (double)mu);
        }
        const bool finite = isfinite(err);
        if (!finite) { if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(&c->bar.status, SPH_STATUS_NONFINITE); }
        converged = (it >= a.min_it && err < (double)a.tol) || !finite;
        ++it;
    }
    if (threadIdx.x == 0) {
        int st = *(volatile int*)&c->bar.status;
        if (blockIdx.x == 0) {
            if (!converged && a.max_it > 0) st |= SPH_STATUS_NOT_CONVERGED;
            *a.iters_out = it;
        }
        if (st) atomicOr(a.status_out, st);
    }
}

// ---------------------------------------------------------------- host side
constexpr size_t kCtlBytes = 256;
static_assert(sizeof(JacobiCtl) <= kCtlBytes, "control block");

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static int64_t dfsph_ws_bytes(int64_t n) { return (int64_t)(kCtlBytes + 3 * align256((size_t)n * sizeof(float))); }

template <int KF, int D>
static int launch_jacobi(JacobiArgs& a, cudaStream_t s) {
    static std::mutex mu;
    static int cached_dev = -1, blocks_per_sm = 0, num_sms = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "jacobi: cudaGetDevice: %s", cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_dev != dev) {
            int coop = 0;
            e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
            if (e != cudaSuccess || !coop) return set_error(SPH_ERR_UNSUPPORTED, "jacobi: device %d has no cooperative launch", dev);
            e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "jacobi: SM count: %s", cudaGetErrorString(e));
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_jacobi<KF, D>, JAC_BLOCK, 0);
            if (e != cudaSuccess || blocks_per_sm < 1) return set_error(SPH_ERR_CUDA, "jacobi: occupancy query failed");
            cached_dev = dev;
        }
    }
    const int64_t need = (a.n + JAC_PPB - 1) / JAC_PPB;
    const int grid = (int)std::min<int64_t>(need, (int64_t)blocks_per_sm * num_sms);
    void* args[] = {&a};
    count_launch();
    e = cudaLaunchCooperativeKernel((const void*)k_jacobi<KF, D>, dim3(grid), dim3(JAC_BLOCK), args, 0, s);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "jacobi: cooperative launch: %s", cudaGetErrorString(e));
    return SPH_OK;
}

static int dfsph_solve(int mode, const SphParams* p, const SphJacobiConfig* cfg, int64_t n, const float* x, const float* H,
                       const float* m, const float* rho, const float* v, const float* dvdt, const float* p_init,
                       const float* dt, const int32_t* offs, const int32_t* cnt, const int32_t* list, void* ws,
                       int64_t ws_bytes, float* p_out, float* accel_out, float* history, int32_t* iterations, int32_t* status,
                       void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(cfg); WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v);
    WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(ws); WSPH_CHECK_PTR(p_out); WSPH_CHECK_PTR(accel_out); WSPH_CHECK_PTR(history);
    WSPH_CHECK_PTR(iterations); WSPH_CHECK_PTR(status); CHECK_CSR();
    if (cfg->init_mode != 0 && cfg->init_mode != 1) return set_error(SPH_ERR_BAD_ARG, "jacobi: init_mode must be 0 or 1");
    if ((mode == 0 || cfg->init_mode == 1) && !p_init) return set_error(SPH_ERR_BAD_ARG, "jacobi: p_init is required");
    if (cfg->max_iterations < 0 || cfg->min_iterations < 0 || cfg->max_iterations > (1 << 20))
        return set_error(SPH_ERR_BAD_ARG, "jacobi: iteration counts out of range");
    if (!(cfg->relaxation == cfg->relaxation) || !(cfg->tolerance == cfg->tolerance))
        return set_error(SPH_ERR_BAD_ARG, "jacobi: NaN relaxation or tolerance");
    if (cfg->barrier_timeout_us < 0) return set_error(SPH_ERR_BAD_ARG, "jacobi: barrier_timeout_us must be >= 0");
    if (ws_bytes < dfsph_ws_bytes(n)) return set_error(SPH_ERR_WORKSPACE, "jacobi: workspace %lld < %lld bytes", (long long)ws_bytes,
                                                       (long long)dfsph_ws_bytes(n));
    if (reinterpret_cast<uintptr_t>(ws) & 255) return set_error(SPH_ERR_BAD_ARG, "jacobi: workspace must be 256-byte aligned");
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt, "dvdt")) ||
        (rc = check_align_vec(P, accel_out, "accel_out")))
        return rc;
    char* w = static_cast<char*>(ws);
    JacobiCtl* ctl = reinterpret_cast<JacobiCtl*>(w);
    const size_t nb = align256((size_t)n * sizeof(float));
    float* praw = reinterpret_cast<float*>(w + kCtlBytes);
    float* src = reinterpret_cast<float*>(w + kCtlBytes + nb);
    float* diag = reinterpret_cast<float*>(w + kCtlBytes + 2 * nb);
    cudaError_t e = cudaMemsetAsync(ctl, 0, kCtlBytes, s);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "jacobi: memset: %s", cudaGetErrorString(e));
    const float rho0 = (float)cfg->rest_density;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_dfsph_prep<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, mode, rho0, x, H, m, rho, v, dvdt, dt, offs, cnt, list, nullptr, nullptr, p_init, cfg->init_mode, src, diag, praw)));
    if ((rc = check_launch("jacobi prep"))) return rc;
    JacobiArgs a;
    a.n = (int)n; a.mode = mode; a.min_it = cfg->min_iterations; a.max_it = cfg->max_iterations;
    a.omega = (float)cfg->relaxation; a.tol = (float)cfg->tolerance; a.P = P;
    a.x = x; a.H = H; a.m = m; a.rho = rho; a.src = src; a.diag = diag; a.dtp = dt;
    a.offs = offs; a.cnt = cnt; a.list = list;
    a.praw = praw; a.p_out = p_out; a.acc = accel_out; a.hist = history;
    a.iters_out = iterations; a.status_out = status; a.ctl = ctl;
    a.barrier_ns = cfg->barrier_timeout_us > 0 ? 1000ull * (unsigned long long)cfg->barrier_timeout_us : kBarrierLimitNs;
    rc = SPH_ERR_UNSUPPORTED;
    WSPH_DISPATCH_KD(P.kernel, P.dim, (rc = launch_jacobi<KF, D>(a, s)));
    return rc;
}

// ---------------------------------------------------------------- learned warm start: input features
// Sums over particles of |src/diag|, the row count and diag (FP64, into the control block).
__global__ void k_feature_sums(int n, const float* __restrict__ src, const float* __restrict__ diag, const int32_t* __restrict__ cnt,
                               double* __restrict__ sums3) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a += fabs((double)src[i] / (double)diag[i]);
        b += (double)cnt[i];
        c += (double)diag[i];
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) { atomicAdd(sums3, a); atomicAdd(sums3 + 1, b); atomicAdd(sums3 + 2, c); }
}

// Eight per-particle features (gather support W(r, H_i), V_j = m_j / rho_j):
//   0  p_jac_i / P           p_jac = src / diag, the diagonal (one-iteration) Jacobi estimate
//   1  sum_j V_j W_ij p_jac_j / P
//   2  p_prev_i / P
//   3  sum_j V_j W_ij p_prev_j / P
//   4  100 (rho_i / rho0 - 1)
//   5  sum_j V_j W_ij - 1    (Shepard deficit: free surface)
//   6  cnt_i / mean(cnt) - 1
//   7  diag_i / mean(diag) - 1
// with P = mean_i |p_jac_i| (written to scale_out[0]); a network output y maps to p = y P.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_features(int n, DevParams P, float rho0, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
           const float* __restrict__ rho, const float* __restrict__ src, const float* __restrict__ diag,
           const float* __restrict__ p_prev, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
           const int32_t* __restrict__ list, const double* __restrict__ sums3, float* __restrict__ feats,
           float* __restrict__ scale_out) {
    Grp<G> g(n);
    const float Pref = (float)(sums3[0] / (double)n);
    const float inv_P = Pref > 0.f ? 1.f / Pref : 0.f;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i];
        const int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float w = __ldg(m + j) / __ldg(rho + j) * kernelW<KF, D>(safe_sqrt(dot<D>(xij, xij)), Hi);
            s0 += w;
            s1 += w * (__ldg(src + j) / __ldg(diag + j));
            s2 += w * __ldg(p_prev + j);
        }
    }
    s0 = gsum<G>(s0); s1 = gsum<G>(s1); s2 = gsum<G>(s2);
    if (blockIdx.x == 0 && threadIdx.x == 0 && scale_out) scale_out[0] = Pref;
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float mean_cnt = (float)(sums3[1] / (double)n), mean_diag = (float)(sums3[2] / (double)n);
    float f[8];
    f[0] = src[i] / diag[i] * inv_P;
    f[1] = s1 * inv_P;
    f[2] = p_prev[i] * inv_P;
    f[3] = s2 * inv_P;
    f[4] = 100.f * (rho[i] / rho0 - 1.f);
    f[5] = s0 - 1.f;
    f[6] = mean_cnt > 0.f ? (float)cnt[i] / mean_cnt - 1.f : 0.f;
    f[7] = mean_diag != 0.f ? diag[i] / mean_diag - 1.f : 0.f;
    float4* o = reinterpret_cast<float4*>(feats + (size_t)i * 8);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
}

}  // namespace wsph

using namespace wsph;

extern "C" {

int sph_dfsph_alpha(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                    const int32_t* offs, const int32_t* cnt, const int32_t* list, float* alpha_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(alpha_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    // v is only read for the divergence; x stands in as a valid vector array
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_dfsph_prep<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, -1, 0.f, x, H, m, rho, x, nullptr, nullptr, offs, cnt, list, nullptr, alpha_out, nullptr, 0, nullptr, nullptr, nullptr)));
    return check_launch("sph_dfsph_alpha");
}

int sph_incompressible_divergence(const SphParams* p, int64_t n, double rest_density, const float* x, const float* H,
                                  const float* m, const float* rho, const float* v, const float* dvdt, const float* dt,
                                  const int32_t* offs, const int32_t* cnt, const int32_t* list, float* div_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(div_out); CHECK_CSR();
    if (dvdt && !dt) return set_error(SPH_ERR_BAD_ARG, "sph_incompressible_divergence: dvdt given without dt");
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt, "dvdt"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_dfsph_prep<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, -1, (float)rest_density, x, H, m, rho, v, dvdt, dt, offs, cnt, list, div_out, nullptr, nullptr, 0, nullptr, nullptr,
        nullptr)));
    return check_launch("sph_incompressible_divergence");
}

int sph_pressure_accel_iisph(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                             const float* pressure, const int32_t* offs, const int32_t* cnt, const int32_t* list, float* accel_out,
                             void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(pressure); WSPH_CHECK_PTR(accel_out);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, accel_out, "accel_out"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_iisph_accel<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, x, H, m, rho, pressure, offs, cnt, list, accel_out)));
    return check_launch("sph_pressure_accel_iisph");
}

int sph_pressure_shift_iisph(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                             const float* accel, const int32_t* offs, const int32_t* cnt, const int32_t* list, float* shift_out,
                             void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(accel); WSPH_CHECK_PTR(shift_out);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, accel, "accel"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_iisph_shift<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, x, H, m, rho, accel, offs, cnt, list, shift_out)));
    return check_launch("sph_pressure_shift_iisph");
}

int sph_dfsph_features(const SphParams* p, const SphJacobiConfig* cfg, int32_t mode, int64_t n, const float* x, const float* H,
                       const float* m, const float* rho, const float* v, const float* dvdt, const float* p_prev, const float* dt,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list, void* workspace, int64_t workspace_bytes,
                       float* feats_out, float* scale_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(cfg); WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v);
    WSPH_CHECK_PTR(p_prev); WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(workspace); WSPH_CHECK_PTR(feats_out); WSPH_CHECK_PTR(scale_out);
    CHECK_CSR();
    if (mode != 0 && mode != 1) return set_error(SPH_ERR_BAD_ARG, "sph_dfsph_features: mode must be 0 or 1");
    if (workspace_bytes < dfsph_ws_bytes(n)) return set_error(SPH_ERR_WORKSPACE, "sph_dfsph_features: workspace too small");
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return set_error(SPH_ERR_BAD_ARG, "sph_dfsph_features: workspace must be 256-byte aligned");
    if (reinterpret_cast<uintptr_t>(feats_out) & 15) return set_error(SPH_ERR_BAD_ARG, "sph_dfsph_features: feats_out must be 16-byte aligned");
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt, "dvdt"))) return rc;
    char* w = static_cast<char*>(workspace);
    const size_t nb = align256((size_t)n * sizeof(float));
    double* sums3 = reinterpret_cast<double*>(w);
    float* p0 = reinterpret_cast<float*>(w + kCtlBytes);
    float* src = reinterpret_cast<float*>(w + kCtlBytes + nb);
    float* diag = reinterpret_cast<float*>(w + kCtlBytes + 2 * nb);
    cudaError_t e = cudaMemsetAsync(sums3, 0, 3 * sizeof(double), s);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_dfsph_features: memset: %s", cudaGetErrorString(e));
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_dfsph_prep<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, mode, (float)cfg->rest_density, x, H, m, rho, v, dvdt, dt, offs, cnt, list, nullptr, nullptr, p_prev, 1, src, diag, p0)));
    int rb = grid_for(n, 256);
    if (rb > 148 * 4) rb = 148 * 4;
    count_launch();
    k_feature_sums<<<rb, 256, 0, s>>>((int)n, src, diag, cnt, sums3);
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_features<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, (float)cfg->rest_density, x, H, m, rho, src, diag, p_prev, offs, cnt, list, sums3, feats_out, scale_out)));
    return check_launch("sph_dfsph_features");
}

int64_t sph_dfsph_workspace_size(int64_t n, int32_t dim) {
    (void)dim;
    return n < 0 ? -1 : dfsph_ws_bytes(n);
}

int sph_dfsph_div_solve(const SphParams* p, const SphJacobiConfig* cfg, int64_t n, const float* x, const float* H, const float* m,
                        const float* rho, const float* v, const float* dvdt, const float* p_init, const float* dt,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list, void* workspace, int64_t workspace_bytes,
                        float* p_out, float* accel_out, float* history, int32_t* iterations, int32_t* status, void* stream) {
    return dfsph_solve(0, p, cfg, n, x, H, m, rho, v, dvdt, p_init, dt, offs, cnt, list, workspace, workspace_bytes, p_out,
                       accel_out, history, iterations, status, stream);
}

int sph_dfsph_density_solve(const SphParams* p, const SphJacobiConfig* cfg, int64_t n, const float* x, const float* H,
                            const float* m, const float* rho, const float* v, const float* dvdt, const float* p_init,
                            const float* dt, const int32_t* offs, const int32_t* cnt, const int32_t* list, void* workspace,
                            int64_t workspace_bytes, float* p_out, float* accel_out, float* history, int32_t* iterations,
                            int32_t* status, void* stream) {
    return dfsph_solve(1, p, cfg, n, x, H, m, rho, v, dvdt, p_init, dt, offs, cnt, list, workspace, workspace_bytes, p_out,
                       accel_out, history, iterations, status, stream);
}

}  // extern "C"
