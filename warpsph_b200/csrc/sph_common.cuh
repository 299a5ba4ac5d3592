// Shared device code for libwarpsph_b200: parameter block, vector helpers,
// Wendland kernels, periodic minimum-image distance and the CRK-corrected
// kernel gradient.  Everything here is header-only and templated on the
// spatial dimension D (1, 2, 3) and the kernel function KF.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "warpsph_b200.h"

namespace wsph {

// ---------------------------------------------------------------- params
struct DomainF {
    float min[3], max[3], L[3], halfL[3];
    int periodic[3];
};

struct DevParams {
    int dim, kernel;
    DomainF dom;
    float verlet_scale;
    float C_l, C_q, Cu_l, Cu_q, K;
    int viscosity_term, monaghan_switch, correct_xi, scale_beta;
    float eta_crit, eta_fold;
    int enable_crk_limiter, enable_vanleer, force_vl_off, force_vl_on;
    float gamma;
    int energy_scheme, limit_xi, kahan, correct_grad_v;
    float alpha_min, alpha_max, beta_xi;
    float target_neighbors;
    float cfl, min_dt, max_dt, dt_growth;
    float c_s;      // sound speed of the viscosity terms without per-particle sound speeds
    float beta_c, beta_d;
    int conductivity_term;
    float kscale;   // H / h  (kernel scale)
    float kxi;      // the kernel "xi" used by CFL, viscosity and switches
};

// ---------------------------------------------------------------- small vectors
template <int D> struct Vec { float v[D]; };
template <int D> struct Mat { float m[D][D]; };

template <int D> __device__ __forceinline__ Vec<D> vzero() { Vec<D> r; _Pragma("unroll") for (int a = 0; a < D; ++a) r.v[a] = 0.f; return r; }
template <int D> __device__ __forceinline__ Mat<D> mzero() { Mat<D> r; _Pragma("unroll") for (int a = 0; a < D; ++a) _Pragma("unroll") for (int b = 0; b < D; ++b) r.m[a][b] = 0.f; return r; }

template <int D> __device__ __forceinline__ Vec<D> load_vec(const float* __restrict__ p, int i) {
    Vec<D> r;
    if constexpr (D == 2) {
        float2 t = __ldg(reinterpret_cast<const float2*>(p) + i);
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        _Pragma("unroll") for (int a = 0; a < D; ++a) r.v[a] = __ldg(p + (size_t)i * D + a);
    }
    return r;
}
template <int D> __device__ __forceinline__ void store_vec(float* __restrict__ p, size_t i, const Vec<D>& x) {
    if constexpr (D == 2) {
        reinterpret_cast<float2*>(p)[i] = make_float2(x.v[0], x.v[1]);
    } else {
        _Pragma("unroll") for (int a = 0; a < D; ++a) p[i * D + a] = x.v[a];
    }
}
template <int D> __device__ __forceinline__ Mat<D> load_mat(const float* __restrict__ p, int i) {
    Mat<D> r;
    _Pragma("unroll") for (int a = 0; a < D; ++a)
        _Pragma("unroll") for (int b = 0; b < D; ++b) r.m[a][b] = __ldg(p + (size_t)i * D * D + a * D + b);
    return r;
}
template <int D> __device__ __forceinline__ void store_mat(float* __restrict__ p, int i, const Mat<D>& x) {
    _Pragma("unroll") for (int a = 0; a < D; ++a)
        _Pragma("unroll") for (int b = 0; b < D; ++b) p[(size_t)i * D * D + a * D + b] = x.m[a][b];
}
template <int D> __device__ __forceinline__ float dot(const Vec<D>& a, const Vec<D>& b) {
    float s = a.v[0] * b.v[0];
    _Pragma("unroll") for (int k = 1; k < D; ++k) s += a.v[k] * b.v[k];
    return s;
}
// y = M x  (y^a = sum_b M[a][b] x^b)
template <int D> __device__ __forceinline__ Vec<D> matvec(const Mat<D>& M, const Vec<D>& x) {
    Vec<D> r;
    _Pragma("unroll") for (int a = 0; a < D; ++a) {
        float s = M.m[a][0] * x.v[0];
        _Pragma("unroll") for (int b = 1; b < D; ++b) s += M.m[a][b] * x.v[b];
        r.v[a] = s;
    }
    return r;
}

// Warp's builtin min/max: `a < b ? a : b` / `a > b ? a : b` (NaN propagates from b).
__device__ __forceinline__ float wmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float wmax(float a, float b) { return a > b ? a : b; }

// Block-wide reduction (blockDim.x a multiple of 32, at most 1024 threads); the result is
// valid in thread 0.  Every thread of the block must call it (it synchronises).  Used by
// the global reductions so that each block issues one atomic instead of one per warp.
template <typename T, typename Op>
__device__ __forceinline__ T block_reduce(T v, T identity, Op op) {
    __shared__ T part[32];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();                              // earlier readers of part[] are done
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : identity;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}
struct OpMinF { __device__ __forceinline__ float operator()(float a, float b) const { return fminf(a, b); } };
struct OpMaxF { __device__ __forceinline__ float operator()(float a, float b) const { return fmaxf(a, b); } };
struct OpMaxU { __device__ __forceinline__ unsigned int operator()(unsigned int a, unsigned int b) const { return a > b ? a : b; } };
__device__ __forceinline__ float safe_sqrt(float x) { return sqrtf(x > 0.f ? x : 0.f); }

// ---------------------------------------------------------------- domain
// Minimum-image x_ij = x_i - x_j. Positions live inside the periodic box, so one
// conditional shift per periodic axis is exact.
// Written with selects rather than branches (same result as the if / else-if form).
template <int D> __device__ __forceinline__ Vec<D> dist_vec(const Vec<D>& xi, const Vec<D>& xj, const DomainF& dom) {
    Vec<D> r;
    _Pragma("unroll") for (int a = 0; a < D; ++a) {
        float d = __fsub_rn(xi.v[a], xj.v[a]);
        if (dom.periodic[a]) {
            const float dp = __fsub_rn(d, dom.L[a]), dm = __fadd_rn(d, dom.L[a]);
            d = d > dom.halfL[a] ? dp : (d < -dom.halfL[a] ? dm : d);
        }
        r.v[a] = d;
    }
    return r;
}
// Squared distance with explicit round-to-nearest steps (no FMA contraction) so the
// neighbour criterion is bit-identical to the CPU oracle.
template <int D> __device__ __forceinline__ float dist2_rn(const Vec<D>& d) {
    float s = __fmul_rn(d.v[0], d.v[0]);
    _Pragma("unroll") for (int a = 1; a < D; ++a) s = __fadd_rn(s, __fmul_rn(d.v[a], d.v[a]));
    return s;
}

// ---------------------------------------------------------------- kernels
// Wendland functions in q = r/H with support radius H:
//   W(r,H)   = C_D / H^D * k(q)
//   dk/dq    = -q * p(q)          (every Wendland derivative carries a factor q)
//   grad_i W = -C_D / H^(D+2) * p(q) * x_ij
//   dW/dH    = -C_D / H^(D+1) * (D k(q) - q^2 p(q))
// Normalisations C_D integrate W to one; they are the standard Wendland (1995)
// values used by Dehnen & Aly (2012).
//
// B7 is the degree-7 B-spline on q in [0, 1] (knots at 1/4, 1/2, 3/4):
//   k(q) = (1-q)^7 - 8 (3/4-q)^7 + 28 (1/2-q)^7 - 56 (1/4-q)^7   (truncated powers)
// with p(q) = -k'(q)/q.  Below q = 1/4 p is the expanded polynomial
//   105/32 - 35 q^2 + 210 q^4 - 245 q^5
// (the constant term of k' cancels there, so dividing by q would lose digits); above it
// the truncated-power sum divided by q.  C_D = 4096/315, 589824/(7435 pi),
// 16384/(105 pi) integrate it to one in 1, 2 and 3 dimensions.
template <int KF, int D> struct KernelTraits;
template <> struct KernelTraits<SPH_KERNEL_WENDLAND2, 1> { static constexpr float C = 1.25f; };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND2, 2> { static constexpr float C = (float)(7.0 / 3.14159265358979323846); };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND2, 3> { static constexpr float C = (float)(21.0 / (2.0 * 3.14159265358979323846)); };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND4, 1> { static constexpr float C = 1.5f; };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND4, 2> { static constexpr float C = (float)(9.0 / 3.14159265358979323846); };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND4, 3> { static constexpr float C = (float)(495.0 / (32.0 * 3.14159265358979323846)); };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND6, 1> { static constexpr float C = 1.71875f; };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND6, 2> { static constexpr float C = (float)(78.0 / (7.0 * 3.14159265358979323846)); };
template <> struct KernelTraits<SPH_KERNEL_WENDLAND6, 3> { static constexpr float C = (float)(1365.0 / (64.0 * 3.14159265358979323846)); };
template <> struct KernelTraits<SPH_KERNEL_B7, 1> { static constexpr float C = (float)(4096.0 / 315.0); };
template <> struct KernelTraits<SPH_KERNEL_B7, 2> { static constexpr float C = (float)(589824.0 / (7435.0 * 3.14159265358979323846)); };
template <> struct KernelTraits<SPH_KERNEL_B7, 3> { static constexpr float C = (float)(16384.0 / (105.0 * 3.14159265358979323846)); };

// Truncated power (a - q)_+^n.
template <int N> __device__ __forceinline__ float tpow(float a, float q) {
    const float t = a - q;
    if (!(t > 0.f)) return 0.f;
    float r = t;
    _Pragma("unroll") for (int i = 1; i < N; ++i) r *= t;
    return r;
}

// k(q) and p(q) for 0 <= q < 1 (callers handle q >= 1).
template <int KF, int D> __device__ __forceinline__ void kernel_kp(float q, float& k, float& p) {
    float t = 1.f - q;
    if constexpr (KF == SPH_KERNEL_B7) {
        k = tpow<7>(1.f, q) - 8.f * tpow<7>(0.75f, q) + 28.f * tpow<7>(0.5f, q) - 56.f * tpow<7>(0.25f, q);
        if (q < 0.25f) {
            const float q2 = q * q;
            p = 3.28125f + q2 * (-35.f + q2 * (210.f - 245.f * q));
        } else {
            p = 7.f * (tpow<6>(1.f, q) - 8.f * tpow<6>(0.75f, q) + 28.f * tpow<6>(0.5f, q)) / q;
        }
    } else if constexpr (KF == SPH_KERNEL_WENDLAND2) {
        if constexpr (D == 1) { float t2 = t * t; k = t2 * t * (1.f + 3.f * q); p = 12.f * t2; }
        else { float t3 = t * t * t; k = t3 * t * (1.f + 4.f * q); p = 20.f * t3; }
    } else if constexpr (KF == SPH_KERNEL_WENDLAND4) {
        if constexpr (D == 1) { float t4 = (t * t) * (t * t); k = t4 * t * (1.f + 5.f * q + 8.f * q * q); p = 14.f * (1.f + 4.f * q) * t4; }
        else { float t5 = (t * t) * (t * t) * t; k = t5 * t * (1.f + 6.f * q + (35.f / 3.f) * q * q); p = (56.f / 3.f) * (1.f + 5.f * q) * t5; }
    } else {
        if constexpr (D == 1) { float t6 = (t * t) * (t * t) * (t * t); k = t6 * t * (1.f + 7.f * q + 19.f * q * q + 21.f * q * q * q); p = 6.f * (3.f + 18.f * q + 35.f * q * q) * t6; }
        else { float t7 = (t * t) * (t * t) * (t * t) * t; k = t7 * t * (1.f + 8.f * q + 25.f * q * q + 32.f * q * q * q); p = 22.f * (1.f + 7.f * q + 16.f * q * q) * t7; }
    }
}

template <int D> __device__ __forceinline__ float ipow(float h) {
    if constexpr (D == 1) return h; else if constexpr (D == 2) return h * h; else return h * h * h;
}

// W(r, H)
template <int KF, int D> __device__ __forceinline__ float kernelW(float r, float H) {
    float q = r / H;
    if (!(q < 1.f)) return 0.f;
    float k, p; kernel_kp<KF, D>(q, k, p);
    return KernelTraits<KF, D>::C / ipow<D>(H) * k;
}
// W and grad_i W at once.
template <int KF, int D> __device__ __forceinline__ void kernelWG(const Vec<D>& xij, float r, float H, float& W, Vec<D>& g) {
    float q = r / H;
    if (!(q < 1.f)) { W = 0.f; g = vzero<D>(); return; }
    float k, p; kernel_kp<KF, D>(q, k, p);
    float cH = KernelTraits<KF, D>::C / ipow<D>(H);
    W = cH * k;
    float s = -cH * p / (H * H);
    _Pragma("unroll") for (int a = 0; a < D; ++a) g.v[a] = s * xij.v[a];
}
// W and dW/dH.
template <int KF, int D> __device__ __forceinline__ void kernelWdH(float r, float H, float& W, float& dWdH) {
    float q = r / H;
    if (!(q < 1.f)) { W = 0.f; dWdH = 0.f; return; }
    float k, p; kernel_kp<KF, D>(q, k, p);
    float cH = KernelTraits<KF, D>::C / ipow<D>(H);
    W = cH * k;
    dWdH = -cH / H * ((float)D * k - q * q * p);
}

// Pair kernel value for a support scheme.
template <int KF, int D> __device__ __forceinline__ float kernelW_mode(float r, float Hi, float Hj, int mode) {
    switch (mode) {
        case SPH_SUPPORT_GATHER: return kernelW<KF, D>(r, Hi);
        case SPH_SUPPORT_SCATTER: return kernelW<KF, D>(r, Hj);
        case SPH_SUPPORT_SYMMETRIC: return kernelW<KF, D>(r, 0.5f * (Hi + Hj));
        case SPH_SUPPORT_SUPERSYMMETRIC: return kernelW<KF, D>(r, wmax(Hi, Hj));
        default: return 0.5f * (kernelW<KF, D>(r, Hi) + kernelW<KF, D>(r, Hj));
    }
}
template <int KF, int D> __device__ __forceinline__ void kernelWG_mode(const Vec<D>& xij, float r, float Hi, float Hj, int mode, float& W, Vec<D>& g) {
    switch (mode) {
        case SPH_SUPPORT_GATHER: kernelWG<KF, D>(xij, r, Hi, W, g); return;
        case SPH_SUPPORT_SCATTER: kernelWG<KF, D>(xij, r, Hj, W, g); return;
        case SPH_SUPPORT_SYMMETRIC: kernelWG<KF, D>(xij, r, 0.5f * (Hi + Hj), W, g); return;
        case SPH_SUPPORT_SUPERSYMMETRIC: kernelWG<KF, D>(xij, r, wmax(Hi, Hj), W, g); return;
        default: {
            float Wa, Wb; Vec<D> ga, gb;
            kernelWG<KF, D>(xij, r, Hi, Wa, ga);
            kernelWG<KF, D>(xij, r, Hj, Wb, gb);
            W = 0.5f * (Wa + Wb);
            _Pragma("unroll") for (int a = 0; a < D; ++a) g.v[a] = 0.5f * (ga.v[a] + gb.v[a]);
        }
    }
}

// CRK-corrected kernel gradient (Frontiere, Raskin & Owen 2017, eq. for d W^R_ij):
//   W^R = A (1 + B.x) W,  x = x_ij
//   d_g W^R = A (1+B.x) d_g W + A B_g W + d_g A (1+B.x) W + A (sum_a dB^a/dx^g x^a) W
// gB[a][g] = dB^a/dx^g.
template <int D> __device__ __forceinline__ Vec<D> crk_grad(const Vec<D>& x, float W, const Vec<D>& gW,
                                                            float A, const Vec<D>& B, const Vec<D>& gA, const Mat<D>& gB) {
    float bx = 1.f + dot<D>(B, x);
    Vec<D> r;
    _Pragma("unroll") for (int g = 0; g < D; ++g) {
        float gbx = gB.m[0][g] * x.v[0];
        _Pragma("unroll") for (int a = 1; a < D; ++a) gbx += gB.m[a][g] * x.v[a];
        r.v[g] = A * bx * gW.v[g] + A * B.v[g] * W + gA.v[g] * bx * W + A * gbx * W;
    }
    return r;
}

// ---------------------------------------------------------------- dispatch helpers
#define WSPH_DISPATCH_DIM(dim, ...)                                  \
    switch (dim) {                                                   \
        case 1: { constexpr int D = 1; __VA_ARGS__; } break;         \
        case 2: { constexpr int D = 2; __VA_ARGS__; } break;         \
        case 3: { constexpr int D = 3; __VA_ARGS__; } break;         \
        default: break;                                              \
    }
#define WSPH_DISPATCH_KD(kernel, dim, ...)                                                            \
    switch (kernel) {                                                                                 \
        case SPH_KERNEL_WENDLAND2: { constexpr int KF = SPH_KERNEL_WENDLAND2; WSPH_DISPATCH_DIM(dim, __VA_ARGS__) } break; \
        case SPH_KERNEL_WENDLAND4: { constexpr int KF = SPH_KERNEL_WENDLAND4; WSPH_DISPATCH_DIM(dim, __VA_ARGS__) } break; \
        case SPH_KERNEL_WENDLAND6: { constexpr int KF = SPH_KERNEL_WENDLAND6; WSPH_DISPATCH_DIM(dim, __VA_ARGS__) } break; \
        case SPH_KERNEL_B7: { constexpr int KF = SPH_KERNEL_B7; WSPH_DISPATCH_DIM(dim, __VA_ARGS__) } break;               \
        default: break;                                                                               \
    }

// ---------------------------------------------------------------- programmatic dependent launch
// A kernel launched by launch_pdl (host side, sph_pair_common.cuh) starts with pdl_entry():
// it lets the next kernel of the stream begin launching once every block of this one has
// started (its blocks then wait on the SMs instead of behind a launch), and waits until the
// kernel before it has completed and its writes are visible before touching memory.
__device__ __forceinline__ void pdl_entry() {
    cudaTriggerProgrammaticLaunchCompletion();
    cudaGridDependencySynchronize();
}

// ---------------------------------------------------------------- host side
int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);
void count_launch();
int params_to_dev(const SphParams* p, DevParams* out);
double kernel_norm(int kernel, int dim);
double kernel_scale(int kernel, int dim);

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }

// Exclusive scan of int32 values with a device int64 total (sph_neighbors.cu), and the
// bytes of workspace it needs for n values.
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, char* ws, long long* total, cudaStream_t s,
                        const unsigned int* gate = nullptr);
int64_t scan_ws_bytes(int64_t n);

}  // namespace wsph

#define WSPH_CHECK_PTR(ptr) do { if (!(ptr)) return wsph::set_error(SPH_ERR_BAD_ARG, "%s: null pointer '%s'", __func__, #ptr); } while (0)
#define WSPH_STREAM(s) (reinterpret_cast<cudaStream_t>(s))
