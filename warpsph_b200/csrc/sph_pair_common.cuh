// Shared pieces of the pair passes: G lanes of a warp per particle, row-entry
// decoding (Verlet rows or their interacting prefixes), kernel
// evaluation with a precomputed 1/H, group reductions, and the host-side argument
// checks and template dispatch of the pair entry points.
#pragma once
#include <cstring>
#include <cuda_runtime.h>
#include "sph_common.cuh"

namespace wsph {

constexpr int PAIR_BLOCK = 128;

// ---------------------------------------------------------------- group helpers
template <int G> struct Grp {
    int i, lane;
    bool valid;
    __device__ __forceinline__ explicit Grp(int n) {
        int t = blockIdx.x * blockDim.x + threadIdx.x;
        i = t / G;
        lane = threadIdx.x & (G - 1);
        valid = i < n;
    }
};
template <int G> __device__ __forceinline__ float gsum(float v) {
    #pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <int G> __device__ __forceinline__ float gmaxw(float v) {
    #pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = wmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Row entry q: neighbour j and the Verlet entry index k that pairwise arrays use (the
// rows a pass walks are Verlet rows or their interacting prefixes, so k = q).
__device__ __forceinline__ void entry(const int32_t* __restrict__ list, int q, int& j, int& k) {
    j = __ldg(list + q); k = q;
}
// One lane's walk over a row (entries q0, q0 + step, ... < e) with the neighbour index loaded
// two entries ahead and the neighbour's D-vector from `src` one entry ahead: the dependent
// global loads of an entry are in flight while the entry before it is computed.  Past the
// row's end the prefetches read index 0 (a valid particle whenever a row is walked).
template <int D> struct RowPipe {
    const int32_t* __restrict__ list;
    const float* __restrict__ src;
    int e, step, j1, j2;
    Vec<D> v1;
    __device__ __forceinline__ RowPipe(const int32_t* __restrict__ l, const float* __restrict__ s, int q0, int e_, int st)
        : list(l), src(s), e(e_), step(st) {
        j1 = q0 < e_ ? __ldg(l + q0) : 0;
        j2 = q0 + st < e_ ? __ldg(l + q0 + st) : 0;
        v1 = load_vec<D>(s, j1);
    }
    // the entry at q (the caller's loop index, q0 + k * step): its neighbour and vector
    __device__ __forceinline__ void take(int q, int& j, Vec<D>& vj) {
        j = j1;
        vj = v1;
        j1 = j2;
        v1 = load_vec<D>(src, j1);
        j2 = q + 2 * step < e ? __ldg(list + q + 2 * step) : 0;
    }
};

template <int G> __host__ __forceinline__ int grid_g(int64_t n) { return (int)((n * G + PAIR_BLOCK - 1) / PAIR_BLOCK); }

// W and grad_i W with a precomputed 1/H.
template <int KF, int D> __device__ __forceinline__ float kW_inv(float r, float invH) {
    float q = r * invH;
    if (!(q < 1.f)) return 0.f;
    float k, p; kernel_kp<KF, D>(q, k, p);
    return KernelTraits<KF, D>::C * ipow<D>(invH) * k;
}
template <int KF, int D> __device__ __forceinline__ void kWG_inv(const Vec<D>& x, float r, float invH, float& W, Vec<D>& g) {
    float q = r * invH;
    if (!(q < 1.f)) { W = 0.f; g = vzero<D>(); return; }
    float k, p; kernel_kp<KF, D>(q, k, p);
    float cH = KernelTraits<KF, D>::C * ipow<D>(invH);
    W = cH * k;
    float s = -cH * p * (invH * invH);
    #pragma unroll
    for (int a = 0; a < D; ++a) g.v[a] = s * x.v[a];
}

// Neumaier-compensated accumulator (DevParams::kahan).
struct KSum {
    float s, c;
    __device__ __forceinline__ void init() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float x, bool comp) {
        if (!comp) { s += x; return; }
        float t = s + x;
        if (fabsf(s) >= fabsf(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
};

// group sizes (lanes per particle) of the pair passes (a build may override them)
#ifndef G_LIGHT
#define G_LIGHT 8
#endif
#ifndef G_HEAVY
#define G_HEAVY 8
#endif
#ifndef G_CRK
#define G_CRK 4
#endif
// Lanes per particle of the light gather passes that walk long rows (adaptive support,
// CRK volume, velocity gradient, Cullen switch): in 3D, 4 lanes with twice the
// iterations each beat 8 (measured on the 128^3 Sedov case: Cullen 13.7 -> 10.8 ms,
// adaptive support 6.1 -> 5.2, velocity gradient 6.9 -> 6.0 per step).
#define G_SCAN(D) ((D) == 3 ? 4 : G_LIGHT)
// Lanes per particle of the CRK accel pass: 4 (measured against 8: 0.241 vs 0.245 ms per
// launch at 512^2 in 2D, 27.6 vs 28.7 ms per step at 128^3 in 3D).
#ifndef G_ACCEL
#define G_ACCEL 4
#endif

#define WSPH_DISPATCH_KDS(params, ...) WSPH_DISPATCH_KD(P.kernel, P.dim, __VA_ARGS__)
#define WSPH_DISPATCH_DS(params, ...) WSPH_DISPATCH_DIM(P.dim, __VA_ARGS__)

// Launch with programmatic stream serialization (the kernel must begin with pdl_entry()).
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    memset(at, 0, sizeof(at));
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, kern, args...);
}

#define PAIR_PRELUDE()                                                        \
    DevParams P;                                                              \
    int rc = params_to_dev(p, &P);                                            \
    if (rc) return rc;                                                        \
    if (n < 0 || n > 0x3fffffff) return set_error(SPH_ERR_BAD_ARG, "%s: n out of range", __func__); \
    if (p->list_stride < 0 || p->list_stride > 1) return set_error(SPH_ERR_BAD_ARG, "%s: list_stride must be 1 (rows are Verlet rows or their interacting prefixes)", __func__); \
    if (n == 0) return SPH_OK;                                                \
    cudaStream_t s = WSPH_STREAM(stream);                                     \
    (void)s;

#define CHECK_CSR() do { WSPH_CHECK_PTR(offs); WSPH_CHECK_PTR(cnt); WSPH_CHECK_PTR(list); } while (0)

inline int check_align_vec(const DevParams& P, const void* ptr, const char* name) {
    if (P.dim == 2 && ptr && (reinterpret_cast<uintptr_t>(ptr) & 7))
        return set_error(SPH_ERR_BAD_ARG, "%s must be 8-byte aligned for dim 2", name);
    return SPH_OK;
}

}  // namespace wsph
