// Pair bodies of the weakly compressible delta-SPH right-hand side, shared by the
// single-list entry point (sph_deltasph.cu) and the batched ensemble (sph_ensemble.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstring>
#include "sph_pair_common.cuh"

namespace wsph {

struct WcDev {
    float rho0, c0, gamma, kappa, delta, nu, alpha;
    int inviscid, density_scheme, pressure_term, eos;
    float xi;           // kernel xi (= kernel scale H/h)
    float visc_nu;      // 2 (d + 2) nu, the viscous factor of wp_viscosityDelta.py:97
};

inline int wc_to_dev(const SphWcParams* w, const DevParams& P, WcDev* o) {
    memset(o, 0, sizeof(*o));
    o->rho0 = (float)w->rest_density; o->c0 = (float)w->sound_speed; o->gamma = (float)w->polytropic_exponent;
    o->kappa = (float)w->kappa; o->delta = (float)w->density_delta; o->nu = (float)w->viscosity_nu; o->alpha = (float)w->inviscid_alpha;
    o->inviscid = w->inviscid; o->density_scheme = w->density_scheme; o->pressure_term = w->pressure_term; o->eos = w->eos;
    o->xi = P.kscale;
    o->visc_nu = 2.f * (float)(P.dim + 2) * o->nu;
    if (o->eos < SPH_EOS_STIFF_TAIT || o->eos > SPH_EOS_MURNAGHAN) return set_error(SPH_ERR_BAD_ARG, "unknown EOS %d", o->eos);
    if (o->density_scheme != SPH_DENSITY_DIFFUSION_DELTA && o->density_scheme != SPH_DENSITY_DIFFUSION_DENSITY_ONLY &&
        o->density_scheme != SPH_DENSITY_DIFFUSION_DELTA_ONLY)
        return set_error(SPH_ERR_UNSUPPORTED, "density diffusion scheme %d is not on this path", o->density_scheme);
    if (o->pressure_term < 0 || o->pressure_term > 5) return set_error(SPH_ERR_BAD_ARG, "unknown pressure term %d", o->pressure_term);
    if (!(o->rho0 > 0.f)) return set_error(SPH_ERR_BAD_ARG, "rest density must be > 0");
    return SPH_OK;
}

// modules/eos/weaklyCompressible.py:4-44
__device__ __forceinline__ float wc_eos(const WcDev& W, float rho) {
    switch (W.eos) {
        case SPH_EOS_STIFF_TAIT: return W.rho0 * W.c0 * W.c0 / W.gamma * (powf(rho / W.rho0, W.gamma) - 1.f);
        case SPH_EOS_TAIT: return W.kappa * (rho - W.rho0);
        case SPH_EOS_ISOTHERMAL: return W.c0 * W.c0 * (rho - W.rho0);
        case SPH_EOS_POLYTROPIC: return W.kappa * powf(rho, W.gamma);
        default: return W.kappa / W.gamma * (powf(rho / W.rho0, W.gamma) - 1.f);
    }
}

static __global__ void k_wc_eos(int n, WcDev W, const float* __restrict__ rho, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = wc_eos(W, rho[i]);
}

// Loads of the pair passes.  CG: ld.global.cg (L2, coherent across blocks) for arrays
// that other blocks rewrite inside one persistent launch; otherwise the read-only path.
template <bool CG> __device__ __forceinline__ float ldf(const float* p) { return CG ? __ldcg(p) : __ldg(p); }
template <int D, bool CG> __device__ __forceinline__ Vec<D> ldv(const float* p, int i) {
    Vec<D> r;
    if constexpr (D == 2) {
        const float2 t = CG ? __ldcg(reinterpret_cast<const float2*>(p) + i) : __ldg(reinterpret_cast<const float2*>(p) + i);
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        #pragma unroll
        for (int a = 0; a < D; ++a) r.v[a] = ldf<CG>(p + (size_t)i * D + a);
    }
    return r;
}

// Renormalisation of pass A: L = M^-1 with M_ab = sum_j V_j gradW_a (x_j - x_i)_b; a
// (near-)singular M (isolated particle) leaves the gradient unrenormalised.
template <int D> __device__ __forceinline__ Vec<D> renormalise(const Mat<D>& M, const Vec<D>& g) {
    Vec<D> r = g;
    if constexpr (D == 1) {
        if (fabsf(M.m[0][0]) > 1e-6f) r.v[0] = g.v[0] / M.m[0][0];
    } else if constexpr (D == 2) {
        const float det = M.m[0][0] * M.m[1][1] - M.m[0][1] * M.m[1][0];
        if (fabsf(det) > 1e-6f) {
            const float id = 1.f / det;
            r.v[0] = id * (M.m[1][1] * g.v[0] - M.m[0][1] * g.v[1]);
            r.v[1] = id * (-M.m[1][0] * g.v[0] + M.m[0][0] * g.v[1]);
        }
    } else {
        const float c00 = M.m[1][1] * M.m[2][2] - M.m[1][2] * M.m[2][1];
        const float c01 = M.m[1][2] * M.m[2][0] - M.m[1][0] * M.m[2][2];
        const float c02 = M.m[1][0] * M.m[2][1] - M.m[1][1] * M.m[2][0];
        const float det = M.m[0][0] * c00 + M.m[0][1] * c01 + M.m[0][2] * c02;
        if (fabsf(det) > 1e-6f) {
            const float id = 1.f / det;
            const float i00 = c00, i01 = M.m[0][2] * M.m[2][1] - M.m[0][1] * M.m[2][2], i02 = M.m[0][1] * M.m[1][2] - M.m[0][2] * M.m[1][1];
            const float i10 = c01, i11 = M.m[0][0] * M.m[2][2] - M.m[0][2] * M.m[2][0], i12 = M.m[0][2] * M.m[1][0] - M.m[0][0] * M.m[1][2];
            const float i20 = c02, i21 = M.m[0][1] * M.m[2][0] - M.m[0][0] * M.m[2][1], i22 = M.m[0][0] * M.m[1][1] - M.m[0][1] * M.m[1][0];
            r.v[0] = id * (i00 * g.v[0] + i01 * g.v[1] + i02 * g.v[2]);
            r.v[1] = id * (i10 * g.v[0] + i11 * g.v[1] + i12 * g.v[2]);
            r.v[2] = id * (i20 * g.v[0] + i21 * g.v[1] + i22 * g.v[2]);
        }
    }
    return r;
}

// Per-lane partial sums of pass A for particle i.
template <int KF, int D, int G, bool CG = false>
__device__ __forceinline__ void passA_partial(int i, int lane, const DevParams& P, const float* x,
                                              const float* __restrict__ H, const float* __restrict__ m,
                                              const float* rho, const int32_t* __restrict__ offs,
                                              const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, Mat<D>& M,
                                              Vec<D>& g) {
    const Vec<D> xi = ldv<D, CG>(x, i);
    const float Hi = H[i], rhoi = ldf<CG>(rho + i);
    const int b = offs[i], e = b + cnt[i];
    for (int q = b + lane; q < e; q += G) {
        int j, k; entry(list, q, j, k);
        const Vec<D> xij = dist_vec<D>(xi, ldv<D, CG>(x, j), P.dom);
        const float r = safe_sqrt(dot<D>(xij, xij));
        float W; Vec<D> gW;
        kernelWG<KF, D>(xij, r, wmax(Hi, __ldg(H + j)), W, gW);
        const float rj = ldf<CG>(rho + j);
        const float Vj = __ldg(m + j) / rj;
        const float dr = rj - rhoi;
        #pragma unroll
        for (int a = 0; a < D; ++a) {
            g.v[a] += Vj * dr * gW.v[a];
            #pragma unroll
            for (int c = 0; c < D; ++c) M.m[a][c] += Vj * gW.v[a] * (-xij.v[c]);
        }
    }
}

template <int D, int G> __device__ __forceinline__ void passA_reduce(Mat<D>& M, Vec<D>& g) {
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        g.v[a] = gsum<G>(g.v[a]);
        #pragma unroll
        for (int c = 0; c < D; ++c) M.m[a][c] = gsum<G>(M.m[a][c]);
    }
}

// Per-lane partial sums of pass B for particle i: cont = sum V (v_j - v_i).gW,
// dd = sum V psi.gW, pf = sum V p_ij gW, visc = sum V mu f gW / rho_bar.  With FULL
// false only cont and visc are formed (gL and Pr are not read): the velocity diffusion
// and continuity of the DFSPH step.  smask (nullable) is the free-surface indicator of
// each particle; the Antuono pressure term takes P_j + P_i when P_i >= 0, P_j >= 0 or
// particle i lies on the free surface (wp_surfaceAware.py:89-92).
template <int KF, int D, int G, bool CG = false, bool FULL = true>
__device__ __forceinline__ void passB_partial(int i, int lane, const DevParams& P, const WcDev& W, const float* x,
                                              const float* __restrict__ H, const float* __restrict__ m, const float* rho,
                                              const float* v, const float* gL, const float* Pr, const int32_t* __restrict__ smask,
                                              const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                                              const int32_t* __restrict__ list, float& cont, float& dd, Vec<D>& pf, Vec<D>& visc) {
    const Vec<D> xi = ldv<D, CG>(x, i), vi = ldv<D, CG>(v, i);
    const Vec<D> gLi = FULL ? ldv<D, CG>(gL, i) : vzero<D>();
    const float Hi = H[i], rhoi = ldf<CG>(rho + i), Pi = FULL ? ldf<CG>(Pr + i) : 0.f;
    const bool surf_i = FULL && smask != nullptr && smask[i] == 1;
    const float eps = 1.0e-14f * Hi;
    const float factor = W.inviscid ? W.alpha * W.c0 * Hi / W.xi : W.visc_nu;
    const int b = offs[i], e = b + cnt[i];
    for (int q = b + lane; q < e; q += G) {
        int j, k; entry(list, q, j, k);
        const Vec<D> xij = dist_vec<D>(xi, ldv<D, CG>(x, j), P.dom);
        const float r2 = dot<D>(xij, xij);
        const float r = safe_sqrt(r2);
        float Wv; Vec<D> gW;
        kernelWG<KF, D>(xij, r, wmax(Hi, __ldg(H + j)), Wv, gW);
        const float rj = ldf<CG>(rho + j);
        const float Vj = __ldg(m + j) / rj;
        const Vec<D> vj = ldv<D, CG>(v, j);
        // continuity (inconsistent.py:19-31): V_j (v_j - v_i).gW
        float t = 0.f;
        #pragma unroll
        for (int a = 0; a < D; ++a) t += (vj.v[a] - vi.v[a]) * gW.v[a];
        cont += Vj * t;
        // density diffusion (wp_densityDelta.py:88-117)
        if constexpr (FULL) {
            const Vec<D> gLj = ldv<D, CG>(gL, j);
            const float inv = 1.f / (r + eps);
            const float s = 2.f * (rj - rhoi) * inv * inv;      // 2 (rho_j - rho_i) n_ij / (r + eps), n_ij = x_ij / (r + eps)
            float pd = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                float psi;
                if (W.density_scheme == SPH_DENSITY_DIFFUSION_DELTA) psi = (gLi.v[a] + gLj.v[a]) - s * xij.v[a];
                else if (W.density_scheme == SPH_DENSITY_DIFFUSION_DENSITY_ONLY) psi = -(s * xij.v[a]);
                else psi = gLi.v[a] + gLj.v[a];
                pd += psi * gW.v[a];
            }
            dd += Vj * pd;
        }
        // pressure (wp_surfaceAware.py:48-102)
        if constexpr (FULL) {
            const float Pj = ldf<CG>(Pr + j);
            float pij;
            switch (W.pressure_term) {
                case SPH_PRESSURE_CONSERVATIVE: pij = Pj - Pi; break;
                case SPH_PRESSURE_NONCONSERVATIVE: pij = Pj + Pi; break;
                case SPH_PRESSURE_ANTUONO: pij = (Pi >= 0.f || Pj >= 0.f || surf_i) ? Pj + Pi : Pj - Pi; break;
                case SPH_PRESSURE_I: pij = Pi; break;
                case SPH_PRESSURE_J: pij = Pj; break;
                default: pij = (Pj / (rj * rj) + Pi / (rhoi * rhoi)) * rj; break;
            }
            #pragma unroll
            for (int a = 0; a < D; ++a) pf.v[a] += Vj * pij * gW.v[a];
        }
        // velocity diffusion (wp_viscosityDelta.py:86-106)
        {
            float vx = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) vx += (vi.v[a] - vj.v[a]) * xij.v[a];
            float mu = vx / (r2 + eps * Hi);
            mu = mu > 0.f ? 0.f : mu;
            const float w = Vj * mu * factor / ((rj + rhoi) / 2.f);
            #pragma unroll
            for (int a = 0; a < D; ++a) visc.v[a] += w * gW.v[a];
        }
    }
}

// pass B output: drhodt = -rho cont + delta (H / xi) c0 dd, dvdt = -pf / rho_i + visc
// (the pressure force is divided by the particle's own density, wp_surfaceAware.py:207-218).
template <int D> __device__ __forceinline__ void passB_finish(const WcDev& W, float rhoi, float Hi, float cont, float dd, const Vec<D>& pf,
                                                               const Vec<D>& visc, float& drho, Vec<D>& dv) {
    drho = -rhoi * cont + W.delta * Hi / W.xi * W.c0 * dd;
    #pragma unroll
    for (int a = 0; a < D; ++a) dv.v[a] = -pf.v[a] / rhoi + visc.v[a];
}

// Pass A: gradRhoL [n, D] and the EOS pressure P [n].
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_ds_passA(int n, DevParams P, WcDev W, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
           const float* __restrict__ rho, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
           const int32_t* __restrict__ list, float* __restrict__ gL, float* __restrict__ Pr) {
    Grp<G> g(n);
    Mat<D> M = mzero<D>();
    Vec<D> s = vzero<D>();
    if (g.valid) passA_partial<KF, D, G>(g.i, g.lane, P, x, H, m, rho, offs, cnt, list, M, s);
    passA_reduce<D, G>(M, s);
    if (g.valid && g.lane == 0) {
        store_vec<D>(gL, g.i, renormalise<D>(M, s));
        Pr[g.i] = wc_eos(W, rho[g.i]);
    }
}

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_ds_passB(int n, DevParams P, WcDev W, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
           const float* __restrict__ rho, const float* __restrict__ v, const float* __restrict__ gL, const float* __restrict__ Pr,
           const int32_t* __restrict__ smask, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
           const int32_t* __restrict__ list, float* __restrict__ dvdt, float* __restrict__ drhodt) {
    Grp<G> g(n);
    float cont = 0.f, dd = 0.f;
    Vec<D> pf = vzero<D>(), visc = vzero<D>();
    if (g.valid) passB_partial<KF, D, G>(g.i, g.lane, P, W, x, H, m, rho, v, gL, Pr, smask, offs, cnt, list, cont, dd, pf, visc);
    cont = gsum<G>(cont); dd = gsum<G>(dd);
    #pragma unroll
    for (int a = 0; a < D; ++a) { pf.v[a] = gsum<G>(pf.v[a]); visc.v[a] = gsum<G>(visc.v[a]); }
    if (!g.valid || g.lane != 0) return;
    float dr; Vec<D> dv;
    passB_finish<D>(W, rho[g.i], H[g.i], cont, dd, pf, visc, dr, dv);
    drhodt[g.i] = dr;
    store_vec<D>(dvdt, g.i, dv);
}

// Velocity diffusion and continuity alone (dfsph.py:100-109): dvdt = visc,
// drhodt = -rho cont, bit for bit what pass B gives with P = 0 and delta = 0.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_visc_cont(int n, DevParams P, WcDev W, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
            const float* __restrict__ rho, const float* __restrict__ v, const int32_t* __restrict__ offs,
            const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float* __restrict__ dvdt, float* __restrict__ drhodt) {
    Grp<G> g(n);
    float cont = 0.f, dd = 0.f;
    Vec<D> pf = vzero<D>(), visc = vzero<D>();
    if (g.valid) passB_partial<KF, D, G, false, false>(g.i, g.lane, P, W, x, H, m, rho, v, nullptr, nullptr, nullptr, offs, cnt, list, cont, dd, pf,
                                                       visc);
    cont = gsum<G>(cont);
    #pragma unroll
    for (int a = 0; a < D; ++a) visc.v[a] = gsum<G>(visc.v[a]);
    if (!g.valid || g.lane != 0) return;
    const float rhoi = rho[g.i];
    drhodt[g.i] = -rhoi * cont + 0.f * dd;
    Vec<D> dv;
    #pragma unroll
    for (int a = 0; a < D; ++a) dv.v[a] = -pf.v[a] + visc.v[a];
    store_vec<D>(dvdt, g.i, dv);
}

// ---------------------------------------------------------------- delta-plus shift
// max_i |v_i| over the finite magnitudes (shifting/delta.py:10-17): red[0] holds the
// float bits of the running maximum (non-negative, so integer order is float order),
// red[1] counts finite magnitudes.
template <int D>
__global__ void k_vmax(int n, const float* __restrict__ v, unsigned int* __restrict__ red) {
    float vmax = 0.f;
    unsigned int finite = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        #pragma unroll
        for (int a = 0; a < D; ++a) { const float c = v[(size_t)i * D + a]; s += c * c; }
        const float mag = sqrtf(s);
        if (isfinite(mag)) { vmax = fmaxf(vmax, mag); finite = 1u; }
    }
    vmax = block_reduce(vmax, 0.f, OpMaxF());
    finite = block_reduce(finite, 0u, OpMaxU());
    if (threadIdx.x == 0) {
        atomicMax(red, __float_as_uint(vmax));
        if (finite) atomicOr(red + 1, 1u);
    }
}

// shift_i = -CFL Ma 2 (H_i / xi)^2 sum_j (1 + R (W_ij / W_0)^n) m_j / (2 (rho_i + rho_j)) gradW_ij
// (sample/wp_deltaShift.py:57-126 and shifting/delta.py:18-45), gather support H_i,
// W_0 = W((m_j / rho0)^(1/d) / xi, H_i), Ma = max|v| / c0 (0.1 below 1e-6), zero for
// particles of kind != 0 (shifting/wrapper.py:100).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_delta_shift(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
              const float* __restrict__ rho, const int32_t* __restrict__ kinds, const int32_t* __restrict__ offs,
              const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float cfl, float c0, float R, int nexp, float rho0,
              const unsigned int* __restrict__ red, float* __restrict__ shift) {
    Grp<G> g(n);
    Vec<D> s = vzero<D>();
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i], rhoi = rho[i];
        const float xi_k = P.kscale;
        const int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            float Wij; Vec<D> gW;
            kernelWG<KF, D>(xij, r, Hi, Wij, gW);
            const float mj = __ldg(m + j);
            const float dxs = powf(mj / rho0, 1.f / (float)D) / xi_k;
            const float q0 = dxs / Hi;
            float k0 = 0.f, p0;
            if (q0 < 1.f) kernel_kp<KF, D>(q0, k0, p0);
            const float W0 = k0 * KernelTraits<KF, D>::C / ipow<D>(Hi);   // eval_k * eval_C_d / h^d
            const float term = 1.f + R * powf(Wij / W0, (float)nexp);
            const float dterm = 0.5f * mj / (rhoi + __ldg(rho + j));
            const float sc = term * dterm;
            #pragma unroll
            for (int a = 0; a < D; ++a) s.v[a] += sc * gW.v[a];
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) s.v[a] = gsum<G>(s.v[a]);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    float cmax = red[1] ? __uint_as_float(red[0]) / c0 : __int_as_float(0x7fc00000);
    const float Ma = cmax < 1e-6f ? 0.1f : cmax;
    const float h = H[i] / P.kscale;
    const float scale = -cfl * Ma * 2.f * (h * h);
    Vec<D> o;
    const bool moving = kinds == nullptr || kinds[i] == 0;
    #pragma unroll
    for (int a = 0; a < D; ++a) o.v[a] = moving ? s.v[a] * scale : 0.f;
    store_vec<D>(shift, i, o);
}

}  // namespace wsph
