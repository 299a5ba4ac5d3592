// SPH pair-interaction kernels of the compressible (CRKSPH / CompSPH) hot path.
//
// Layout: G lanes of a warp cooperate on one particle i.  Lane l walks the entries
// b+l, b+l+G, ... of i's neighbour row, so the G lanes read G consecutive entries
// (coalesced index loads and pair-array stores), accumulate per-lane partial sums,
// and reduce them with warp shuffles inside the group.  A row is either a whole Verlet
// row or its interacting prefix (the list builder stores the entries with
// r < max(H_i, H_j) first), which removes the beyond-support entries -- about half of
// a Verlet row -- from every pass that only needs W != 0.  The entry index of a pair
// is its position in the Verlet list in both cases.
//
// Arithmetic restates the reference (file:line at each kernel); divisions by the
// same quantity are replaced by multiplications with a reciprocal, so results
// differ from the CPU oracle by rounding only.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cfloat>
#include <atomic>
#include <mutex>
#include "sph_pair_common.cuh"
#include "sph_pinv.cuh"

namespace wsph {

// ---------------------------------------------------------------- density (modules/density/density.py:16-28)
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_density(int n, int mode, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
          const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
          float* __restrict__ rho) {
    pdl_entry();
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) {
        Vec<D> xi = load_vec<D>(x, g.i);
        float Hi = H[g.i];
        int b = offs[g.i], e = b + cnt[g.i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            s += __ldg(m + j) * kernelW_mode<KF, D>(r, Hi, __ldg(H + j), mode);
        }
    }
    s = gsum<G>(s);
    if (g.valid && g.lane == 0) rho[g.i] = s;
}

// ---------------------------------------------------------------- adaptive support
// h(V) of utils/support.py:24-44 (volumeToSupportHelper)
template <int D> __device__ __forceinline__ float volume_to_support(float V, float nH) {
    if constexpr (D == 1) return nH * V / 2.f;
    else if constexpr (D == 2) return sqrtf(nH * V / 3.14159265358979f);
    else return powf(nH * V / 3.14159265358979f * 3.f / 4.f, 1.f / 3.f);
}

// One Newton iteration of modules/adaptiveSupport/optimalSupportMonaghan.py:87-125
// with Omega of modules/adaptiveSupport/wp_omega.py:40-60 (gather support).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_adaptive_h(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
             const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
             const float* __restrict__ hb, float* __restrict__ rho_out, float* __restrict__ H_out, float* __restrict__ ratio) {
    pdl_entry();
    Grp<G> g(n);
    float rs = 0.f, ds = 0.f, Hi = 1.f;
    if (g.valid) {
        Vec<D> xi = load_vec<D>(x, g.i);
        Hi = H[g.i];
        int b = offs[g.i], e = b + cnt[g.i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            // the mass ahead of the kernel evaluation in 1D and 2D; in 3D most Verlet entries
            // lie outside the support, whose kernel values are 0 (the load is skipped for them)
            const float mj_ahead = D < 3 ? __ldg(m + j) : 0.f;
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W, dWdH;
            kernelWdH<KF, D>(r, Hi, W, dWdH);
            const float mj = D < 3 ? mj_ahead : (W != 0.f || dWdH != 0.f ? __ldg(m + j) : 0.f);
            rs += mj * W;
            ds += mj * dWdH;
        }
    }
    rs = gsum<G>(rs);
    ds = gsum<G>(ds);
    if (!g.valid || g.lane != 0) return;
    float rho = rs;
    float safe_rho = isfinite(rho) ? fmaxf(rho, 1e-12f) : 1.f;
    float Fv = Hi - volume_to_support<D>(m[g.i] / safe_rho, P.target_neighbors);
    float dh_drho = -Hi / (rho * (float)D);
    float omega = 1.f - dh_drho * ds;
    if (!isfinite(omega)) omega = 0.f;
    float step = Fv / (omega + 1e-6f);
    if (!isfinite(step)) step = 0.f;
    float hn = Hi - step;
    if (!isfinite(hn)) hn = Hi;
    hn = fminf(fmaxf(hn, hb[0] * 0.25f), hb[1] * 4.f);
    rho_out[g.i] = rho;
    H_out[g.i] = hn;
    if (ratio) ratio[g.i] = hn / (Hi + 1e-6f);
}

// ---------------------------------------------------------------- Owen adaptive support
// One iteration of modules/adaptiveSupport/optimalSupportOwen.py:70-108 for every particle:
//   psi0_i  = (sum_j h_i^d W(r_ij, h_i))^(1/d), psi0H_i = (sum_j h_i^(d+1) |grad W(r_ij, h_i)|)^(1/d)
//             (wp_psi0.py:46-98, gather support; h^k taken as 1 / h^-k as there),
//   n_h_i   = the (psiH -> n_h) table linearly interpolated at psi0H_i in FP64 (owenLUT.py:6-12,
//             64-67: index of the last entry <= psi0H, clamped to the table, weight clamped to [0, 1]),
//   s = target / n_h_i, a = 0.4 (1 + s^-3) if s >= 1 else 0.4 (1 + s^2), h_new = (1 - a + a s) h
//             (optimalSupportOwen.py:27-33), clamped to [hbounds[0] / 4, 4 hbounds[1]] (:96);
//   ratio   = h_new / h (:100).
__device__ __forceinline__ float owen_nh(const double* __restrict__ lut_nh, const double* __restrict__ lut_psiH, int nlut, float psiH) {
    const double x = (double)psiH;
    int lo = 0, hi = nlut;                       // first index with lut_psiH[idx] > x
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(lut_psiH + mid) <= x) lo = mid + 1; else hi = mid;
    }
    int il = lo - 1;
    il = il < 0 ? 0 : (il > nlut - 2 ? nlut - 2 : il);
    const double xl = __ldg(lut_psiH + il), xr = __ldg(lut_psiH + il + 1);
    double alpha = (x - xl) / (xr - xl);
    alpha = alpha < 0.0 ? 0.0 : (alpha > 1.0 ? 1.0 : alpha);
    return (float)(__ldg(lut_nh + il) * (1.0 - alpha) + __ldg(lut_nh + il + 1) * alpha);
}

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_owen(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H,
       const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
       const double* __restrict__ lut_nh, const double* __restrict__ lut_psiH, int nlut, float target,
       const float* __restrict__ hb, float* __restrict__ psi0_out, float* __restrict__ psiH_out,
       float* __restrict__ H_out, float* __restrict__ ratio) {
    pdl_entry();
    Grp<G> g(n);
    float sW = 0.f, sG = 0.f, Hi = 1.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        Hi = H[i];
        const float invHi = 1.f / Hi;
        const float hsW = 1.f / powf(Hi, -(float)D), hsG = 1.f / powf(Hi, -(float)(D + 1));
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, r, invHi, W, gW);
            sW += hsW * W;
            sG += hsG * safe_sqrt(dot<D>(gW, gW));
        }
    }
    sW = gsum<G>(sW);
    sG = gsum<G>(sG);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float psi0 = powf(sW, 1.f / (float)D), psiH = powf(sG, 1.f / (float)D);
    const float nh = owen_nh(lut_nh, lut_psiH, nlut, psiH);
    const float s = target / nh;
    const float a = s >= 1.f ? 0.4f * (1.f + powf(s, -3.f)) : 0.4f * (1.f + powf(s, 2.f));
    float hn = (1.f - a + a * s) * Hi;
    hn = fminf(fmaxf(hn, hb[0] * 0.25f), hb[1] * 4.f);
    if (psi0_out) psi0_out[i] = psi0;
    if (psiH_out) psiH_out[i] = psiH;
    H_out[i] = hn;
    if (ratio) ratio[i] = hn / Hi;
}

// ---------------------------------------------------------------- CRK volume (scatter support)
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_crk_volume(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H,
             const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
             float* __restrict__ V) {
    pdl_entry();
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) {
        Vec<D> xi = load_vec<D>(x, g.i);
        int b = offs[g.i], e = b + cnt[g.i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            s += kW_inv<KF, D>(r, 1.f / __ldg(H + j));
        }
    }
    s = gsum<G>(s);
    if (g.valid && g.lane == 0) V[g.i] = 1.f / s;
}

// Inverse of a symmetric DxD matrix in double; returns the determinant.
template <int D> __device__ __forceinline__ double inv_sym(const double (&a)[D][D], double (&r)[D][D]) {
    if constexpr (D == 1) {
        r[0][0] = 1.0 / a[0][0];
        return a[0][0];
    } else if constexpr (D == 2) {
        double det = a[0][0] * a[1][1] - a[0][1] * a[1][0];
        double id = 1.0 / det;
        r[0][0] = a[1][1] * id; r[1][1] = a[0][0] * id;
        r[0][1] = -a[0][1] * id; r[1][0] = -a[1][0] * id;
        return det;
    } else {
        double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
        double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
        double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
        double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
        double id = 1.0 / det;
        r[0][0] = c00 * id;
        r[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id;
        r[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
        r[1][0] = c01 * id;
        r[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
        r[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
        r[2][0] = c02 * id;
        r[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id;
        r[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
        return det;
    }
}

// CRK moments (FP32 sums, W_ij = W(r_ij, H_j)), FP64 solve for A, B, gradA, gradB
// (Frontiere, Raskin & Owen 2017: linear reproducing conditions) and the CRK density
// sum_j m_j W^R_ij.  A singular second moment (fewer than D+1 effective neighbours)
// falls back to the zeroth-order correction.
template <int D> struct CrkAcc {
    float m0, s0, m1[D], s1[D], dm0[D], m2[D][D], dm1[D][D], dm2[D][D][D];
};
// The ideal-gas EOS of one particle (modules/eos/idealGas.py:16-36), as k_eos computes it:
// fused into the epilogue of the pass that produces the density.
struct EosOut { const float* u; float* A; float* P; float* c; float gamma; };
__device__ __forceinline__ void eos_ideal_gas_at(int i, const EosOut& eo, float r) {
    const float gamma = eo.gamma, ui = eo.u[i];
    if (eo.c) eo.c[i] = sqrtf(fabsf(ui) * gamma * (gamma - 1.f));
    if (eo.P) eo.P[i] = (gamma - 1.f) * r * ui;
    if (eo.A) eo.A[i] = ui * (gamma - 1.f) * powf(r, 1.f - gamma);
}

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_crk_factors(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
              const float* __restrict__ V, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
              const int32_t* __restrict__ list, float* __restrict__ Aout, float* __restrict__ Bout,
              float* __restrict__ gAout, float* __restrict__ gBout, float* __restrict__ rho_out, EosOut eo) {
    pdl_entry();
    Grp<G> g(n);
    CrkAcc<D> a;
    {
        float* f = reinterpret_cast<float*>(&a);
        #pragma unroll
        for (int q = 0; q < (int)(sizeof(CrkAcc<D>) / 4); ++q) f[q] = 0.f;
    }
    if (g.valid) {
        Vec<D> xi = load_vec<D>(x, g.i);
        int b = offs[g.i], e = b + cnt[g.i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            const float Hj = __ldg(H + j), Vj = __ldg(V + j), mj = __ldg(m + j);   // gathers issued together
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, r, 1.f / Hj, W, gW);
            if (W == 0.f) continue;
            float VW = Vj * W, mW = mj * W;
            a.m0 += VW;
            a.s0 += mW;
            #pragma unroll
            for (int u = 0; u < D; ++u) {
                a.m1[u] += VW * xij.v[u];
                a.s1[u] += mW * xij.v[u];
                a.dm0[u] += Vj * gW.v[u];
                #pragma unroll
                for (int c = 0; c < D; ++c) {
                    a.m2[u][c] += VW * xij.v[u] * xij.v[c];
                    a.dm1[u][c] += Vj * (xij.v[u] * gW.v[c] + (u == c ? W : 0.f));
                }
            }
            #pragma unroll
            for (int u = 0; u < D; ++u)
                #pragma unroll
                for (int c = u; c < D; ++c)
                    #pragma unroll
                    for (int w = 0; w < D; ++w)
                        a.dm2[u][c][w] += Vj * (xij.v[u] * xij.v[c] * gW.v[w] + ((u == w ? xij.v[c] : 0.f) + (c == w ? xij.v[u] : 0.f)) * W);
        }
    }
    {
        float* f = reinterpret_cast<float*>(&a);
        #pragma unroll
        for (int q = 0; q < (int)(sizeof(CrkAcc<D>) / 4); ++q) f[q] = gsum<G>(f[q]);
    }
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    double M2[D][D], Mi[D][D], tr = 0.0;
    #pragma unroll
    for (int u = 0; u < D; ++u) {
        #pragma unroll
        for (int c = 0; c < D; ++c) M2[u][c] = (double)(u <= c ? a.m2[u][c] : a.m2[c][u]);
        tr += M2[u][u];
    }
    double det = inv_sym<D>(M2, Mi);
    double sc = tr / D, sD = sc;
    #pragma unroll
    for (int u = 1; u < D; ++u) sD *= sc;
    bool ok = isfinite(det) && fabs(det) > 1e-10 * fabs(sD) && a.m0 > 0.f;
    double A, Bv[D], gA[D], gB[D][D];
    if (ok) {
        double mb = a.m0;
        #pragma unroll
        for (int u = 0; u < D; ++u) {
            double t = 0.0;
            #pragma unroll
            for (int c = 0; c < D; ++c) t -= Mi[u][c] * (double)a.m1[c];
            Bv[u] = t;
        }
        #pragma unroll
        for (int u = 0; u < D; ++u) mb += (double)a.m1[u] * Bv[u];
        A = 1.0 / mb;
        #pragma unroll
        for (int w = 0; w < D; ++w) {
            double rhs[D];
            #pragma unroll
            for (int u = 0; u < D; ++u) {
                double t = (double)a.dm1[u][w];
                #pragma unroll
                for (int c = 0; c < D; ++c) t += (double)(u <= c ? a.dm2[u][c][w] : a.dm2[c][u][w]) * Bv[c];
                rhs[u] = t;
            }
            #pragma unroll
            for (int u = 0; u < D; ++u) {
                double t = 0.0;
                #pragma unroll
                for (int c = 0; c < D; ++c) t -= Mi[u][c] * rhs[c];
                gB[u][w] = t;
            }
        }
        #pragma unroll
        for (int w = 0; w < D; ++w) {
            double t = (double)a.dm0[w];
            #pragma unroll
            for (int u = 0; u < D; ++u) t += (double)a.dm1[u][w] * Bv[u] + (double)a.m1[u] * gB[u][w];
            gA[w] = -A * A * t;
        }
    } else {
        double m0d = (double)a.m0;
        A = 1.0 / m0d;
        #pragma unroll
        for (int u = 0; u < D; ++u) {
            Bv[u] = 0.0;
            gA[u] = -(double)a.dm0[u] / (m0d * m0d);
            #pragma unroll
            for (int c = 0; c < D; ++c) gB[u][c] = 0.0;
        }
    }
    double rho = (double)a.s0;
    #pragma unroll
    for (int u = 0; u < D; ++u) rho += Bv[u] * (double)a.s1[u];
    rho *= A;
    Aout[i] = (float)A;
    #pragma unroll
    for (int u = 0; u < D; ++u) {
        Bout[(size_t)i * D + u] = (float)Bv[u];
        gAout[(size_t)i * D + u] = (float)gA[u];
        #pragma unroll
        for (int c = 0; c < D; ++c) gBout[(size_t)i * D * D + u * D + c] = (float)gB[u][c];
    }
    if (rho_out) rho_out[i] = (float)rho;
    if (eo.u) eos_ideal_gas_at(i, eo, (float)rho);
}

// ---------------------------------------------------------------- EOS (modules/eos/idealGas.py:16-36)
__global__ void k_eos(int n, float gamma, const float* __restrict__ u, const float* __restrict__ rho,
                      float* __restrict__ Aout, float* __restrict__ Pout, float* __restrict__ cout) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ui = u[i], r = rho[i];
    if (cout) cout[i] = sqrtf(fabsf(ui) * gamma * (gamma - 1.f));
    if (Pout) Pout[i] = (gamma - 1.f) * r * ui;
    if (Aout) Aout[i] = ui * (gamma - 1.f) * powf(r, 1.f - gamma);
}

// ---------------------------------------------------------------- CRK velocity gradient (+ Cullen div, v_sig)
// schemes/crkSPH.py:158-172 (difference form, scatter support, CRK kernel, .mT),
// CullenDehnen2010.py:246-257 (super-symmetric divergence), wp_vsig.py:55-90.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_grad_v(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
         const float* __restrict__ rho, const float* __restrict__ V, const float* __restrict__ A, const float* __restrict__ B,
         const float* __restrict__ gA, const float* __restrict__ gB, const float* __restrict__ v, const float* __restrict__ c,
         const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
         float* __restrict__ DvDx, float* __restrict__ drhodt, float* __restrict__ div_out, float* __restrict__ vsig_out) {
    pdl_entry();
    Grp<G> g(n);
    const bool want_div = div_out != nullptr, want_vs = vsig_out != nullptr;
    Mat<D> Gm = mzero<D>();
    float div = 0.f, vsig = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i), vi = load_vec<D>(v, i);
        float Hi = H[i], Ai = A[i];
        Vec<D> Bi = load_vec<D>(B, i), gAi = load_vec<D>(gA, i);
        Mat<D> gBi = load_mat<D>(gB, i);
        float ci = want_vs ? c[i] : 0.f;
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            const float Hj = __ldg(H + j), Vj = __ldg(V + j);   // gathers issued together
            const float mj = want_div ? __ldg(m + j) : 0.f, rhoj = want_div ? __ldg(rho + j) : 1.f;
            const Vec<D> vj = load_vec<D>(v, j);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, r, 1.f / Hj, W, gW);
            if (W != 0.f) {
                Vec<D> gR = crk_grad<D>(xij, W, gW, Ai, Bi, gAi, gBi);
                #pragma unroll
                for (int a = 0; a < D; ++a) {
                    float dv = Vj * (vj.v[a] - vi.v[a]);
                    #pragma unroll
                    for (int w = 0; w < D; ++w) Gm.m[a][w] += dv * gR.v[w];
                }
            }
            float Hs = wmax(Hi, Hj);
            if (want_div && r < Hs) {
                float W2; Vec<D> g2;
                kWG_inv<KF, D>(xij, r, 1.f / Hs, W2, g2);
                float vol = mj / rhoj;
                float s = 0.f;
                #pragma unroll
                for (int a = 0; a < D; ++a) s += (vj.v[a] - vi.v[a]) * g2.v[a];
                div += vol * s;
            }
            if (want_vs && r < P.verlet_scale * Hs) {
                float mu = 0.f;
                #pragma unroll
                for (int a = 0; a < D; ++a) mu += (vi.v[a] - vj.v[a]) * xij.v[a];
                mu = mu / (r + 1e-14f * Hi);
                float vsv = 0.5f * (ci + __ldg(c + j)) - mu;
                if (mu > 0.f) vsv = 0.f;
                vsig = wmax(vsig, vsv);
            }
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int w = 0; w < D; ++w) Gm.m[a][w] = gsum<G>(Gm.m[a][w]);
    if (want_div) div = gsum<G>(div);
    if (want_vs) vsig = gmaxw<G>(vsig);
    if (!g.valid || g.lane != 0) return;
    store_mat<D>(DvDx, g.i, Gm);
    if (drhodt) {
        float tr = Gm.m[0][0];
        #pragma unroll
        for (int a = 1; a < D; ++a) tr += Gm.m[a][a];
        drhodt[g.i] = -tr * rho[g.i];
    }
    if (want_div) div_out[g.i] = div;
    if (want_vs) vsig_out[g.i] = fabsf(vsig);
}

// ---------------------------------------------------------------- Cullen-Dehnen switch
// R (CullenDehnen2010.py:121-164, gather interpolation of rho_j sgn(div_j) / rho_j * m_j),
// v_sig over the Verlet set when not supplied (wp_vsig.py:55-90), Xi (:166-191) and the
// alpha / alpha0 update (:281-314).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_cullen(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
         const float* __restrict__ rho, const float* __restrict__ div, const float* __restrict__ div_prev,
         const float* __restrict__ vsig_in, const float* __restrict__ v, const float* __restrict__ c,
         const float* __restrict__ alpha0_prev, const float* __restrict__ dtp,
         const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
         float* __restrict__ alpha_out, float* __restrict__ R_out, float* __restrict__ vsig_out) {
    pdl_entry();
    Grp<G> g(n);
    const bool want_vs = vsig_in == nullptr;
    float s = 0.f, vsig = 0.f;
    float Hi = 1.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        Hi = H[i];
        const float invHi = 1.f / Hi;
        Vec<D> vi = want_vs ? load_vec<D>(v, i) : vzero<D>();
        float ci = want_vs ? c[i] : 0.f;
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            // every gather of the entry issued together, ahead of the tests that select them;
            // in 3D, where about two thirds of a Verlet row lie outside the support, the
            // divergence and the mass are loaded only for the entries inside it (measured:
            // 11.3 against 12.8 ms per step at 128^3; in 2D loading them ahead wins)
            const float dj_ahead = D < 3 ? __ldg(div + j) : 0.f, mj_ahead = D < 3 ? __ldg(m + j) : 0.f;
            const float Hj = want_vs ? __ldg(H + j) : 0.f, cj = want_vs ? __ldg(c + j) : 0.f;
            const Vec<D> vj = want_vs ? load_vec<D>(v, j) : vzero<D>();
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W = kW_inv<KF, D>(r, invHi);   // gather support
            if (W != 0.f) {
                const float dj = D < 3 ? dj_ahead : __ldg(div + j), mj = D < 3 ? mj_ahead : __ldg(m + j);
                float sg = dj > 0.f ? 1.f : (dj < 0.f ? -1.f : 0.f);
                s += mj * sg * W;
            }
            if (want_vs) {
                float Hs = wmax(Hi, Hj);
                if (r < P.verlet_scale * Hs) {
                    float mu = 0.f;
                    #pragma unroll
                    for (int a = 0; a < D; ++a) mu += (vi.v[a] - vj.v[a]) * xij.v[a];
                    mu = mu / (r + 1e-14f * Hi);
                    float vsv = 0.5f * (ci + cj) - mu;
                    if (mu > 0.f) vsv = 0.f;
                    vsig = wmax(vsig, vsv);
                }
            }
        }
    }
    s = gsum<G>(s);
    if (want_vs) vsig = gmaxw<G>(vsig);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    float vs = want_vs ? fabsf(vsig) : vsig_in[i];
    if (want_vs && vsig_out) vsig_out[i] = vs;
    float rhoi = rho[i];
    float R = 1.f / rhoi * s;
    float dv = div[i];
    float dt = *dtp;
    float omr = 1.f - R;
    float omr2 = omr * omr;
    float nom = P.beta_xi * (omr2 * omr2) * dv;
    float Xi = P.limit_xi ? (nom * nom + 1e-14f * Hi) / (nom * nom + 0.f + 1e-14f * Hi)
                          : (nom * nom) / (nom * nom + 0.f + 1e-14f * Hi);
    float ddiv = (dv - div_prev[i]) / dt;
    float Ai = Xi * fmaxf(-ddiv, 0.f);
    float scaling = Hi * Hi * Ai / (vs * vs + Hi * Hi * Ai + 1e-14f * Hi);
    float alphas = fminf(fmaxf(P.alpha_max * scaling, P.alpha_min), P.alpha_max);
    float a0 = alpha0_prev[i];
    float tau = Hi * (1.f / P.kxi) / (2.f * 0.05f * vs);
    float adot = (alphas - a0) / tau;
    a0 = alphas > a0 ? alphas : a0;
    a0 = alphas < a0 ? a0 + adot * dt : a0;
    alpha_out[i] = fminf(fmaxf(a0, P.alpha_min), P.alpha_max);
    if (R_out) R_out[i] = R;
}

// ---------------------------------------------------------------- Cullen-Hopkins switch
// modules/shockCapturing/CullenHopkins.py:7-45 (computeHopkinsTerms): the gather difference
// gradient V_i = sum_j m_j/rho_j (v_j - v_i) (x) grad W(r_ij, H_i) (computeShearTensor,
// common.py:41-85), its trace (the divergence) and |S|^2 = tr(S S^T) of the traceless
// symmetric part S.  With correctVelocityGradient the same pass accumulates the moment
// matrix M_i = -sum_j m_j x_ij (x) grad W(r_ij, H_i) (common.py:10-25, wp_computeM.py:55-86)
// and the gradient becomes pinv(M_i) V_i (common.py:76-78).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_hopkins_grad(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
               const float* __restrict__ rho, const float* __restrict__ v,
               const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
               float* __restrict__ div_out, float* __restrict__ shear2_out) {
    pdl_entry();
    Grp<G> g(n);
    Mat<D> Gm = mzero<D>(), Mm = mzero<D>();
    const bool corr = P.correct_grad_v != 0;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i), vi = load_vec<D>(v, i);
        const float invHi = 1.f / H[i];
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, r, invHi, W, gW);
            if (W == 0.f) continue;
            const float mj = __ldg(m + j);
            const float Vj = mj / __ldg(rho + j);
            Vec<D> vj = load_vec<D>(v, j);
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                const float dv = Vj * (vj.v[a] - vi.v[a]);
                #pragma unroll
                for (int w = 0; w < D; ++w) Gm.m[a][w] += dv * gW.v[w];
            }
            if (corr) {
                #pragma unroll
                for (int a = 0; a < D; ++a)
                    #pragma unroll
                    for (int w = 0; w < D; ++w) Mm.m[a][w] -= mj * xij.v[a] * gW.v[w];
            }
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int w = 0; w < D; ++w) Gm.m[a][w] = gsum<G>(Gm.m[a][w]);
    if (corr) {
        #pragma unroll
        for (int a = 0; a < D; ++a)
            #pragma unroll
            for (int w = 0; w < D; ++w) Mm.m[a][w] = gsum<G>(Mm.m[a][w]);
    }
    if (!g.valid || g.lane != 0) return;
    if (corr) {
        double Md[D][D], Pd[D][D];
        #pragma unroll
        for (int a = 0; a < D; ++a)
            #pragma unroll
            for (int w = 0; w < D; ++w) Md[a][w] = (double)Mm.m[a][w];
        pinv_jacobi<D>(Md, Pd, (double)D * (double)FLT_EPSILON);
        Mat<D> C;
        #pragma unroll
        for (int a = 0; a < D; ++a)
            #pragma unroll
            for (int w = 0; w < D; ++w) {
                double acc = 0.0;
                #pragma unroll
                for (int c = 0; c < D; ++c) acc += Pd[a][c] * (double)Gm.m[c][w];
                C.m[a][w] = (float)acc;
            }
        Gm = C;
    }
    float tr = Gm.m[0][0];
    #pragma unroll
    for (int a = 1; a < D; ++a) tr += Gm.m[a][a];
    float s2 = 0.f;
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int w = 0; w < D; ++w) {
            float sv = (Gm.m[a][w] + Gm.m[w][a]) / 2.f - (a == w ? tr / (float)D : 0.f);
            s2 += sv * sv;
        }
    div_out[g.i] = tr;
    shear2_out[g.i] = s2;
}

// R (CullenDehnen2010.py:121-164, gather), Xi with the shear term (:166-191) and
// alpha = max(Xi alpha0, alpha_min) (CullenHopkins.py:25).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_hopkins_alpha(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                const float* __restrict__ rho, const float* __restrict__ div, const float* __restrict__ shear2,
                const float* __restrict__ alpha0, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                const int32_t* __restrict__ list, float* __restrict__ alpha_out, float* __restrict__ R_out) {
    pdl_entry();
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        const float invHi = 1.f / H[i];
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float W = kW_inv<KF, D>(safe_sqrt(dot<D>(xij, xij)), invHi);
            if (W == 0.f) continue;
            float dj = __ldg(div + j);
            float sg = dj > 0.f ? 1.f : (dj < 0.f ? -1.f : 0.f);
            s += __ldg(m + j) * sg * W;
        }
    }
    s = gsum<G>(s);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float Hi = H[i];
    const float R = 1.f / rho[i] * s;
    const float omr = 1.f - R, omr2 = omr * omr;
    const float nom = P.beta_xi * (omr2 * omr2) * div[i];
    const float Xi = P.limit_xi ? (nom * nom + 1e-14f * Hi) / (nom * nom + shear2[i] + 1e-14f * Hi)
                                : (nom * nom) / (nom * nom + shear2[i] + 1e-14f * Hi);
    alpha_out[i] = fmaxf(Xi * alpha0[i], P.alpha_min);
    if (R_out) R_out[i] = R;
}

// computeHopkinsUpdate (CullenHopkins.py:48-149): v_sig over the Verlet rows
// (wp_vsig.py:55-90), d(div)/dt = (div - div_prev) / dt, the local alpha_tmp and the
// relaxation of alpha0 towards it.
template <int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_hopkins_update(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ v,
                 const float* __restrict__ c, const float* __restrict__ div, const float* __restrict__ div_prev,
                 const float* __restrict__ alpha0, const float* __restrict__ dtp,
                 const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
                 float* __restrict__ alpha0_out, float* __restrict__ vsig_out) {
    pdl_entry();
    Grp<G> g(n);
    float vsig = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i), vi = load_vec<D>(v, i);
        const float Hi = H[i], ci = c[i];
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r = safe_sqrt(dot<D>(xij, xij));
            if (!(r < P.verlet_scale * wmax(Hi, __ldg(H + j)))) continue;
            Vec<D> vj = load_vec<D>(v, j);
            float mu = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) mu += (vi.v[a] - vj.v[a]) * xij.v[a];
            mu = mu / (r + 1e-14f * Hi);
            float vsv = 0.5f * (ci + __ldg(c + j)) - mu;
            if (mu > 0.f) vsv = 0.f;
            vsig = wmax(vsig, vsv);
        }
    }
    vsig = gmaxw<G>(vsig);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float vs = fabsf(vsig);
    const float dt = *dtp;
    const float Hi = H[i], ci = c[i], dv = div[i];
    const float f_kern = 1.f / P.kxi;
    const float ddiv = (dv - div_prev[i]) / dt;
    const float ad = fabsf(ddiv);
    const float fh = f_kern * Hi;
    float at = P.alpha_max * ad / (ad + P.beta_c * (ci * ci) / (fh * fh) + 1e-14f);
    if (ddiv > 0.f || dv > 0.f) at = 0.f;
    const float a0 = alpha0[i];
    const float next = at + (a0 - at) * expf(-P.beta_d * dt * vs / (2.f * f_kern * Hi));
    alpha0_out[i] = at >= a0 ? at : next;
    if (vsig_out) vsig_out[i] = vs;
}

// Balsara switch from the velocity gradient (schemes/crkSPH.py:132-133 comment).
template <int D>
__global__ void k_balsara(int n, const float* __restrict__ DvDx, const float* __restrict__ c, float* __restrict__ alpha) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Mat<D> Gm = load_mat<D>(DvDx, i);
    float dv = Gm.m[0][0];
    for (int a = 1; a < D; ++a) dv += Gm.m[a][a];
    float curl2 = 0.f;
    if constexpr (D == 2) { float w = Gm.m[1][0] - Gm.m[0][1]; curl2 = w * w; }
    if constexpr (D == 3) {
        float w0 = Gm.m[2][1] - Gm.m[1][2], w1 = Gm.m[0][2] - Gm.m[2][0], w2 = Gm.m[1][0] - Gm.m[0][1];
        curl2 = w0 * w0 + w1 * w1 + w2 * w2;
    }
    float ad = fabsf(dv);
    float bal = ad / (ad + sqrtf(curl2) + 1e-4f * c[i]);
    alpha[i] = fminf(fmaxf(bal, 0.f), 1.f);
}

// ---------------------------------------------------------------- CRK accel + dudt
// modules/crk/limiter.py:10-16
__device__ __forceinline__ float limiter_vl(float x) {
    if (x <= 0.f) return 0.f;
    float vL = __fdividef(2.f, 1.f + x);
    return x * vL * vL;
}
__device__ __forceinline__ float sgn_pos(float x) { return x >= 0.f ? 1.f : -1.f; }

// modules/crk/limiter.py:27-86 (quadratic-form Van Leer) with g = (G h).h, h = x_ij / 2,
// from the products G_i x_ij and G_j x_ij the pass needs anyway: halving is exact in
// floating point, so (G h).h = (G x_ij).x_ij / 4 (outside the subnormal range).
template <int D>
__device__ __forceinline__ float van_leer(const Vec<D>& xij_, const Vec<D>& Gix, const Vec<D>& Gjx) {
    float gi = 0.25f * dot<D>(Gix, xij_);
    float gj = 0.25f * dot<D>(Gjx, xij_);
    float ri = __fdividef(gi, sgn_pos(gj) * fabsf(gj));
    float rj = __fdividef(gj, sgn_pos(gi) * fabsf(gi));
    if (ri != ri) ri = 1.f;
    if (rj != rj) rj = 1.f;
    return limiter_vl(wmin(ri, rj));
}

// Zero pairwise outputs of the entries [offs + cnt, offs + vcnt) of a row: the Verlet
// entries after the interacting prefix, which carry no interaction (contiguous stores).
template <int D, int G>
__device__ __forceinline__ void zero_row_tail(int lane, int e, int te, float* __restrict__ ap, float* __restrict__ av) {
    for (int q = e + lane; q < te; q += G) {
        if (ap) store_vec<D>(ap, q, vzero<D>());
        if (av) store_vec<D>(av, q, vzero<D>());
    }
}

// Packed per-particle record of the CRK accel pass: every field a pair reads from
// particle j (and the pass reads from particle i) in one block of R floats, R a multiple
// of 4, so a pair's neighbour gather is R/4 128-bit loads from adjacent sectors instead
// of 2D^2+4D+6 scalar loads from as many arrays (D = 2: 6 loads and 3 sectors instead of
// 22 loads and 22 sectors).  The fields are in the order the pair body first uses them,
// and the body loads them in three groups of 16-byte granules: position and support
// (before the distance test), velocity, gradient, sound speed and pressure (the limiter
// and Q), and the rest (the corrected gradient of W_ji), which keeps fewer of them live.
template <int D> struct CrkRec {
    static constexpr int X = 0, H = D, RHO = D + 1, V = D + 2, G = 2 * D + 2, C = 2 * D + 2 + D * D, P = C + 1,
                         VOL = C + 2, A = C + 3, B = C + 4, GA = B + D, GB = GA + D, END = GB + D * D,
                         R = (END + 3) / 4 * 4;
    static constexpr int K1 = (H + 1 + 3) / 4;      // granules of the first group
    static constexpr int K2 = (P + 1 + 3) / 4;      // ... of the first two groups
    static constexpr int K3 = R / 4;
};
template <int D, int K0, int K1>
__device__ __forceinline__ void rec_granules(const float4* __restrict__ src, float (&r)[CrkRec<D>::R]) {
    #pragma unroll
    for (int k = K0; k < K1; ++k) {
        float4 t = __ldg(src + k);
        r[4 * k] = t.x; r[4 * k + 1] = t.y; r[4 * k + 2] = t.z; r[4 * k + 3] = t.w;
    }
}

template <int D>
__global__ void k_crk_pack(int n, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ rho,
                           const float* __restrict__ V, const float* __restrict__ A, const float* __restrict__ B,
                           const float* __restrict__ gA, const float* __restrict__ gB, const float* __restrict__ v,
                           const float* __restrict__ c, const float* __restrict__ Pr, const float* __restrict__ DvDx,
                           float* __restrict__ rec) {
    pdl_entry();
    using L = CrkRec<D>;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r[L::R];
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        r[L::X + a] = x[(size_t)i * D + a];
        r[L::V + a] = v[(size_t)i * D + a];
        r[L::B + a] = B[(size_t)i * D + a];
        r[L::GA + a] = gA[(size_t)i * D + a];
    }
    #pragma unroll
    for (int a = 0; a < D * D; ++a) {
        r[L::GB + a] = gB[(size_t)i * D * D + a];
        r[L::G + a] = DvDx[(size_t)i * D * D + a];
    }
    r[L::H] = H[i]; r[L::RHO] = rho[i]; r[L::VOL] = V[i]; r[L::C] = c[i]; r[L::P] = Pr[i]; r[L::A] = A[i];
    #pragma unroll
    for (int a = L::END; a < L::R; ++a) r[a] = 0.f;
    float4* dst = reinterpret_cast<float4*>(rec + (size_t)i * L::R);
    #pragma unroll
    for (int k = 0; k < L::R / 4; ++k) dst[k] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
}

// The fields of one particle as the accel pass uses them.
template <int D> struct CrkPart {
    Vec<D> x, v, B, gA;
    Mat<D> gB, G;
    float H, rho, V, c, P, A;
};
// Group 1: position and support; group 2: velocity, velocity gradient, density, sound
// speed, pressure; group 3: volume and the CRK correction fields.
template <int D> __device__ __forceinline__ void crk_unpack1(const float (&r)[CrkRec<D>::R], CrkPart<D>& o) {
    using L = CrkRec<D>;
    #pragma unroll
    for (int a = 0; a < D; ++a) o.x.v[a] = r[L::X + a];
    o.H = r[L::H];
}
template <int D> __device__ __forceinline__ void crk_unpack2(const float (&r)[CrkRec<D>::R], CrkPart<D>& o) {
    using L = CrkRec<D>;
    #pragma unroll
    for (int a = 0; a < D; ++a) o.v.v[a] = r[L::V + a];
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) o.G.m[a][b] = r[L::G + a * D + b];
    o.rho = r[L::RHO]; o.c = r[L::C]; o.P = r[L::P];
}
template <int D> __device__ __forceinline__ void crk_unpack3(const float (&r)[CrkRec<D>::R], CrkPart<D>& o) {
    using L = CrkRec<D>;
    #pragma unroll
    for (int a = 0; a < D; ++a) { o.B.v[a] = r[L::B + a]; o.gA.v[a] = r[L::GA + a]; }
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) o.gB.m[a][b] = r[L::GB + a * D + b];
    o.V = r[L::VOL]; o.A = r[L::A];
}

// modules/crk/accel.py:65-250 and modules/crk/dudt.py:62-229 in one pass.  The pair
// body's quotients (Van Leer ratios, 1/H_j, the mu_ij denominators) use the fast FP32
// divide (about 2 ulp): about a tenth of the pass's time, well inside the pass's parity
// tolerance against the oracle's IEEE quotients.  The
// unused computePi_actual calls of the reference (accel.py:143-168, dudt.py:128-153)
// have no effect on the outputs and are not evaluated.  dE/dt = m v.dv/dt + m du/dt
// (schemes/crkSPH.py:330) is written per particle.  Walking the interacting prefix of
// each Verlet row (cnt = interacting counts) with vcnt = the Verlet counts, the
// ap_ij / av_ij entries of the rest of the row are written as zeros.
#ifndef CRK_REC_BLOCKS
#define CRK_REC_BLOCKS 7
#endif
template <int KF, int D, int G, bool REC>
__global__ void __launch_bounds__(PAIR_BLOCK, (D == 3 ? 5 : (REC ? CRK_REC_BLOCKS : 8)))
k_crk_accel_dudt(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                 const float* __restrict__ rho, const float* __restrict__ V, const float* __restrict__ A,
                 const float* __restrict__ B, const float* __restrict__ gA, const float* __restrict__ gB,
                 const float* __restrict__ v, const float* __restrict__ c, const float* __restrict__ Pr,
                 const float* __restrict__ DvDx, const float* __restrict__ rec, const int32_t* __restrict__ offs,
                 const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, const int32_t* __restrict__ vcnt,
                 float* __restrict__ dvdt, float* __restrict__ dudt, float* __restrict__ dEdt, float* __restrict__ ap,
                 float* __restrict__ av) {
    pdl_entry();
    Grp<G> g(n);
    const bool comp = P.kahan != 0;
    KSum acc[D], du;
    #pragma unroll
    for (int a = 0; a < D; ++a) acc[a].init();
    du.init();
    if (g.valid) {
        const int i = g.i;
        CrkPart<D> pi;
        if constexpr (REC) {
            float r[CrkRec<D>::R];
            rec_granules<D, 0, CrkRec<D>::K3>(reinterpret_cast<const float4*>(rec + (size_t)i * CrkRec<D>::R), r);
            crk_unpack1<D>(r, pi); crk_unpack2<D>(r, pi); crk_unpack3<D>(r, pi);
        } else {
            pi.x = load_vec<D>(x, i); pi.v = load_vec<D>(v, i); pi.B = load_vec<D>(B, i); pi.gA = load_vec<D>(gA, i);
            pi.gB = load_mat<D>(gB, i); pi.G = load_mat<D>(DvDx, i);
            pi.H = H[i]; pi.rho = rho[i]; pi.V = V[i]; pi.c = c[i]; pi.P = Pr[i]; pi.A = A[i];
        }
        const float Hi = pi.H, rhoi = pi.rho, ci = pi.c, Pi = pi.P;
        const float invHi = 1.f / Hi;
        const float Vi_m = pi.V / m[i];          // V_i / m_i
        const float ks = P.kscale;
        const float inv_smooth_i = ks * invHi;   // 1 / (H_i / ks)
        const float sm_i = Hi / ks;
        const float eps_i = 1.0e-7f * sm_i * sm_i;
        int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            CrkPart<D> pj;
            float rj[CrkRec<D>::R];
            const float4* sj = REC ? reinterpret_cast<const float4*>(rec + (size_t)j * CrkRec<D>::R) : nullptr;
            if constexpr (REC) {
                // the first two groups issued together (walked rows are interacting prefixes, so
                // the range test below almost never discards the second)
                rec_granules<D, 0, CrkRec<D>::K2>(sj, rj);
                crk_unpack1<D>(rj, pj);
            }
            else { pj.x = load_vec<D>(x, j); pj.H = __ldg(H + j); }
            Vec<D> xij = dist_vec<D>(pi.x, pj.x, P.dom);
            float r2 = dot<D>(xij, xij);
            const float Hj = pj.H;
            float Hm = wmax(Hi, Hj);
            if (!(r2 < Hm * Hm)) {
                if (ap) store_vec<D>(ap, k, vzero<D>());
                if (av) store_vec<D>(av, k, vzero<D>());
                continue;
            }
            if constexpr (REC) {
                crk_unpack2<D>(rj, pj);
            } else {
                pj.v = load_vec<D>(v, j);
                pj.rho = __ldg(rho + j); pj.c = __ldg(c + j); pj.P = __ldg(Pr + j);
                pj.G = load_mat<D>(DvDx, j);
            }
            float r = safe_sqrt(r2);
            const float invHj = __fdividef(1.f, Hj);
            const float rhoj = pj.rho, cj = pj.c, Pj = pj.P;
            // CRK limiter (limiter.py:89-128), eta measured in supports
            float factor = 1.f;
            if (P.enable_crk_limiter) {
                float eta = r * wmin(invHi, invHj);
                if (eta < P.eta_crit) { float t = (eta - P.eta_crit) / P.eta_fold; factor = expf(-(t * t)); }
            }
            Vec<D> Gix = matvec<D>(pi.G, xij), Gjx = matvec<D>(pj.G, xij);
            float phi = 0.f;
            if (P.enable_vanleer) phi = van_leer<D>(xij, Gix, Gjx) * factor;
            if (P.force_vl_off) phi = 0.f;
            if (P.force_vl_on) phi = 1.f;
            phi = wmax(wmin(phi, 1.f), 0.f);
            float hp = 0.5f * phi;
            // v_dot_i - v_dot_j (accel.py:137-141; dudt.py:122-126 uses gradV_j . (-x_ij))
            Vec<D> da, dd;
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                float vdi = pi.v.v[a] - hp * Gix.v[a];
                da.v[a] = vdi - (pj.v.v[a] + hp * Gjx.v[a]);
                dd.v[a] = vdi - (pj.v.v[a] - hp * Gjx.v[a]);
            }
            // corrected gradients (accel.py:170-187, dudt.py:155-170)
            float Wi; Vec<D> gWi;
            kWG_inv<KF, D>(xij, r, invHj, Wi, gWi);
            Vec<D> gradw_i = crk_grad<D>(xij, Wi, gWi, pi.A, pi.B, pi.gA, pi.gB);
            if constexpr (REC) {
                rec_granules<D, CrkRec<D>::K2, CrkRec<D>::K3>(sj, rj); crk_unpack3<D>(rj, pj);
            } else {
                pj.V = __ldg(V + j);
                pj.A = __ldg(A + j); pj.B = load_vec<D>(B, j); pj.gA = load_vec<D>(gA, j); pj.gB = load_mat<D>(gB, j);
            }
            Vec<D> xji;
            #pragma unroll
            for (int a = 0; a < D; ++a) xji.v[a] = -xij.v[a];
            float Wj; Vec<D> gWj;
            kWG_inv<KF, D>(xji, r, invHi, Wj, gWj);
            Vec<D> gradw_j = crk_grad<D>(xji, Wj, gWj, pj.A, pj.B, pj.gA, pj.gB);
            Vec<D> gij;
            #pragma unroll
            for (int a = 0; a < D; ++a) gij.v[a] = 0.5f * (gradw_i.v[a] - gradw_j.v[a]);
            // mu_ij, mu_ji and Q (accel.py:189-206): eta = x_ij / smoothing length
            const float inv_smooth_j = ks * invHj;
            const float sm_j = Hj / ks;
            const float eps_j = 1.0e-7f * sm_j * sm_j;
            float den_i = r2 * (inv_smooth_i * inv_smooth_i) + eps_i;
            float den_j = r2 * (inv_smooth_j * inv_smooth_j) + eps_j;
            float xa = dot<D>(da, xij), xd = dot<D>(dd, xij);
            float idi = __fdividef(inv_smooth_i, den_i), idj = __fdividef(inv_smooth_j, den_j);
            float mia = wmin(0.f, xa * idi), mja = wmin(0.f, xa * idj);
            float mid = wmin(0.f, xd * idi), mjd = wmin(0.f, xd * idj);
            float Qa = rhoi * (-P.C_l * ci * mia + P.C_q * mia * mia) + rhoj * (-P.C_l * cj * mja + P.C_q * mja * mja);
            float Qd = rhoi * (-P.C_l * ci * mid + P.C_q * mid * mid) + rhoj * (-P.C_l * cj * mjd + P.C_q * mjd * mjd);
            // accel.py:228-249 (mu_ij = 1 there)
            const float w = pj.V * Vi_m;   // V_i V_j / m_i
            Vec<D> pt, vt;
            float dotu = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                pt.v[a] = -(Pi + Pj) * gij.v[a] * w;
                vt.v[a] = -Qa * gij.v[a] * w;
                acc[a].add(pt.v[a] + vt.v[a], comp);
                dotu += (pi.v.v[a] - pj.v.v[a]) * gij.v[a];
            }
            if (ap) store_vec<D>(ap, k, pt);
            if (av) store_vec<D>(av, k, vt);
            // dudt.py:208-226
            du.add((Pj + 0.5f * Qd) * dotu * w, comp);
        }
        if (vcnt && (ap || av)) zero_row_tail<D, G>(g.lane, e, b + __ldg(vcnt + i), ap, av);
    }
    float o[D], od;
    #pragma unroll
    for (int a = 0; a < D; ++a) o[a] = gsum<G>(acc[a].s) + gsum<G>(acc[a].c);
    od = gsum<G>(du.s) + gsum<G>(du.c);
    if (!g.valid || g.lane != 0) return;
    Vec<D> ov;
    #pragma unroll
    for (int a = 0; a < D; ++a) ov.v[a] = o[a];
    if (dvdt) store_vec<D>(dvdt, g.i, ov);
    if (dudt) dudt[g.i] = od;
    if (dEdt) {
        const float mi = m[g.i];
        Vec<D> vi;
        if constexpr (REC) {
            #pragma unroll
            for (int a = 0; a < D; ++a) vi.v[a] = __ldg(rec + (size_t)g.i * CrkRec<D>::R + CrkRec<D>::V + a);
        } else {
            vi = load_vec<D>(v, g.i);
        }
        dEdt[g.i] = mi * dot<D>(vi, ov) + mi * od;
    }
}

// ---------------------------------------------------------------- energy partition f_ij (modules/compSPH/balance.py:62-154)
__device__ __forceinline__ float sgn0(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// Per-particle prologue: half-step velocity v + dt/2 dv/dt (schemes/crkSPH.py:341) and
// the CRK entropy P / rho^gamma (balance.py:126-127).
template <int D>
__global__ void k_balance_prep(int n, DevParams P, const float* __restrict__ rho, const float* __restrict__ Pr,
                               const float* __restrict__ v, const float* __restrict__ dvdt, const float* __restrict__ dtp,
                               float* __restrict__ vh, float* __restrict__ sarr) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float hdt = 0.5f * (*dtp);
    Vec<D> vi = load_vec<D>(v, i), ai = load_vec<D>(dvdt, i);
    #pragma unroll
    for (int a = 0; a < D; ++a) vi.v[a] = vi.v[a] + hdt * ai.v[a];
    store_vec<D>(vh, i, vi);
    sarr[i] = Pr[i] / powf(rho[i], P.gamma);
}

template <int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_balance(int n, DevParams P, const float* __restrict__ m, const float* __restrict__ rho, const float* __restrict__ Pr,
          const float* __restrict__ u, const float* __restrict__ vh, const float* __restrict__ sarr, const float* __restrict__ dtp,
          const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
          const int32_t* __restrict__ icnt, const float* __restrict__ ap, const float* __restrict__ av, float* __restrict__ fout) {
    pdl_entry();
    Grp<G> g(n);
    if (!g.valid) return;
    const int i = g.i;
    const float dt = *dtp;
    Vec<D> vi = load_vec<D>(vh, i);
    const float mi = m[i], rhoi = rho[i], Pi = Pr[i], ui = u[i], si = sarr[i];
    const int scheme = P.energy_scheme;
    int b = offs[i], e = b + cnt[i];
    // entries past the interacting prefix carry ap = av = 0, so their dE is 0 (the same
    // value the loads would give) and their pair arrays and half-step velocities are not read
    const int ie = icnt ? b + icnt[i] : e;
    for (int q = b + g.lane; q < e; q += G) {
        int j, k; entry(list, q, j, k);
        const float sj_crk = scheme == SPH_ENERGY_CRK ? __ldg(sarr + j) : 0.f;   // issued with the entry's other gathers
        float dE = 0.f;
        if (q < ie) {
            Vec<D> vj = load_vec<D>(vh, j);
            Vec<D> apk = load_vec<D>(ap, k), avk = load_vec<D>(av, k);
            #pragma unroll
            for (int a = 0; a < D; ++a) dE += (vj.v[a] - vi.v[a]) * (apk.v[a] + avk.v[a]);
        }
        dE = mi * dE * dt;
        float f = 0.5f;
        if (scheme == SPH_ENERGY_CRK) {
            const float sj = sj_crk;
            float smin = wmin(fabsf(si), fabsf(sj)), smax = wmax(fabsf(si), fabsf(sj));
            bool mA = fabsf(si - sj) == 0.f;
            bool mB = (dE >= 0.f && si >= sj) || (dE < 0.f && si < sj);
            bool mC = (dE >= 0.f && si < sj) || (dE < 0.f && si >= sj);
            if (!mA && mB) f = smin / (smin + smax + 1.0e-14f);
            if (!mA && !mB && mC) f = smax / (smin + smax + 1.0e-14f);
            f = wmax(0.f, wmin(1.f, f));
        } else if (scheme == SPH_ENERGY_PDV) {
            float rhoj = __ldg(rho + j), Pj = __ldg(Pr + j);
            f = (Pi / (rhoi * rhoi)) / (Pi / (rhoi * rhoi) + Pj / (rhoj * rhoj));
        } else if (scheme == SPH_ENERGY_DIMINISHING) {
            float uji = __ldg(u + j) - ui, un = fabsf(uji);
            f = 0.5f * (1.f + (uji * sgn0(dE)) / (un + 1.f / (1.f + un)));
        } else if (scheme == SPH_ENERGY_MONOTONIC || scheme == SPH_ENERGY_HYBRID) {
            float mj = __ldg(m + j), uj = __ldg(u + j), uji = uj - ui;
            float Aq = dE / (uji + 1.0e-14f);
            float Bq = Aq >= 0.f ? Aq / mi : Aq / mj;
            float t1 = wmax(0.f, sgn0(Bq));
            float t2 = mi / (dE + 1.0e-14f) * ((dE + mi * ui + mj * uj) / (mi + mj) - ui);
            float fm = fabsf(Bq) <= 1.f ? t1 : t2;
            if (scheme == SPH_ENERGY_MONOTONIC) f = fm;
            else {
                float un = fabsf(uji);
                float fsm = 0.5f * (1.f + (uji * sgn0(dE)) / (un + 1.f / (1.f + un)));
                float chi = fabsf(uji) / (fabsf(ui) + fabsf(uj) + 1.0e-14f);
                f = chi * fm + (1.f - chi) * fsm;
            }
        }
        fout[k] = f;
    }
}

// ---------------------------------------------------------------- CFL dt (modules/timestep/compressible.py:18-61)
__global__ void k_cfl_reduce(int n, float gamma, const float* __restrict__ H, const float* __restrict__ u,
                             float* __restrict__ red /* [0]=min H, [1]=max c */) {
    pdl_entry();
    float hmin = __int_as_float(0x7f800000), cmax = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        hmin = fminf(hmin, H[i]);
        cmax = fmaxf(cmax, sqrtf(fabsf(u[i]) * gamma * (gamma - 1.f)));
    }
    hmin = block_reduce(hmin, __int_as_float(0x7f800000), OpMinF());
    cmax = block_reduce(cmax, 0.f, OpMaxF());
    if (threadIdx.x == 0) {
        atomicMin(reinterpret_cast<int*>(red), __float_as_int(hmin));
        atomicMax(reinterpret_cast<int*>(red + 1), __float_as_int(cmax));
    }
}
__global__ void k_cfl_init(float* red) {
    pdl_entry(); red[0] = __int_as_float(0x7f800000); red[1] = 0.f; }
__global__ void k_cfl_final(DevParams P, const float* __restrict__ red, const float* __restrict__ dt_prev, float* __restrict__ dt_out) {
    pdl_entry();
    // min_i cfl*h/(c_i*xi) is attained at max_i c_i (the map c -> cfl*h/(c*xi) is monotone)
    float dt = P.cfl * red[0] / (red[1] * P.kxi);
    dt = fminf(fmaxf(dt, P.min_dt), P.max_dt);
    if (dt_prev) {
        float prev = *dt_prev;
        if (dt > prev) dt = fminf(dt, P.dt_growth * prev);
    }
    *dt_out = dt;
}

// ---------------------------------------------------------------- RK stage combination
struct KPtrs { const float* k[8]; float w[8]; };
__global__ void k_rk_combine(int64_t count, const float* __restrict__ y0, int nk, KPtrs K, const float* __restrict__ dtp,
                             int wrap_dim, DomainF dom, float* __restrict__ y) {
    pdl_entry();
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    float dt = *dtp;
    // explicitly rounded (no FMA) so the CPU oracle reproduces the stage states bit for bit
    float s = 0.f;
    for (int q = 0; q < nk; ++q) s = __fadd_rn(s, __fmul_rn(K.w[q], K.k[q][idx]));
    float val = __fadd_rn(y0[idx], __fmul_rn(dt, s));
    if (wrap_dim > 0) {
        int a = (int)(idx % wrap_dim);
        if (dom.periodic[a]) {
            if (val >= dom.max[a]) val = __fsub_rn(val, dom.L[a]);
            else if (val < dom.min[a]) val = __fadd_rn(val, dom.L[a]);
        }
    }
    y[idx] = val;
}

// Several fields combined in one launch (the integrator's positions, velocities and
// energies of one stage): the same arithmetic as k_rk_combine per element.
constexpr int RKF_MAX = 4;
struct FieldPtrs {
    const float* y0[RKF_MAX];
    float* y[RKF_MAX];
    const float* k[RKF_MAX][8];
    int64_t end[RKF_MAX];        // cumulative element counts
    int wrap[RKF_MAX];
    float w[8];
};
__global__ void k_rk_combine_fields(int nf, int nk, FieldPtrs F, const float* __restrict__ dtp, DomainF dom) {
    pdl_entry();
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= F.end[nf - 1]) return;
    int f = 0;
    #pragma unroll
    for (int q = 0; q < RKF_MAX - 1; ++q) f += (q < nf - 1 && g >= F.end[q]) ? 1 : 0;
    const int64_t idx = g - (f > 0 ? F.end[f - 1] : 0);
    const float dt = *dtp;
    float s = 0.f;
    for (int q = 0; q < nk; ++q) s = __fadd_rn(s, __fmul_rn(F.w[q], F.k[f][q][idx]));
    float val = __fadd_rn(F.y0[f][idx], __fmul_rn(dt, s));
    const int wd = F.wrap[f];
    if (wd > 0) {
        int a = (int)(idx % wd);
        if (dom.periodic[a]) {
            if (val >= dom.max[a]) val = __fsub_rn(val, dom.L[a]);
            else if (val < dom.min[a]) val = __fadd_rn(val, dom.L[a]);
        }
    }
    F.y[f][idx] = val;
}

// ---------------------------------------------------------------- compatible energy
// modules/compSPH/multistep.py:52-94 and systems/compSPH.py:100-111
struct StagePtrs {
    const float* dvdt[8];
    const int32_t* offs[8];
    const int32_t* cnt[8];
    const int32_t* list[8];
    const float* f[8];
    const float* ap[8];
    const float* av[8];
    float w[8];
};
template <int D>
__global__ void k_vhalf(int n, int ns, StagePtrs S, const float* __restrict__ dtp, const float* __restrict__ v0, float* __restrict__ vh) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float dt = *dtp;
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        float fa = 0.f;
        for (int s = 0; s < ns; ++s) fa += S.w[s] * S.dvdt[s][(size_t)i * D + a];
        vh[(size_t)i * D + a] = v0[(size_t)i * D + a] + 0.5f * fa * dt;
    }
}
template <int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_finalize(int n, int ns, StagePtrs S, int pdv, const float* __restrict__ dtp, const float* __restrict__ vh,
           const float* __restrict__ u0, float* __restrict__ u_out, float* __restrict__ du_out) {
    pdl_entry();
    Grp<G> g(n);
    float du = 0.f;
    if (g.valid) {
        Vec<D> vi = load_vec<D>(vh, g.i);
        for (int s = 0; s < ns; ++s) {
            const int32_t* __restrict__ lst = S.list[s];
            const float* __restrict__ f = S.f[s];
            const float* __restrict__ ap = S.ap[s];
            const float* __restrict__ av = S.av[s];
            const float w = S.w[s];
            int b = S.offs[s][g.i], e = b + S.cnt[s][g.i];
            float acc = 0.f;
            for (int q = b + g.lane; q < e; q += G) {
                int j, k; entry(lst, q, j, k);
                Vec<D> vj = load_vec<D>(vh, j);
                Vec<D> a1 = load_vec<D>(ap, k), a2 = load_vec<D>(av, k);
                float fk = __ldg(f + k);
                float d1 = 0.f, d2 = 0.f;
                #pragma unroll
                for (int a = 0; a < D; ++a) { float vji = vj.v[a] - vi.v[a]; d1 += vji * a1.v[a]; d2 += vji * a2.v[a]; }
                acc += pdv ? (w * fk * d1 + w * 0.5f * d2) : (w * fk * (d1 + d2));
            }
            du += acc;
        }
    }
    du = gsum<G>(du);
    if (!g.valid || g.lane != 0) return;
    float dt = *dtp;
    if (du_out) du_out[g.i] = du;
    u_out[g.i] = u0[g.i] + du * dt;
}

// ---------------------------------------------------------------- conservation sums (FP64)
template <int D>
__global__ void k_cons(int n, const float* __restrict__ m, const float* __restrict__ v, const float* __restrict__ u, double* out) {
    pdl_entry();
    double M = 0, KE = 0, IE = 0, p[3] = {0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double mi = m[i];
        double v2 = 0;
        for (int a = 0; a < D; ++a) { double va = v[(size_t)i * D + a]; v2 += va * va; p[a] += mi * va; }
        M += mi; KE += 0.5 * mi * v2; IE += mi * (double)u[i];
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        M += __shfl_xor_sync(0xffffffffu, M, o); KE += __shfl_xor_sync(0xffffffffu, KE, o); IE += __shfl_xor_sync(0xffffffffu, IE, o);
        for (int a = 0; a < 3; ++a) p[a] += __shfl_xor_sync(0xffffffffu, p[a], o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 0, M); atomicAdd(out + 1, KE); atomicAdd(out + 2, IE); atomicAdd(out + 3, KE + IE);
        for (int a = 0; a < D; ++a) atomicAdd(out + 4 + a, p[a]);
    }
}

}  // namespace wsph

using namespace wsph;

// Fixed scratch for sph_compsph_balance_noalloc: n*(dim+1) floats (half-step
// velocities, then P/rho^gamma).  One copy per device, placed by the module loader,
// so the entry point that uses it never calls an allocator.  Every element the
// balance kernel reads is written first by the prep kernel of the same call, so
// nothing in it has to start at zero.
static __device__ __align__(256) float g_balance_scratch[SPH_BALANCE_NOALLOC_MAX_FLOATS];

constexpr int kMaxDevices = 64;

// The scratch address is a property of the context that loaded this module: a
// cudaDeviceReset (or another context made current on the same device) loads the module
// again and may place the array elsewhere.  So the address is cached per device together
// with the unique id of the context it was resolved in (cuCtxGetId, reached through
// cudaGetDriverEntryPoint, so the library does not link the driver API), and resolved
// again with cudaGetSymbolAddress whenever the current context's id differs.
struct ScratchSlot {
    unsigned long long ctx_id;
    float* ptr;
};
static ScratchSlot g_balance_scratch_slot[kMaxDevices];
static std::mutex g_balance_scratch_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The unique id of the context current on this thread; 0 when none is current yet.
static int current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id)
        return set_error(SPH_ERR_CUDA, "sph_compsph_balance_noalloc: the driver does not provide cuCtxGetCurrent/cuCtxGetId");
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return set_error(SPH_ERR_CUDA, "sph_compsph_balance_noalloc: cuCtxGetCurrent failed");
    *id = 0;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return set_error(SPH_ERR_CUDA, "sph_compsph_balance_noalloc: cuCtxGetId failed");
    return SPH_OK;
}

// Address of g_balance_scratch in the current context, resolved once per device and
// context with cudaGetSymbolAddress while that device is current.
static int balance_scratch_on_current_device(float** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_compsph_balance_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(SPH_ERR_BAD_ARG, "sph_compsph_balance_noalloc: device %d >= %d", dev, kMaxDevices);
    unsigned long long id = 0;
    int rc = current_context_id(&id);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(g_balance_scratch_mu);
    ScratchSlot& slot = g_balance_scratch_slot[dev];
    if (id == 0 || !slot.ptr || slot.ctx_id != id) {
        // cudaGetSymbolAddress also initialises the device's primary context when no
        // context was current yet; the id is read again after it
        void* sym = nullptr;
        e = cudaGetSymbolAddress(&sym, g_balance_scratch);
        if (e != cudaSuccess || !sym)
            return set_error(SPH_ERR_CUDA, "sph_compsph_balance_noalloc: cudaGetSymbolAddress on device %d: %s", dev,
                             cudaGetErrorString(e));
        if (id == 0 && (rc = current_context_id(&id))) return rc;
        slot.ptr = static_cast<float*>(sym);
        slot.ctx_id = id;
    }
    *out = slot.ptr;
    return SPH_OK;
}

extern "C" {

int sph_density_gather(const SphParams* p, int64_t n, int32_t support_mode, const float* x, const float* H, const float* m,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list, float* rho_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho_out); CHECK_CSR();
    if (support_mode < 0 || support_mode > 4) return set_error(SPH_ERR_BAD_ARG, "bad support mode %d", support_mode);
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_density<KF, D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, support_mode, P, x, H, m, offs, cnt, list, rho_out)));
    return check_launch("sph_density_gather");
}

int sph_adaptive_h_iter(const SphParams* p, int64_t n, int32_t support_mode, const float* x, const float* H, const float* m,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list, const float* hbounds,
                        float* rho_out, float* H_out, float* ratio_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(hbounds); WSPH_CHECK_PTR(rho_out); WSPH_CHECK_PTR(H_out); CHECK_CSR();
    if (support_mode != SPH_SUPPORT_GATHER) return set_error(SPH_ERR_UNSUPPORTED, "adaptive support: only the gather scheme is implemented");
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_adaptive_h<KF, D, G_SCAN(D)>, grid_g<G_SCAN(D)>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, offs, cnt, list, hbounds, rho_out, H_out, ratio_out)));
    return check_launch("sph_adaptive_h_iter");
}

int sph_owen_iter(const SphParams* p, int64_t n, const float* x, const float* H, const int32_t* offs, const int32_t* cnt,
                  const int32_t* list, const double* lut_nh, const double* lut_psiH, int32_t nlut, double target_nh,
                  const float* hbounds, float* psi0_out, float* psiH_out, float* H_out, float* ratio_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(lut_nh); WSPH_CHECK_PTR(lut_psiH); WSPH_CHECK_PTR(hbounds);
    WSPH_CHECK_PTR(H_out); CHECK_CSR();
    if (nlut < 2) return set_error(SPH_ERR_BAD_ARG, "sph_owen_iter: the table needs at least 2 entries");
    if (!(target_nh > 0.0)) return set_error(SPH_ERR_BAD_ARG, "sph_owen_iter: target n_h must be positive");
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_owen<KF, D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, offs, cnt, list, lut_nh, lut_psiH,
                                                                                             (int)nlut, (float)target_nh, hbounds, psi0_out,
                                                                                             psiH_out, H_out, ratio_out)));
    return check_launch("sph_owen_iter");
}

int sph_crk_volume(const SphParams* p, int64_t n, const float* x, const float* H, const int32_t* offs, const int32_t* cnt,
                   const int32_t* list, float* V_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(V_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_crk_volume<KF, D, G_SCAN(D)>, grid_g<G_SCAN(D)>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, offs, cnt, list, V_out)));
    return check_launch("sph_crk_volume");
}

int sph_crk_factors(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* V,
                    const int32_t* offs, const int32_t* cnt, const int32_t* list, float* A, float* B, float* gradA,
                    float* gradB, float* rho_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(V);
    WSPH_CHECK_PTR(A); WSPH_CHECK_PTR(B); WSPH_CHECK_PTR(gradA); WSPH_CHECK_PTR(gradB); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_crk_factors<KF, D, G_CRK>, grid_g<G_CRK>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, V, offs, cnt, list, A, B, gradA, gradB, rho_out,
                                                                                                   EosOut{nullptr, nullptr, nullptr, nullptr, 0.f})));
    return check_launch("sph_crk_factors");
}

int sph_crk_factors_eos(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* V,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list, float* A, float* B, float* gradA,
                        float* gradB, float* rho_out, const float* u, float* entropy_out, float* P_out, float* c_out,
                        void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(V);
    WSPH_CHECK_PTR(A); WSPH_CHECK_PTR(B); WSPH_CHECK_PTR(gradA); WSPH_CHECK_PTR(gradB); WSPH_CHECK_PTR(rho_out); WSPH_CHECK_PTR(u);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_crk_factors<KF, D, G_CRK>, grid_g<G_CRK>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, V, offs, cnt, list, A, B, gradA, gradB, rho_out,
                                                                                                   EosOut{u, entropy_out, P_out, c_out, P.gamma})));
    return check_launch("sph_crk_factors_eos");
}

int sph_eos_ideal_gas(const SphParams* p, int64_t n, const float* u, const float* rho, float* A_out, float* P_out,
                      float* c_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(u); WSPH_CHECK_PTR(rho);
    wsph::count_launch(); launch_pdl(k_eos, grid_for(n, 256), 256, 0, s, (int)n, P.gamma, u, rho, A_out, P_out, c_out);
    return check_launch("sph_eos_ideal_gas");
}

int sph_grad_v(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
               const float* V, const float* A, const float* B, const float* gradA, const float* gradB, const float* v,
               const float* c, const int32_t* offs, const int32_t* cnt, const int32_t* list, float* DvDx_out,
               float* drhodt_out, float* div_out, float* vsig_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(V); WSPH_CHECK_PTR(A); WSPH_CHECK_PTR(B);
    WSPH_CHECK_PTR(gradA); WSPH_CHECK_PTR(gradB); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(DvDx_out); CHECK_CSR();
    if (div_out) WSPH_CHECK_PTR(m);
    if (vsig_out) WSPH_CHECK_PTR(c);
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, B, "B")) ||
        (rc = check_align_vec(P, gradA, "gradA")))
        return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_grad_v<KF, D, G_SCAN(D)>, grid_g<G_SCAN(D)>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, V, A, B, gradA, gradB, v, c,
                                                                                                  offs, cnt, list, DvDx_out, drhodt_out, div_out, vsig_out)));
    return check_launch("sph_grad_v");
}

int sph_switch_cullen(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                      const float* div, const float* div_prev, const float* vsig, const float* v, const float* c,
                      const float* alpha0_prev, const float* dt, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                      float* alpha_out, float* R_out, float* vsig_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(div); WSPH_CHECK_PTR(div_prev);
    WSPH_CHECK_PTR(alpha0_prev); WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(alpha_out); CHECK_CSR();
    if (!vsig) { WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(c); }   // v_sig needs the whole Verlet rows
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_cullen<KF, D, G_SCAN(D)>, grid_g<G_SCAN(D)>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, div, div_prev, vsig, v, c,
                                                                                                  alpha0_prev, dt, offs, cnt, list, alpha_out, R_out, vsig_out)));
    return check_launch("sph_switch_cullen");
}

int sph_switch_hopkins_terms(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                             const float* v, const float* alpha0, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                             float* div_out, float* shear2_out, float* alpha_out, float* R_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(alpha0);
    WSPH_CHECK_PTR(div_out); WSPH_CHECK_PTR(shear2_out); WSPH_CHECK_PTR(alpha_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_hopkins_grad<KF, D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, v, offs, cnt, list,
                                                                                                       div_out, shear2_out)));
    if ((rc = check_launch("sph_switch_hopkins_terms"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_hopkins_alpha<KF, D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, div_out, shear2_out,
                                                                                                        alpha0, offs, cnt, list, alpha_out, R_out)));
    return check_launch("sph_switch_hopkins_terms");
}

int sph_switch_hopkins_update(const SphParams* p, int64_t n, const float* x, const float* H, const float* v, const float* c,
                              const float* div, const float* div_prev, const float* alpha0, const float* dt,
                              const int32_t* offs, const int32_t* cnt, const int32_t* list, float* alpha0_out, float* vsig_out,
                              void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(c); WSPH_CHECK_PTR(div); WSPH_CHECK_PTR(div_prev);
    WSPH_CHECK_PTR(alpha0); WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(alpha0_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_DS(*p, (launch_pdl(k_hopkins_update<D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, v, c, div, div_prev, alpha0, dt,
                                                                                                  offs, cnt, list, alpha0_out, vsig_out)));
    return check_launch("sph_switch_hopkins_update");
}

int sph_switch_balsara(const SphParams* p, int64_t n, const float* DvDx, const float* c, float* alpha_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(DvDx); WSPH_CHECK_PTR(c); WSPH_CHECK_PTR(alpha_out);
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (launch_pdl(k_balsara<D>, grid_for(n, 256), 256, 0, s, (int)n, DvDx, c, alpha_out)));
    return check_launch("sph_switch_balsara");
}

static int crk_accel_dudt_impl(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                               const float* rho, const float* V, const float* A, const float* B, const float* gradA,
                               const float* gradB, const float* v, const float* c, const float* Pr, const float* DvDx,
                               const int32_t* offs, const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt,
                               float* dvdt_out, float* dudt_out, float* dEdt_out, float* ap_ij, float* av_ij, float* records,
                               void* stream, const char* name) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(V); WSPH_CHECK_PTR(A);
    WSPH_CHECK_PTR(B); WSPH_CHECK_PTR(gradA); WSPH_CHECK_PTR(gradB); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(c); WSPH_CHECK_PTR(Pr);
    WSPH_CHECK_PTR(DvDx); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, B, "B")) ||
        (rc = check_align_vec(P, gradA, "gradA")) || (rc = check_align_vec(P, dvdt_out, "dvdt")) ||
        (rc = check_align_vec(P, ap_ij, "ap_ij")) || (rc = check_align_vec(P, av_ij, "av_ij")))
        return rc;
    if (records && (reinterpret_cast<uintptr_t>(records) & 15))
        return set_error(SPH_ERR_BAD_ARG, "%s: records must be 16-byte aligned", name);
    if (records) {
        wsph::count_launch();
        WSPH_DISPATCH_DS(*p, (launch_pdl(k_crk_pack<D>, (unsigned)((n + 255) / 256), 256, 0, s, (int)n, x, H, rho, V, A, B, gradA, gradB, v, c,
                                                                                       Pr, DvDx, records)));
        wsph::count_launch();
        WSPH_DISPATCH_KDS(*p, (launch_pdl(k_crk_accel_dudt<KF, D, G_ACCEL, true>, grid_g<G_ACCEL>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, V, A, B, gradA, gradB, v, c, Pr, DvDx, records, offs, cnt, list,
                                  verlet_cnt, dvdt_out, dudt_out, dEdt_out, ap_ij, av_ij)));
    } else {
        wsph::count_launch();
        WSPH_DISPATCH_KDS(*p, (launch_pdl(k_crk_accel_dudt<KF, D, G_ACCEL, false>, grid_g<G_ACCEL>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, V, A, B, gradA, gradB, v, c, Pr, DvDx, nullptr, offs, cnt, list,
                                  verlet_cnt, dvdt_out, dudt_out, dEdt_out, ap_ij, av_ij)));
    }
    return check_launch(name);
}

int sph_crk_accel_dudt(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                       const float* V, const float* A, const float* B, const float* gradA, const float* gradB,
                       const float* v, const float* c, const float* Pr, const float* DvDx, const int32_t* offs,
                       const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt, float* dvdt_out, float* dudt_out,
                       float* dEdt_out, float* ap_ij, float* av_ij, void* stream) {
    return crk_accel_dudt_impl(p, n, x, H, m, rho, V, A, B, gradA, gradB, v, c, Pr, DvDx, offs, cnt, list, verlet_cnt, dvdt_out,
                               dudt_out, dEdt_out, ap_ij, av_ij, nullptr, stream, "sph_crk_accel_dudt");
}

int sph_crk_record_floats(int32_t dim) {
    return dim == 1 ? CrkRec<1>::R : dim == 2 ? CrkRec<2>::R : dim == 3 ? CrkRec<3>::R : 0;
}

int sph_crk_accel_dudt_packed(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                              const float* V, const float* A, const float* B, const float* gradA, const float* gradB,
                              const float* v, const float* c, const float* Pr, const float* DvDx, const int32_t* offs,
                              const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt, float* dvdt_out,
                              float* dudt_out, float* dEdt_out, float* ap_ij, float* av_ij, float* records, void* stream) {
    WSPH_CHECK_PTR(records);
    return crk_accel_dudt_impl(p, n, x, H, m, rho, V, A, B, gradA, gradB, v, c, Pr, DvDx, offs, cnt, list, verlet_cnt, dvdt_out,
                               dudt_out, dEdt_out, ap_ij, av_ij, records, stream, "sph_crk_accel_dudt_packed");
}

int sph_crk_accel(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                  const float* V, const float* A, const float* B, const float* gradA, const float* gradB, const float* v,
                  const float* c, const float* P, const float* DvDx, const int32_t* offs, const int32_t* cnt,
                  const int32_t* list, const int32_t* verlet_cnt, float* dvdt_out, float* ap_ij, float* av_ij, void* stream) {
    return sph_crk_accel_dudt(p, n, x, H, m, rho, V, A, B, gradA, gradB, v, c, P, DvDx, offs, cnt, list, verlet_cnt, dvdt_out,
                              nullptr, nullptr, ap_ij, av_ij, stream);
}

int sph_crk_dudt(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                 const float* V, const float* A, const float* B, const float* gradA, const float* gradB, const float* v,
                 const float* c, const float* P, const float* DvDx, const int32_t* offs, const int32_t* cnt,
                 const int32_t* list, float* dudt_out, void* stream) {
    return sph_crk_accel_dudt(p, n, x, H, m, rho, V, A, B, gradA, gradB, v, c, P, DvDx, offs, cnt, list, nullptr, nullptr, dudt_out,
                              nullptr, nullptr, nullptr, stream);
}

int sph_compsph_balance(const SphParams* p, int64_t n, const float* m, const float* rho, const float* Pr, const float* u,
                        const float* v, const float* dvdt, const float* dt, const int32_t* offs, const int32_t* cnt,
                        const int32_t* list, const int32_t* inter_counts, const float* ap_ij, const float* av_ij, float* scratch,
                        float* f_ij_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(Pr); WSPH_CHECK_PTR(u); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(dvdt);
    WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(ap_ij); WSPH_CHECK_PTR(av_ij); WSPH_CHECK_PTR(scratch); WSPH_CHECK_PTR(f_ij_out); CHECK_CSR();
    if (P.energy_scheme < 0 || P.energy_scheme > 5) return set_error(SPH_ERR_BAD_ARG, "bad energy scheme %d", P.energy_scheme);
    if ((rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt, "dvdt")) || (rc = check_align_vec(P, ap_ij, "ap_ij")) ||
        (rc = check_align_vec(P, av_ij, "av_ij")) || (rc = check_align_vec(P, scratch, "scratch")))
        return rc;
    float* vh = scratch;
    float* sarr = scratch + n * P.dim;
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (launch_pdl(k_balance_prep<D>, grid_for(n, 256), 256, 0, s, (int)n, P, rho, Pr, v, dvdt, dt, vh, sarr)));
    wsph::count_launch();
    WSPH_DISPATCH_DS(*p, (launch_pdl(k_balance<D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, m, rho, Pr, u, vh, sarr, dt, offs, cnt, list, inter_counts, ap_ij, av_ij, f_ij_out)));
    return check_launch("sph_compsph_balance");
}

// sph_compsph_balance with its scratch taken from g_balance_scratch instead of the
// caller.  For callers that cannot allocate device memory on the step path: a plain C
// or Fortran host code bound through the FFI with no caching allocator of its own, or
// a timed inner loop, where cudaMalloc/cudaFree would synchronise the whole device.
// The first call on each device (and the first after that device's context was replaced,
// e.g. by cudaDeviceReset) resolves the scratch address (cudaGetSymbolAddress); make that
// first call before any stream capture.  Every device that loads the library holds the
// 16 MiB array until the process exits.  Calls in flight at the same time on one device
// (different streams, or different host threads) share the scratch and race.
int sph_compsph_balance_noalloc(const SphParams* p, int64_t n, const float* m, const float* rho, const float* Pr,
                                const float* u, const float* v, const float* dvdt, const float* dt, const int32_t* offs,
                                const int32_t* cnt, const int32_t* list, const float* ap_ij, const float* av_ij,
                                float* f_ij_out, void* stream) {
    if (!p) return set_error(SPH_ERR_BAD_ARG, "sph_compsph_balance_noalloc: null params");
    if (p->dim < 1 || p->dim > 3) return set_error(SPH_ERR_BAD_ARG, "sph_compsph_balance_noalloc: dim must be 1, 2 or 3");
    if (n > 0 && n * (int64_t)(p->dim + 1) > (int64_t)SPH_BALANCE_NOALLOC_MAX_FLOATS)
        return set_error(SPH_ERR_BAD_ARG, "sph_compsph_balance_noalloc: n*(dim+1) = %lld exceeds the fixed scratch of %d floats",
                         (long long)(n * (p->dim + 1)), SPH_BALANCE_NOALLOC_MAX_FLOATS);
    if (n <= 0) return sph_compsph_balance(p, n, m, rho, Pr, u, v, dvdt, dt, offs, cnt, list, nullptr, ap_ij, av_ij, nullptr, f_ij_out, stream);
    float* scratch = nullptr;
    int rc = balance_scratch_on_current_device(&scratch);
    if (rc) return rc;
    return sph_compsph_balance(p, n, m, rho, Pr, u, v, dvdt, dt, offs, cnt, list, nullptr, ap_ij, av_ij, scratch, f_ij_out, stream);
}

int sph_cfl_dt(const SphParams* p, int64_t n, const float* H, const float* u, const float* rho, const float* dt_prev,
               float* dt_out, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (n <= 0 || n > 0x7fffffff) return set_error(SPH_ERR_BAD_ARG, "sph_cfl_dt: n must be in [1, 2^31)");
    WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(u); WSPH_CHECK_PTR(dt_out);
    (void)rho;
    cudaStream_t s = WSPH_STREAM(stream);
    float* red = dt_out + 1;
    wsph::count_launch(); launch_pdl(k_cfl_init, 1, 1, 0, s, red);
    int blocks = (int)((n + 1023) / 1024);
    if (blocks > 148 * 4) blocks = 148 * 4;
    wsph::count_launch(); launch_pdl(k_cfl_reduce, blocks, 256, 0, s, (int)n, P.gamma, H, u, red);
    wsph::count_launch(); launch_pdl(k_cfl_final, 1, 1, 0, s, P, red, dt_prev, dt_out);
    return check_launch("sph_cfl_dt");
}

int sph_rk_combine(const SphParams* p, int64_t count, const float* y0, int32_t nk, const float* const* k_ptrs,
                   const double* weights, const float* dt, int32_t wrap_dim, float* y_out, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (count < 0) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine: count < 0");
    if (count == 0) return SPH_OK;
    if (nk < 0 || nk > 8) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine: nk must be in [0, 8]");
    WSPH_CHECK_PTR(y0); WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(y_out);
    KPtrs K;
    for (int q = 0; q < 8; ++q) { K.k[q] = nullptr; K.w[q] = 0.f; }
    for (int q = 0; q < nk; ++q) {
        if (!k_ptrs || !k_ptrs[q] || !weights) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine: null derivative %d", q);
        K.k[q] = k_ptrs[q]; K.w[q] = (float)weights[q];
    }
    wsph::count_launch(); launch_pdl(k_rk_combine, grid_for(count, 256), 256, 0, WSPH_STREAM(stream), count, y0, nk, K, dt, wrap_dim, P.dom, y_out);
    return check_launch("sph_rk_combine");
}

int sph_rk_combine_fields(const SphParams* p, int32_t nfields, const int64_t* counts, const float* const* y0s,
                          float* const* y_outs, const int32_t* wrap_dims, int32_t nk, const float* const* k_ptrs,
                          const double* weights, const float* dt, void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    if (nfields < 1 || nfields > RKF_MAX) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: nfields must be in [1, %d]", RKF_MAX);
    if (nk < 0 || nk > 8) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: nk must be in [0, 8]");
    WSPH_CHECK_PTR(counts); WSPH_CHECK_PTR(y0s); WSPH_CHECK_PTR(y_outs); WSPH_CHECK_PTR(wrap_dims); WSPH_CHECK_PTR(dt);
    if (nk > 0) { WSPH_CHECK_PTR(k_ptrs); WSPH_CHECK_PTR(weights); }
    FieldPtrs F;
    memset(&F, 0, sizeof(F));
    int64_t total = 0;
    for (int f = 0; f < nfields; ++f) {
        if (counts[f] < 0) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: count %d < 0", f);
        if (counts[f] > 0 && (!y0s[f] || !y_outs[f])) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: null field %d", f);
        if (wrap_dims[f] < 0 || wrap_dims[f] > 3) return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: wrap_dim %d out of range", f);
        F.y0[f] = y0s[f]; F.y[f] = y_outs[f]; F.wrap[f] = wrap_dims[f];
        for (int q = 0; q < nk; ++q) {
            if (counts[f] > 0 && !k_ptrs[f * nk + q])
                return set_error(SPH_ERR_BAD_ARG, "sph_rk_combine_fields: null derivative %d of field %d", q, f);
            F.k[f][q] = k_ptrs[f * nk + q];
        }
        total += counts[f];
        F.end[f] = total;
    }
    for (int q = 0; q < nk; ++q) F.w[q] = (float)weights[q];
    if (total == 0) return SPH_OK;
    wsph::count_launch();
    launch_pdl(k_rk_combine_fields, grid_for(total, 256), 256, 0, WSPH_STREAM(stream), nfields, nk, F, dt, P.dom);
    return check_launch("sph_rk_combine_fields");
}

int sph_finalize_compatible_energy(const SphParams* p, int64_t n, int32_t nstages, const double* weights, const float* dt,
                                   const float* v0, const float* u0, const float* const* dvdt_s,
                                   const int32_t* const* offs_s, const int32_t* const* cnt_s, const int32_t* const* list_s,
                                   const float* const* f_ij_s, const float* const* ap_ij_s, const float* const* av_ij_s,
                                   float* u_out, float* du_out, void* stream) {
    PAIR_PRELUDE();
    if (nstages < 1 || nstages > 8) return set_error(SPH_ERR_BAD_ARG, "nstages must be in [1, 8]");
    WSPH_CHECK_PTR(weights); WSPH_CHECK_PTR(dt); WSPH_CHECK_PTR(v0); WSPH_CHECK_PTR(u0); WSPH_CHECK_PTR(u_out);
    WSPH_CHECK_PTR(dvdt_s); WSPH_CHECK_PTR(offs_s); WSPH_CHECK_PTR(cnt_s); WSPH_CHECK_PTR(list_s);
    WSPH_CHECK_PTR(f_ij_s); WSPH_CHECK_PTR(ap_ij_s); WSPH_CHECK_PTR(av_ij_s);
    StagePtrs S;
    for (int q = 0; q < nstages; ++q) {
        if (!dvdt_s[q] || !offs_s[q] || !cnt_s[q] || !list_s[q] || !f_ij_s[q] || !ap_ij_s[q] || !av_ij_s[q])
            return set_error(SPH_ERR_BAD_ARG, "finalize: null array for stage %d", q);
        S.dvdt[q] = dvdt_s[q]; S.offs[q] = offs_s[q]; S.cnt[q] = cnt_s[q]; S.list[q] = list_s[q];
        S.f[q] = f_ij_s[q]; S.ap[q] = ap_ij_s[q]; S.av[q] = av_ij_s[q]; S.w[q] = (float)weights[q];
    }
    if (!du_out) return set_error(SPH_ERR_BAD_ARG, "finalize: du_out must hold n*(1+dim) floats (du and v_half scratch)");
    float* vh = du_out + n;
    int pdv = P.energy_scheme == SPH_ENERGY_PDV;
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (launch_pdl(k_vhalf<D>, grid_for(n, 256), 256, 0, s, (int)n, nstages, S, dt, v0, vh)));
    wsph::count_launch();
    WSPH_DISPATCH_DS(*p, (launch_pdl(k_finalize<D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, nstages, S, pdv, dt, vh, u0, u_out, du_out)));
    return check_launch("sph_finalize_compatible_energy");
}

int sph_conservation_sums(const SphParams* p, int64_t n, const float* m, const float* v, const float* u, double* out,
                          void* stream) {
    DevParams P;
    int rc = params_to_dev(p, &P);
    if (rc) return rc;
    WSPH_CHECK_PTR(out);
    cudaStream_t s = WSPH_STREAM(stream);
    cudaMemsetAsync(out, 0, sizeof(double) * 7, s);
    if (n <= 0) return check_launch("sph_conservation_sums");
    WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(u);
    int blocks = grid_for(n, 256);
    if (blocks > 148 * 4) blocks = 148 * 4;
    wsph::count_launch(); WSPH_DISPATCH_DIM(P.dim, (launch_pdl(k_cons<D>, blocks, 256, 0, s, (int)n, m, v, u, out)));
    return check_launch("sph_conservation_sums");
}

}  // extern "C"
