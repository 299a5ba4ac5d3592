// Pair passes of the CompSPH (grad-h, compatibly differenced) and Monaghan compressible
// schemes.  Same lane layout as the CRK passes: G lanes of a warp per particle, over
// Verlet rows or their interacting prefixes (r < max(H_i, H_j)).
//
//   k_compsph_prep        Omega (grad-h, gather), the super-symmetric velocity divergence
//                         of the Cullen switch and the consistent continuity d rho/dt,
//                         all from one walk of the row (three reference passes).
//   k_compsph_accel_dudt  CompSPH momentum and energy right-hand sides, pairwise
//                         pressure / viscous accelerations for the energy partition.
//   k_monaghan_rhs        symmetric pressure force, PdV work, artificial viscosity,
//                         conductivity and viscous heating of the Monaghan scheme.
//
// Arithmetic restates the reference at the file:line given at each kernel.
#include <cuda_runtime.h>
#include "sph_pair_common.cuh"
#include "sph_pi.cuh"

namespace wsph {

// ---------------------------------------------------------------- Omega, divergence, continuity
// Omega_i = 1 - sum_j (-H_i / (rho_i d)) m_j dW/dH(r_ij, H_i)
//   (modules/adaptiveSupport/wp_omega.py:11-78, :140; gather support at schemes/compSPH.py:90-97);
// div_i = sum_j m_j / rho_j (v_j - v_i) . grad W(r_ij, max(H_i, H_j))
//   (difference divergence, super-symmetric support: CullenDehnen2010.py:246-257);
// d rho_i/dt = -(rho_i / Omega_i) (1 / rho_i) sum_j m_j (v_j - v_i) . grad W(r_ij, max(H_i, H_j))
//   (modules/momentum/consistent.py:8-35, the consistent divergence weighting each
//   neighbour by m_j / rho_i, so that rho_i cancels).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_compsph_prep(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
               const float* __restrict__ rho, const float* __restrict__ v,
               const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
               float* __restrict__ omega, float* __restrict__ div, float* __restrict__ drhodt) {
    pdl_entry();
    Grp<G> g(n);
    const bool want_om = omega != nullptr, want_div = div != nullptr, want_con = drhodt != nullptr;
    float sdh = 0.f, sdiv = 0.f, scon = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        Vec<D> vi = (want_div || want_con) ? load_vec<D>(v, i) : vzero<D>();
        const float Hi = H[i];
        int b = offs[i], e = b + cnt[i];
        RowPipe<D> rp(list, x, b + g.lane, e, G);
        for (int q = b + g.lane; q < e; q += G) {
            int j; Vec<D> xj; rp.take(q, j, xj);
            // every gather of the entry issued together, ahead of the tests that select them
            const float Hj = __ldg(H + j), mj = __ldg(m + j);
            const float rhoj = want_div ? __ldg(rho + j) : 1.f;
            const Vec<D> vj = (want_div || want_con) ? load_vec<D>(v, j) : vzero<D>();
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r2 = dot<D>(xij, xij);
            float Hs = wmax(Hi, Hj);
            if (!(r2 < Hs * Hs)) continue;
            float r = safe_sqrt(r2);
            if (want_om && r < Hi) {
                float W, dWdH;
                kernelWdH<KF, D>(r, Hi, W, dWdH);
                sdh += mj * dWdH;
            }
            if (want_div || want_con) {
                float W; Vec<D> gS;
                kWG_inv<KF, D>(xij, r, 1.f / Hs, W, gS);
                float s = 0.f;
                #pragma unroll
                for (int a = 0; a < D; ++a) s += (vj.v[a] - vi.v[a]) * gS.v[a];
                if (want_div) sdiv += mj / rhoj * s;
                scon += mj * s;
            }
        }
    }
    if (want_om) sdh = gsum<G>(sdh);
    if (want_div) sdiv = gsum<G>(sdiv);
    if (want_con) scon = gsum<G>(scon);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    float om = 1.f;
    if (want_om) {
        const float dh_drho = -H[i] / (rho[i] * (float)D);
        om = 1.f - dh_drho * sdh;
        omega[i] = om;
    }
    if (want_div) div[i] = sdiv;
    if (want_con) drhodt[i] = -scon / om;
}

// ---------------------------------------------------------------- CompSPH accel + dudt
// modules/compSPH/accel.py:60-154 (kernel-mean gradient (grad W(H_i) + grad W(H_j)) / 2,
// grad-h pressure terms P / (rho^2 Omega), Pi from computePi_actual scaled by rho_bar / rho)
// and modules/compSPH/dudt.py:60-139 (gather gradient grad W(H_i)) in one pass; dE/dt of
// schemes/compSPH.py:170 per particle.  Without Omega the grad-h terms are 1, without
// alpha the switch is 1 and without c the sound speed is DiffusionParameters.c_s
// (accel.py:195-198).  Walking the interacting prefix of each Verlet row (cnt =
// interacting counts) with vcnt = the Verlet counts, the ap_ij / av_ij entries of the
// rest of the row are written as zeros.
// Packed per-particle record of the CompSPH accel pass: position and support first (read
// before the distance test), then velocity, mass, density, pressure, sound speed, switch
// and grad-h factor, in one block of R floats (16-byte granules), so a neighbour is R/4
// 128-bit loads from one record instead of 2D + 8 scalar loads from as many arrays.  The
// optional fields take their defaults at pack time (sound speed c_s, switch 1, Omega 1).
template <int D> struct CompRec {
    static constexpr int X = 0, H = D, V = D + 1, M = 2 * D + 1, RHO = M + 1, P = M + 2, C = M + 3, AL = M + 4, OM = M + 5,
                         END = M + 6, R = (END + 3) / 4 * 4, K1 = (H + 1 + 3) / 4, K2 = R / 4;
};

template <int D>
__global__ void k_compsph_pack(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                               const float* __restrict__ rho, const float* __restrict__ v, const float* __restrict__ c,
                               const float* __restrict__ alpha, const float* __restrict__ Pr, const float* __restrict__ omega,
                               float* __restrict__ rec) {
    pdl_entry();
    using L = CompRec<D>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r[L::R];
    #pragma unroll
    for (int a = 0; a < D; ++a) { r[L::X + a] = x[(size_t)i * D + a]; r[L::V + a] = v[(size_t)i * D + a]; }
    r[L::H] = H[i]; r[L::M] = m[i]; r[L::RHO] = rho[i]; r[L::P] = Pr[i];
    r[L::C] = c ? c[i] : P.c_s; r[L::AL] = alpha ? alpha[i] : 1.f; r[L::OM] = omega ? omega[i] : 1.f;
    #pragma unroll
    for (int a = L::END; a < L::R; ++a) r[a] = 0.f;
    float4* dst = reinterpret_cast<float4*>(rec + (size_t)i * L::R);
    #pragma unroll
    for (int k = 0; k < L::R / 4; ++k) dst[k] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
}

template <int D, int K0, int K1>
__device__ __forceinline__ void comp_granules(const float4* __restrict__ src, float (&r)[CompRec<D>::R]) {
    #pragma unroll
    for (int k = K0; k < K1; ++k) {
        const float4 t = __ldg(src + k);
        r[4 * k] = t.x; r[4 * k + 1] = t.y; r[4 * k + 2] = t.z; r[4 * k + 3] = t.w;
    }
}

template <int KF, int D, int G, bool REC>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_compsph_accel_dudt(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                     const float* __restrict__ rho, const float* __restrict__ v, const float* __restrict__ c,
                     const float* __restrict__ alpha, const float* __restrict__ Pr, const float* __restrict__ omega,
                     const float* __restrict__ rec,
                     const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
                     const int32_t* __restrict__ vcnt, float* __restrict__ dvdt, float* __restrict__ dudt,
                     float* __restrict__ dEdt, float* __restrict__ ap, float* __restrict__ av) {
    pdl_entry();
    Grp<G> g(n);
    const bool comp = P.kahan != 0;
    KSum acc[D], du;
    #pragma unroll
    for (int a = 0; a < D; ++a) acc[a].init();
    du.init();
    if (g.valid) {
        const int i = g.i;
        using L = CompRec<D>;
        Vec<D> xi, vi;
        float Hi, rhoi, Pi, ci, ai, omi;
        if constexpr (REC) {
            float r[L::R];
            comp_granules<D, 0, L::K2>(reinterpret_cast<const float4*>(rec + (size_t)i * L::R), r);
            #pragma unroll
            for (int a = 0; a < D; ++a) { xi.v[a] = r[L::X + a]; vi.v[a] = r[L::V + a]; }
            Hi = r[L::H]; rhoi = r[L::RHO]; Pi = r[L::P]; ci = r[L::C]; ai = r[L::AL]; omi = r[L::OM];
        } else {
            xi = load_vec<D>(x, i); vi = load_vec<D>(v, i);
            Hi = H[i]; rhoi = rho[i]; Pi = Pr[i];
            ci = c ? c[i] : P.c_s; ai = alpha ? alpha[i] : 1.f; omi = omega ? omega[i] : 1.f;
        }
        const float invHi = 1.f / Hi;
        const float pTi = Pi / (rhoi * rhoi) / omi;
        int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            float rj[L::R];
            const float4* sj = REC ? reinterpret_cast<const float4*>(rec + (size_t)j * L::R) : nullptr;
            Vec<D> xj;
            float Hj;
            if constexpr (REC) {
                // the first two groups issued together (walked rows are interacting prefixes, so
                // the range test below almost never discards the second)
                comp_granules<D, 0, L::K2>(sj, rj);
                #pragma unroll
                for (int a = 0; a < D; ++a) xj.v[a] = rj[L::X + a];
                Hj = rj[L::H];
            } else {
                xj = load_vec<D>(x, j);
                Hj = __ldg(H + j);
            }
            Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            float r2 = dot<D>(xij, xij);
            float Hm = wmax(Hi, Hj);
            if (!(r2 < Hm * Hm)) {
                if (ap) store_vec<D>(ap, k, vzero<D>());
                if (av) store_vec<D>(av, k, vzero<D>());
                continue;
            }
            float r = safe_sqrt(r2);
            Vec<D> vj;
            float mj, rhoj, Pj, cj, aj, omj;
            if constexpr (REC) {
                #pragma unroll
                for (int a = 0; a < D; ++a) vj.v[a] = rj[L::V + a];
                mj = rj[L::M]; rhoj = rj[L::RHO]; Pj = rj[L::P]; cj = rj[L::C]; aj = rj[L::AL]; omj = rj[L::OM];
            } else {
                vj = load_vec<D>(v, j);
                mj = __ldg(m + j); rhoj = __ldg(rho + j); Pj = __ldg(Pr + j);
                cj = c ? __ldg(c + j) : P.c_s; aj = alpha ? __ldg(alpha + j) : 1.f; omj = omega ? __ldg(omega + j) : 1.f;
            }
            const float Vj = mj / rhoj;
            const float rho_bar = 0.5f * (rhoi + rhoj);
            float ux = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) ux += (vi.v[a] - vj.v[a]) * xij.v[a];
            const float pi_i = pi_actual(P, D, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, true, ci, cj, ai, aj, false, false) * (rho_bar / rhoi);
            const float pi_j = pi_actual(P, D, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, true, ci, cj, ai, aj, true, false) * (rho_bar / rhoj);
            float Wi, Wj; Vec<D> gi, gj;
            kWG_inv<KF, D>(xij, r, invHi, Wi, gi);
            kWG_inv<KF, D>(xij, r, 1.f / Hj, Wj, gj);
            const float pTj = Pj / (rhoj * rhoj) / omj;
            // (v_j - v_i) . x_ij / (r + 1e-14 H_i)
            const float mu = -ux / (r + 1.0e-14f * Hi);
            Vec<D> pt, vt;
            float dotg = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                const float gw = 0.5f * (gi.v[a] + gj.v[a]);
                pt.v[a] = -(pTi * gw + pTj * gw) * mj;
                vt.v[a] = -0.5f * (pi_i * gw + pi_j * gw) * Vj * mu;
                acc[a].add(pt.v[a] + vt.v[a], comp);
                dotg += (vj.v[a] - vi.v[a]) * gi.v[a];
            }
            if (ap) store_vec<D>(ap, k, pt);
            if (av) store_vec<D>(av, k, vt);
            const float pTerm = -Vj * pTi * rhoj * dotg;
            const float vTerm = -0.5f * Vj * pi_i * mu * dotg;
            du.add(pTerm + vTerm, comp);
        }
        if (vcnt && (ap || av)) {
            const int te = b + __ldg(vcnt + i);
            for (int q = e + g.lane; q < te; q += G) {
                if (ap) store_vec<D>(ap, q, vzero<D>());
                if (av) store_vec<D>(av, q, vzero<D>());
            }
        }
    }
    float o[D], od;
    #pragma unroll
    for (int a = 0; a < D; ++a) o[a] = gsum<G>(acc[a].s) + gsum<G>(acc[a].c);
    od = gsum<G>(du.s) + gsum<G>(du.c);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    Vec<D> ov;
    #pragma unroll
    for (int a = 0; a < D; ++a) ov.v[a] = o[a];
    if (dvdt) store_vec<D>(dvdt, i, ov);
    if (dudt) dudt[i] = od;
    if (dEdt) {
        Vec<D> vi;
        float mi;
        if constexpr (REC) {
            #pragma unroll
            for (int a = 0; a < D; ++a) vi.v[a] = __ldg(rec + (size_t)i * CompRec<D>::R + CompRec<D>::V + a);
            mi = __ldg(rec + (size_t)i * CompRec<D>::R + CompRec<D>::M);
        } else {
            vi = load_vec<D>(v, i);
            mi = m[i];
        }
        dEdt[i] = mi * dot<D>(vi, ov) + mi * od;
    }
}

// ---------------------------------------------------------------- Monaghan scheme right-hand side
// schemes/monaghan.py:77-143 with kernel-mean support grad W = (grad W(H_i) + grad W(H_j)) / 2:
//   pressure   -(grad P)_sym / rho with grad-h terms: -sum_j m_j (P_i/(rho_i^2 Omega_i)
//              + P_j/(rho_j^2 Omega_j)) grad W (pressure/symmetricForce.py:7-27)
//   PdV        -(P_i / (rho_i Omega_i)) (1/rho_i) sum_j m_j (v_j - v_i) . grad W
//              (internalEnergy/dudt.py:7-33, consistent divergence)
//   viscosity  sum_j V_j Pi_ij grad W mu_ij, mu_ij = (v_i - v_j).x_ij / (r + 1e-14 H_i)
//              (dissipation/wp_diffusion.py:71-107)
//   conduction -1/2 sum_j V_j Pi^u_ij (u_j - u_i) grad W . x_ij / (r + 1e-14 H_i)
//              (dissipation/wp_conductivity.py:59-115, conductivity coefficients and form)
//   heating    -sum_j V_j Pi_ij ((v_j - v_i).x_ij / (r + 1e-14 H_i))^2 grad W . x_ij / (r + 1e-14 H_i)
//              (dissipation/wp_dissipation.py:59-119)
// dv/dt = pressure + viscosity; du/dt = PdV + conduction + heating;
// dE/dt = m_i v_i . dv/dt + m_i (PdV + conduction) (monaghan.py:143).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_monaghan_rhs(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
               const float* __restrict__ rho, const float* __restrict__ v, const float* __restrict__ u,
               const float* __restrict__ c, const float* __restrict__ alpha, const float* __restrict__ Pr,
               const float* __restrict__ omega,
               const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
               float* __restrict__ dvdt, float* __restrict__ dudt, float* __restrict__ dEdt,
               float* __restrict__ dvdt_p, float* __restrict__ dvdt_visc, float* __restrict__ dudt_pdv,
               float* __restrict__ dudt_cond, float* __restrict__ dudt_heat) {
    pdl_entry();
    Grp<G> g(n);
    const bool comp = P.kahan != 0;
    KSum sp[D], sv[D], spdv, scond, sheat;
    #pragma unroll
    for (int a = 0; a < D; ++a) { sp[a].init(); sv[a].init(); }
    spdv.init(); scond.init(); sheat.init();
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i), vi = load_vec<D>(v, i);
        const float Hi = H[i], rhoi = rho[i], Pi = Pr[i], ui = u[i];
        const float ci = c ? c[i] : P.c_s, ai = alpha ? alpha[i] : 1.f, omi = omega ? omega[i] : 1.f;
        const float invHi = 1.f / Hi;
        const float pTi = Pi / (rhoi * rhoi) / omi;
        int b = offs[i], e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            float r2 = dot<D>(xij, xij);
            float Hj = __ldg(H + j);
            float Hm = wmax(Hi, Hj);
            if (!(r2 < Hm * Hm)) continue;
            float r = safe_sqrt(r2);
            Vec<D> vj = load_vec<D>(v, j);
            const float mj = __ldg(m + j), rhoj = __ldg(rho + j), Pj = __ldg(Pr + j), uj = __ldg(u + j);
            const float cj = c ? __ldg(c + j) : P.c_s, aj = alpha ? __ldg(alpha + j) : 1.f, omj = omega ? __ldg(omega + j) : 1.f;
            const float Vj = mj / rhoj;
            float ux = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) ux += (vi.v[a] - vj.v[a]) * xij.v[a];
            const float pi_v = pi_actual(P, D, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, true, ci, cj, ai, aj, false, false);
            const float pi_u = pi_actual(P, D, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, true, ci, cj, ai, aj, false, true);
            float Wi, Wj; Vec<D> gi, gj;
            kWG_inv<KF, D>(xij, r, invHi, Wi, gi);
            kWG_inv<KF, D>(xij, r, 1.f / Hj, Wj, gj);
            const float pTj = Pj / (rhoj * rhoj) / omj;
            const float den = r + 1.0e-14f * Hi;
            const float mu = ux / den;
            const float mup = -ux / den;
            const float cp = mj * (pTi + pTj);
            float dvg = 0.f, lap = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) {
                const float gk = 0.5f * (gi.v[a] + gj.v[a]);
                sp[a].add(cp * gk, comp);
                sv[a].add(Vj * pi_v * gk * mu, comp);
                dvg += (vj.v[a] - vi.v[a]) * gk;
                lap += gk * (xij.v[a] / den);
            }
            spdv.add(mj * dvg, comp);
            scond.add(-0.5f * Vj * pi_u * (uj - ui) * lap, comp);
            sheat.add(-Vj * pi_v * (mup * mup) * lap, comp);
        }
    }
    float p_[D], v_[D];
    #pragma unroll
    for (int a = 0; a < D; ++a) {
        p_[a] = gsum<G>(sp[a].s) + gsum<G>(sp[a].c);
        v_[a] = gsum<G>(sv[a].s) + gsum<G>(sv[a].c);
    }
    float pdv = gsum<G>(spdv.s) + gsum<G>(spdv.c);
    float cond = gsum<G>(scond.s) + gsum<G>(scond.c);
    float heat = gsum<G>(sheat.s) + gsum<G>(sheat.c);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const float Pi = Pr[i], rhoi = rho[i], omi = omega ? omega[i] : 1.f;
    const float pTi = Pi / (rhoi * rhoi) / omi;
    Vec<D> ap, avv, tot;
    #pragma unroll
    for (int a = 0; a < D; ++a) { ap.v[a] = -p_[a]; avv.v[a] = v_[a]; tot.v[a] = ap.v[a] + avv.v[a]; }
    const float du_pdv = -pTi * pdv;
    if (dvdt_p) store_vec<D>(dvdt_p, i, ap);
    if (dvdt_visc) store_vec<D>(dvdt_visc, i, avv);
    if (dvdt) store_vec<D>(dvdt, i, tot);
    if (dudt_pdv) dudt_pdv[i] = du_pdv;
    if (dudt_cond) dudt_cond[i] = cond;
    if (dudt_heat) dudt_heat[i] = heat;
    if (dudt) dudt[i] = du_pdv + cond + heat;
    if (dEdt) {
        Vec<D> vi = load_vec<D>(v, i);
        const float mi = m[i];
        dEdt[i] = mi * dot<D>(vi, tot) + mi * (du_pdv + cond);
    }
}

}  // namespace wsph

using namespace wsph;

extern "C" {

int sph_compsph_prep(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                     const float* v, const int32_t* offs, const int32_t* cnt, const int32_t* list, float* omega_out,
                     float* div_out, float* drhodt_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); CHECK_CSR();
    if (div_out || drhodt_out) WSPH_CHECK_PTR(v);
    if (!omega_out && !div_out && !drhodt_out) return SPH_OK;
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v"))) return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_compsph_prep<KF, D, G_LIGHT>, grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, v, offs, cnt, list,
                                                                                                        omega_out, div_out, drhodt_out)));
    return check_launch("sph_compsph_prep");
}

int sph_grad_h_omega(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list, float* omega_out, void* stream) {
    if (!omega_out) return set_error(SPH_ERR_BAD_ARG, "sph_grad_h_omega: null pointer 'omega_out'");
    return sph_compsph_prep(p, n, x, H, m, rho, nullptr, offs, cnt, list, omega_out, nullptr, nullptr, stream);
}

int sph_compsph_accel_dudt(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                           const float* v, const float* c, const float* alpha, const float* Pr, const float* omega,
                           const int32_t* offs, const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt,
                           float* dvdt_out, float* dudt_out, float* dEdt_out, float* ap_ij, float* av_ij, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(Pr);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt_out, "dvdt")) ||
        (rc = check_align_vec(P, ap_ij, "ap_ij")) || (rc = check_align_vec(P, av_ij, "av_ij")))
        return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_compsph_accel_dudt<KF, D, G_HEAVY, false>, grid_g<G_HEAVY>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, v, c, alpha, Pr, omega, nullptr, offs, cnt, list, verlet_cnt, dvdt_out, dudt_out,
                              dEdt_out, ap_ij, av_ij)));
    return check_launch("sph_compsph_accel_dudt");
}

int sph_compsph_record_floats(int32_t dim) {
    return dim == 1 ? CompRec<1>::R : dim == 2 ? CompRec<2>::R : dim == 3 ? CompRec<3>::R : 0;
}

int sph_compsph_accel_dudt_packed(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                                  const float* v, const float* c, const float* alpha, const float* Pr, const float* omega,
                                  const int32_t* offs, const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt,
                                  float* dvdt_out, float* dudt_out, float* dEdt_out, float* ap_ij, float* av_ij, float* records,
                                  void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(Pr);
    WSPH_CHECK_PTR(records);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt_out, "dvdt")) ||
        (rc = check_align_vec(P, ap_ij, "ap_ij")) || (rc = check_align_vec(P, av_ij, "av_ij")))
        return rc;
    if (reinterpret_cast<uintptr_t>(records) & 15) return set_error(SPH_ERR_BAD_ARG, "sph_compsph_accel_dudt_packed: records must be 16-byte aligned");
    wsph::count_launch();
    WSPH_DISPATCH_DS(*p, (launch_pdl(k_compsph_pack<D>, (unsigned)((n + 255) / 256), 256, 0, s, (int)n, P, x, H, m, rho, v, c, alpha, Pr, omega,
                                                                                        records)));
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_compsph_accel_dudt<KF, D, G_HEAVY, true>, grid_g<G_HEAVY>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, v, c, alpha, Pr, omega, records, offs, cnt, list, verlet_cnt, dvdt_out, dudt_out,
                              dEdt_out, ap_ij, av_ij)));
    return check_launch("sph_compsph_accel_dudt_packed");
}

int sph_compsph_accel(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                      const float* v, const float* c, const float* alpha, const float* P, const float* omega,
                      const int32_t* offs, const int32_t* cnt, const int32_t* list, const int32_t* verlet_cnt,
                      float* dvdt_out, float* ap_ij, float* av_ij, void* stream) {
    return sph_compsph_accel_dudt(p, n, x, H, m, rho, v, c, alpha, P, omega, offs, cnt, list, verlet_cnt, dvdt_out, nullptr, nullptr,
                                  ap_ij, av_ij, stream);
}

int sph_compsph_dudt(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                     const float* v, const float* c, const float* alpha, const float* P, const float* omega,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list, float* dudt_out, void* stream) {
    return sph_compsph_accel_dudt(p, n, x, H, m, rho, v, c, alpha, P, omega, offs, cnt, list, nullptr, nullptr, dudt_out, nullptr,
                                  nullptr, nullptr, stream);
}

int sph_monaghan_rhs(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                     const float* v, const float* u, const float* c, const float* alpha, const float* Pr, const float* omega,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list, float* dvdt_out, float* dudt_out,
                     float* dEdt_out, float* dvdt_pressure, float* dvdt_viscosity, float* dudt_pdv,
                     float* dudt_conductivity, float* dudt_heating, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(u);
    WSPH_CHECK_PTR(Pr); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt_out, "dvdt")) ||
        (rc = check_align_vec(P, dvdt_pressure, "dvdt_pressure")) || (rc = check_align_vec(P, dvdt_viscosity, "dvdt_viscosity")))
        return rc;
    wsph::count_launch();
    WSPH_DISPATCH_KDS(*p, (launch_pdl(k_monaghan_rhs<KF, D, G_HEAVY>, grid_g<G_HEAVY>(n), PAIR_BLOCK, 0, s, (int)n, P, x, H, m, rho, v, u, c, alpha, Pr, omega, offs, cnt, list, dvdt_out, dudt_out, dEdt_out,
                              dvdt_pressure, dvdt_viscosity, dudt_pdv, dudt_conductivity, dudt_heating)));
    return check_launch("sph_monaghan_rhs");
}

}  // extern "C"
