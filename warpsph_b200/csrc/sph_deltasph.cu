// Weakly compressible delta-SPH right-hand side (schemes/deltaSPH.py:11-208 without
// boundaries, forcing, gravity and shifting; the free-surface indicators enter the Antuono
// pressure term when the caller passes them):
//
//   pass A  L_i = (sum_j V_j gradW_ij (x) (x_j - x_i))^-1      renormalisation matrix
//           gradRhoL_i = L_i sum_j V_j (rho_j - rho_i) gradW_ij (modules/density/gradRhoL.py:33-56)
//   pass B  drhodt_i   = -rho_i sum_j V_j (v_j - v_i).gradW_ij  (modules/momentum/inconsistent.py:16-31)
//                      + delta (H_i / xi) c0 sum_j V_j psi_ij.gradW_ij
//                        (modules/deltaSPH/densityDiffusion.py:17-35, wp_densityDelta.py:14-118)
//           dvdt_i     = -sum_j V_j p_ij gradW_ij / rho_i       (modules/pressure/wp_surfaceAware.py:10-102, :207)
//                      + sum_j V_j mu_ij f gradW_ij / ((rho_i + rho_j) / 2)
//                        (modules/deltaSPH/wp_viscosityDelta.py:14-108)
// with V_j = m_j / rho_j, gradW_ij = grad_i W(x_i - x_j, max(H_i, H_j)) (super-symmetric
// support), the EOS of modules/eos/weaklyCompressible.py:4-44 evaluated per particle,
// and the delta-SPH, Antuono and viscosity forms selected by SphWcParams.
//
// The same pair bodies serve the batched ensemble (sph_ensemble.cu).
#include <cuda_runtime.h>
#include "sph_deltasph.cuh"

using namespace wsph;

extern "C" {

int sph_deltasph_rhs(const SphParams* p, const SphWcParams* wc, int64_t n, const float* x, const float* H, const float* m,
                     const float* rho, const float* v, const int32_t* surface_mask, const int32_t* offs, const int32_t* cnt,
                     const int32_t* list, float* scratch, float* dvdt_out, float* drhodt_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(wc); WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v);
    WSPH_CHECK_PTR(scratch); WSPH_CHECK_PTR(dvdt_out); WSPH_CHECK_PTR(drhodt_out); CHECK_CSR();
    WcDev W;
    if ((rc = wc_to_dev(wc, P, &W))) return rc;
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, scratch, "scratch")) ||
        (rc = check_align_vec(P, dvdt_out, "dvdt")))
        return rc;
    float* gL = scratch;
    float* Pr = scratch + n * P.dim;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_ds_passA<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, W, x, H, m, rho, offs, cnt,
                                                                                                     list, gL, Pr)));
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_ds_passB<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, W, x, H, m, rho, v,
                                                                                                     gL, Pr, surface_mask, offs, cnt,
                                                                                                     list, dvdt_out, drhodt_out)));
    return check_launch("sph_deltasph_rhs");
}

int sph_wc_visc_continuity(const SphParams* p, const SphWcParams* wc, int64_t n, const float* x, const float* H, const float* m,
                           const float* rho, const float* v, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                           float* dvdt_out, float* drhodt_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(wc); WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v);
    WSPH_CHECK_PTR(dvdt_out); WSPH_CHECK_PTR(drhodt_out); CHECK_CSR();
    WcDev W;
    if ((rc = wc_to_dev(wc, P, &W))) return rc;
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, dvdt_out, "dvdt"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_visc_cont<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, W, x, H, m, rho, v, offs, cnt,
                                                                                                      list, dvdt_out, drhodt_out)));
    return check_launch("sph_wc_visc_continuity");
}

int sph_delta_shift(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho, const float* v,
                    const int32_t* kinds, const int32_t* offs, const int32_t* cnt, const int32_t* list, float cfl, float c0,
                    float R, int32_t nexp, float rho0, uint32_t* scratch, float* shift_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(scratch);
    WSPH_CHECK_PTR(shift_out); CHECK_CSR();
    if (!(c0 > 0.f) || !(rho0 > 0.f)) return set_error(SPH_ERR_BAD_ARG, "sph_delta_shift: c0 and rho0 must be > 0");
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, shift_out, "shift"))) return rc;
    cudaMemsetAsync(scratch, 0, 2 * sizeof(uint32_t), s);
    int blocks = (int)((n + 1023) / 1024);
    if (blocks > 148 * 4) blocks = 148 * 4;
    count_launch();
    WSPH_DISPATCH_DIM(P.dim, (k_vmax<D><<<blocks, 256, 0, s>>>((int)n, v, scratch)));
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_delta_shift<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, m, rho, kinds, offs, cnt,
                                                                                                        list, cfl, c0, R, (int)nexp, rho0,
                                                                                                        scratch, shift_out)));
    return check_launch("sph_delta_shift");
}

int sph_wc_eos(const SphWcParams* wc, int64_t n, const float* rho, float* P_out, void* stream) {
    WSPH_CHECK_PTR(wc);
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_wc_eos: n < 0");
    if (n == 0) return SPH_OK;
    WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(P_out);
    DevParams P;
    memset(&P, 0, sizeof(P));
    WcDev W;
    int rc = wc_to_dev(wc, P, &W);
    if (rc) return rc;
    count_launch();
    k_wc_eos<<<grid_for(n, 256), 256, 0, WSPH_STREAM(stream)>>>((int)n, W, rho, P_out);
    return check_launch("sph_wc_eos");
}

}  // extern "C"
