// Artificial viscosity Pi_ij of modules/dissipation/pi.py:8-161 (computePi_actual) with
// compute_mu_ij and compute_bars of modules/dissipation/util.py:6-134, for the twelve
// ViscosityTerms (configurations/moduleConfigurations/diffusionParameters.py:8-20).
// Shared by the CompSPH and Monaghan pair passes.
#pragma once
#include "sph_common.cuh"

namespace wsph {

// x_ij = x_i - x_j, r = |x_ij|, ux = (v_i - v_j).x_ij; H are supports; useJ selects the j
// particle's values where a term does not use the pair average (compute_bars); thermal
// selects the conductivity coefficients and form and disables the Monaghan switch.  The
// result is Pi_ij multiplied by rho_j, as in the reference.
__device__ __forceinline__ float pi_actual(const DevParams& P, int dim, float r, float ux, float hi, float hj, float rhoi, float rhoj,
                                           float Pi_, float Pj_, bool explicitP, float ci, float cj, float ai, float aj, bool useJ,
                                           bool thermal) {
    const float rho_bar = 0.5f * (rhoi + rhoj), c_bar = 0.5f * (ci + cj), h_bar = 0.5f * (hi + hj);
    const float xi = P.correct_xi ? P.kxi : 1.f;
    const float Cl0 = thermal ? P.Cu_l : P.C_l, Cq0 = thermal ? P.Cu_q : P.C_q;
    const float C_l = 0.5f * (ai + aj) * Cl0;
    float C_q = 0.5f * (ai + aj) * Cq0;
    if (P.scale_beta) C_q = C_q * C_l;
    const int term = thermal ? P.conductivity_term : P.viscosity_term;
    // compute_mu_ij (util.py:6-38)
    const float den = r + 1e-14f * h_bar;
    const float mu0 = ux / den;
    const float sfac = h_bar / xi / den;
    float mu, sf;
    switch (term) {
        case SPH_VISC_CLEARY1998: case SPH_VISC_MONAGHAN1997A: case SPH_VISC_MONAGHAN1997B: case SPH_VISC_DUKOWICZ:
        case SPH_VISC_PRICE2012_98: case SPH_VISC_PRICE2012: case SPH_VISC_PRICE2008: case SPH_VISC_WADSLEY2008:
            mu = mu0; sf = 1.f; break;
        case SPH_VISC_MONAGHAN1992: mu = mu0 * sfac; sf = 1.f * sfac; break;
        default: mu = mu0 * sfac; sf = h_bar / xi; break;      // Default, MonaghanGingold1983, DeltaSPH
    }
    // compute_bars (util.py:40-134)
    bool ub_rho = true, ub_c = true, ub_h = true;
    if (term == SPH_VISC_CLEARY1998) { ub_rho = false; ub_c = false; ub_h = false; }
    else if (term == SPH_VISC_MONAGHAN1992) { ub_c = false; }
    else if (term == SPH_VISC_DELTASPH) { ub_rho = false; }
    const float rho = ub_rho ? rho_bar : (useJ ? rhoj : rhoi);
    const float c = ub_c ? c_bar : (useJ ? cj : ci);
    const float h = ub_h ? h_bar : (useJ ? hj : hi);
    float v_sig = 0.f;
    switch (term) {
        case SPH_VISC_MONAGHANGINGOLD1983: v_sig = c; break;
        case SPH_VISC_CLEARY1998: {
            const float f = 1.f / (2.f * ((float)dim + 2.f));
            const float mi = f * ai * C_l * hi * ci * rhoi / xi, mj = f * aj * C_l * hj * cj * rhoj / xi;
            v_sig = 19.8f * mi * mj / (rhoi * rhoj * (mi + mj)) / (r + 1e-14f * h);
            break;
        }
        case SPH_VISC_MONAGHAN1992: case SPH_VISC_MONAGHAN1997A: case SPH_VISC_PRICE2012_98: v_sig = C_l * c - C_q * mu; break;
        case SPH_VISC_MONAGHAN1997B: v_sig = safe_sqrt(ci * ci + C_q * mu * mu) + safe_sqrt(cj * cj + C_q * mu * mu) - mu; break;
        case SPH_VISC_DUKOWICZ: v_sig = C_l * c - 3.f / 4.f * C_q * mu; break;
        case SPH_VISC_PRICE2012: v_sig = C_l * c - C_q / 2.f * mu; break;
        case SPH_VISC_PRICE2008: {
            const float pi_ = explicitP ? Pi_ : rhoi * ci * ci, pj_ = explicitP ? Pj_ : rhoj * cj * cj;
            v_sig = C_l * safe_sqrt(fabsf(pi_ - pj_) / ((rhoi + rhoj) / 2.f + 1e-14f * h));
            break;
        }
        case SPH_VISC_WADSLEY2008: v_sig = C_l * fabsf(mu); break;
        default: v_sig = C_l * c - C_q * mu; break;          // DeltaSPH, Default
    }
    float val = rhoj * 1.f / rho * v_sig * sf;
    if (P.monaghan_switch && !thermal && ux > 0.f) val = 0.f;
    return val;
}

}  // namespace wsph
