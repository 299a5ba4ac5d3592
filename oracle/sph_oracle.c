/*
 * sph_oracle.c -- CPU oracle for the warpSPH per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the algorithms of the
 * reference (wi-re/warpSPH) that the CUDA library implements, so that tests can
 * check the GPU results.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product path never does.
 *
 * Precision: compiled twice, with REAL=float (liboracle32.so) and REAL=double
 * (liboracle64.so).  The neighbour search always runs in float with explicitly
 * ordered operations (no FMA contraction: built with -ffp-contract=off), so its
 * permutation and CSR lists are bit-identical to the GPU's.
 *
 * Parity status: the reference-resident arithmetic (pair bodies of
 * modules/crk/accel.py, modules/crk/dudt.py, modules/crk/limiter.py,
 * modules/compSPH/balance.py, modules/shockCapturing (CullenDehnen2010.py, wp_vsig.py), modules/eos/idealGas.py,
 * modules/timestep/compressible.py, modules/compSPH/multistep.py) is pinned by the
 * golden vectors in tests/golden (generated by executing the reference's own
 * Python source, see tests/golden/make_golden.py).  The parts that live in the
 * absent warpSPHCore / warpSPHIntegrators packages (kernel functions, neighbour
 * search, CRK coefficients, generic SPH operators, Runge-Kutta bookkeeping) are
 * restated from the published methods; for those, parity with the reference is
 * unpinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "../include/warpsph_b200.h"

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

#define PI_R ((real)3.14159265358979323846)

static inline real wmin(real a, real b) { return a < b ? a : b; }   /* Warp builtin min */
static inline real wmax(real a, real b) { return a > b ? a : b; }   /* Warp builtin max */
static inline real rsqrt_safe(real x) { return (real)sqrt((double)(x > 0 ? x : 0)); }
#if defined(ORACLE_FLOAT)
#define SQRT sqrtf
#define EXP expf
#define POW powf
#define FABS fabsf
#define FLOOR floorf
#define ACOS acosf
#else
#define SQRT sqrt
#define EXP exp
#define POW pow
#define FABS fabs
#define FLOOR floor
#define ACOS acos
#endif

/* ------------------------------------------------------------------ parameters */
typedef struct {
    int dim, kernel;
    real dmin[3], dmax[3], L[3], halfL[3];
    int periodic[3];
    real vs;
    real C_l, C_q;
    real eta_crit, eta_fold;
    int crk_lim, vl, vl_off, vl_on;
    real gamma;
    int energy_scheme, limit_xi, kahan, correct_grad_v;
    real alpha_min, alpha_max, beta_xi;
    real target_neighbors;
    real cfl, min_dt, max_dt, dt_growth;
    real kscale, kxi;
    real Cu_l, Cu_q, c_s, beta_c, beta_d;
    int visc_term, cond_term, mswitch, correct_xi, scale_beta;
} OP;

/* Kernel scale H/h: Dehnen & Aly (2012) Table 1 for the Wendland kernels; for B7 the
 * factor of the reference's CFL step as its notebooks print it (1D Woodward-Colella, 2D
 * Gresho-Chan; 3D by the quintic spline's moment ratio sqrt(15/14) from 1D). */
static double kscale_tab(int kernel, int dim) {
    static const double t[4][3] = {{1.620185175, 1.897366596, 1.936491673},
                                   {1.936491673, 2.171240593, 2.207940217},
                                   {2.207940217, 2.415229458, 2.449489743},
                                   {3.865656972, 3.932734728, 4.001335111}};
    return t[kernel - 1][dim - 1];
}

static OP op_from(const SphParams* p) {
    OP o;
    memset(&o, 0, sizeof(o));
    o.dim = p->dim; o.kernel = p->kernel;
    for (int a = 0; a < 3; ++a) {
        /* float first: identical domain constants to the GPU's float parameters */
        float mn = (float)p->domain_min[a], mx = (float)p->domain_max[a], L = (float)(p->domain_max[a] - p->domain_min[a]);
        o.dmin[a] = (real)mn; o.dmax[a] = (real)mx; o.L[a] = (real)L; o.halfL[a] = (real)(0.5f * L);
        o.periodic[a] = p->periodic[a] ? 1 : 0;
    }
    o.vs = (real)p->verlet_scale;
    o.C_l = (real)p->C_l; o.C_q = (real)p->C_q;
    o.eta_crit = (real)p->eta_crit; o.eta_fold = (real)p->eta_fold;
    o.crk_lim = p->enable_crk_limiter; o.vl = p->enable_vanleer_limiter; o.vl_off = p->force_vanleer_off; o.vl_on = p->force_vanleer_on;
    o.gamma = (real)p->gamma; o.energy_scheme = p->energy_scheme; o.limit_xi = p->limit_xi; o.kahan = p->kahan;
    o.correct_grad_v = p->correct_velocity_gradient;
    o.alpha_min = (real)p->alpha_min; o.alpha_max = (real)p->alpha_max; o.beta_xi = (real)p->beta_xi;
    o.target_neighbors = (real)p->target_neighbors;
    o.cfl = (real)p->cfl; o.min_dt = (real)p->min_dt; o.max_dt = (real)p->max_dt; o.dt_growth = (real)p->dt_growth;
    o.kscale = (real)kscale_tab(p->kernel, p->dim);
    o.kxi = o.kscale;
    o.Cu_l = (real)p->Cu_l; o.Cu_q = (real)p->Cu_q; o.c_s = (real)p->c_s;
    o.beta_c = (real)p->beta_c; o.beta_d = (real)p->beta_d;
    o.visc_term = p->viscosity_term; o.cond_term = p->conductivity_term;
    o.mswitch = p->monaghan_switch; o.correct_xi = p->correct_xi; o.scale_beta = p->scale_beta;
    return o;
}

/* ------------------------------------------------------------------ kernels
 * Wendland (1995) functions with support radius H, q = r/H, normalisations C_d
 * (Dehnen & Aly 2012):  W = C_d/H^d k(q),  dk/dq = -q p(q).
 * B7 (K = 4): the degree-7 B-spline k(q) = sum_j c_j (a_j - q)_+^7, a = 1, 3/4, 1/2, 1/4,
 * c = 1, -8, 28, -56; p = -k'/q, from the expanded polynomial below q = 1/4 (where the
 * constant term of k' cancels) and from the truncated powers above. */
static real tpow(real a, real q, int n) {
    real t = a - q, r = t;
    if (!(t > 0)) return 0;
    for (int i = 1; i < n; ++i) r *= t;
    return r;
}
static real kernel_C(int K, int D) {
    if (K == 4) return D == 1 ? (real)(4096.0 / 315.0) : (D == 2 ? (real)(589824.0 / (7435.0 * 3.14159265358979323846))
                                                              : (real)(16384.0 / (105.0 * 3.14159265358979323846)));
    if (K == 1) return D == 1 ? (real)1.25 : (D == 2 ? (real)(7.0 / 3.14159265358979323846) : (real)(21.0 / (2.0 * 3.14159265358979323846)));
    if (K == 2) return D == 1 ? (real)1.5 : (D == 2 ? (real)(9.0 / 3.14159265358979323846) : (real)(495.0 / (32.0 * 3.14159265358979323846)));
    return D == 1 ? (real)1.71875 : (D == 2 ? (real)(78.0 / (7.0 * 3.14159265358979323846)) : (real)(1365.0 / (64.0 * 3.14159265358979323846)));
}
static void kernel_kp(int K, int D, real q, real* k, real* p) {
    real t = 1 - q;
    if (K == 4) {
        *k = tpow(1, q, 7) - 8 * tpow((real)0.75, q, 7) + 28 * tpow((real)0.5, q, 7) - 56 * tpow((real)0.25, q, 7);
        if (q < (real)0.25) {
            real q2 = q * q;
            *p = (real)3.28125 + q2 * ((real)-35 + q2 * ((real)210 - (real)245 * q));
        } else {
            *p = 7 * (tpow(1, q, 6) - 8 * tpow((real)0.75, q, 6) + 28 * tpow((real)0.5, q, 6)) / q;
        }
        (void)D;
    } else if (K == 1) {
        if (D == 1) { real t2 = t * t; *k = t2 * t * (1 + 3 * q); *p = 12 * t2; }
        else { real t3 = t * t * t; *k = t3 * t * (1 + 4 * q); *p = 20 * t3; }
    } else if (K == 2) {
        if (D == 1) { real t4 = (t * t) * (t * t); *k = t4 * t * (1 + 5 * q + 8 * q * q); *p = 14 * (1 + 4 * q) * t4; }
        else { real t5 = (t * t) * (t * t) * t; *k = t5 * t * (1 + 6 * q + ((real)35 / (real)3) * q * q); *p = ((real)56 / (real)3) * (1 + 5 * q) * t5; }
    } else {
        if (D == 1) { real t6 = (t * t) * (t * t) * (t * t); *k = t6 * t * (1 + 7 * q + 19 * q * q + 21 * q * q * q); *p = 6 * (3 + 18 * q + 35 * q * q) * t6; }
        else { real t7 = (t * t) * (t * t) * (t * t) * t; *k = t7 * t * (1 + 8 * q + 25 * q * q + 32 * q * q * q); *p = 22 * (1 + 7 * q + 16 * q * q) * t7; }
    }
}
static real ipowD(real h, int D) { return D == 1 ? h : (D == 2 ? h * h : h * h * h); }

static real kW(const OP* o, real r, real H) {
    real q = r / H;
    if (!(q < 1)) return 0;
    real k, p; kernel_kp(o->kernel, o->dim, q, &k, &p);
    return kernel_C(o->kernel, o->dim) / ipowD(H, o->dim) * k;
}
static void kWG(const OP* o, const real* x, real r, real H, real* W, real* g) {
    real q = r / H;
    int D = o->dim;
    if (!(q < 1)) { *W = 0; for (int a = 0; a < D; ++a) g[a] = 0; return; }
    real k, p; kernel_kp(o->kernel, D, q, &k, &p);
    real cH = kernel_C(o->kernel, D) / ipowD(H, D);
    *W = cH * k;
    real s = -cH * p / (H * H);
    for (int a = 0; a < D; ++a) g[a] = s * x[a];
}
static void kWdH(const OP* o, real r, real H, real* W, real* dWdH) {
    real q = r / H;
    int D = o->dim;
    if (!(q < 1)) { *W = 0; *dWdH = 0; return; }
    real k, p; kernel_kp(o->kernel, D, q, &k, &p);
    real cH = kernel_C(o->kernel, D) / ipowD(H, D);
    *W = cH * k;
    *dWdH = -cH / H * ((real)D * k - q * q * p);
}
static real kW_mode(const OP* o, real r, real Hi, real Hj, int mode) {
    switch (mode) {
        case SPH_SUPPORT_GATHER: return kW(o, r, Hi);
        case SPH_SUPPORT_SCATTER: return kW(o, r, Hj);
        case SPH_SUPPORT_SYMMETRIC: return kW(o, r, (real)0.5 * (Hi + Hj));
        case SPH_SUPPORT_SUPERSYMMETRIC: return kW(o, r, wmax(Hi, Hj));
        default: return (real)0.5 * (kW(o, r, Hi) + kW(o, r, Hj));
    }
}

/* minimum-image x_ij = x_i - x_j (warpSPHCore computeDistanceVec, restated) */
static void dist_vec(const OP* o, const real* xi, const real* xj, real* d) {
    for (int a = 0; a < o->dim; ++a) {
        real v = xi[a] - xj[a];
        if (o->periodic[a]) {
            if (v > o->halfL[a]) v = v - o->L[a];
            else if (v < -o->halfL[a]) v = v + o->L[a];
        }
        d[a] = v;
    }
}
static real dotD(const real* a, const real* b, int D) { real s = a[0] * b[0]; for (int k = 1; k < D; ++k) s += a[k] * b[k]; return s; }

/* CRK corrected gradient (Frontiere, Raskin & Owen 2017); gB[a*D+g] = dB^a/dx^g */
static void crk_grad(int D, const real* x, real W, const real* gW, real A, const real* B, const real* gA, const real* gB, real* out) {
    real bx = 1 + dotD(B, x, D);
    for (int g = 0; g < D; ++g) {
        real gbx = gB[0 * D + g] * x[0];
        for (int a = 1; a < D; ++a) gbx += gB[a * D + g] * x[a];
        out[g] = A * bx * gW[g] + A * B[g] * W + gA[g] * bx * W + A * gbx * W;
    }
}

/* ------------------------------------------------------------------ neighbour search (float) */
static uint32_t spread2(uint32_t x) {
    x &= 0x0000ffffu; x = (x | (x << 8)) & 0x00ff00ffu; x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u; x = (x | (x << 1)) & 0x55555555u; return x;
}
static uint32_t spread3(uint32_t x) {
    x &= 0x000003ffu; x = (x | (x << 16)) & 0x030000ffu; x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u; x = (x | (x << 2)) & 0x09249249u; return x;
}
static uint32_t morton(int D, const int* c) {
    if (D == 1) return (uint32_t)c[0];
    if (D == 2) return spread2((uint32_t)c[0]) | (spread2((uint32_t)c[1]) << 1);
    return spread3((uint32_t)c[0]) | (spread3((uint32_t)c[1]) << 1) | (spread3((uint32_t)c[2]) << 2);
}
static int max_bits_for(int dim, int64_t cap) {
    int lb = 0;
    while (((int64_t)1 << (lb + 1)) <= cap) ++lb;
    int mb = lb / dim;
    int lim = dim == 1 ? 30 : (dim == 2 ? 16 : 10);
    return mb > lim ? lim : mb;
}

typedef struct { int G[3]; float inv[3]; float dmin[3], L[3], halfL[3]; int periodic[3]; } NGrid;

static void cell_coords_f(const NGrid* g, int D, const float* x, int* c) {
    for (int a = 0; a < D; ++a) {
        float t = (x[a] - g->dmin[a]) * g->inv[a];
        int ci = (int)floorf(t);
        c[a] = ci < 0 ? 0 : (ci >= g->G[a] ? g->G[a] - 1 : ci);
    }
}

/* Verlet list, same definition and canonical order as the GPU (see header).  With
 * inter_counts, each row holds its interacting entries (fl(sqrt(r^2))/max(H_i,H_j) < 1)
 * first and the rest after them, both in walk order; inter_counts[i] is the prefix length. */
int oracle_neighbors_build(const SphParams* p, int64_t n, const float* x, const float* H, int64_t cell_capacity,
                           int32_t* sort_index, uint32_t* sorted_keys, int32_t* grid_out,
                           int32_t* offsets, int32_t* counts, int32_t* inter_counts, int32_t* list, int64_t list_capacity,
                           int64_t* nnz_out) {
    int D = p->dim;
    NGrid g;
    memset(&g, 0, sizeof(g));
    float Lmax = 0.f, hmax = 0.f;
    for (int a = 0; a < 3; ++a) {
        g.dmin[a] = (float)p->domain_min[a];
        g.L[a] = (float)(p->domain_max[a] - p->domain_min[a]);
        g.halfL[a] = 0.5f * g.L[a];
        g.periodic[a] = p->periodic[a] ? 1 : 0;
        g.G[a] = 1;
    }
    for (int a = 0; a < D; ++a) Lmax = fmaxf(Lmax, g.L[a]);
    for (int64_t i = 0; i < n; ++i) hmax = fmaxf(hmax, H[i]);
    float vs = (float)p->verlet_scale;
    float cell = (vs * hmax) * 1.001f + Lmax * 1e-6f;
    int mb = max_bits_for(D, cell_capacity);
    int bits[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) {
        float f = floorf(g.L[a] / cell);
        int gmax = 1 << mb;
        int gi = (f >= (float)gmax) ? gmax : (f < 1.f ? 1 : (int)f);
        int b = 0;
        while ((1 << b) < gi) ++b;
        g.G[a] = gi; bits[a] = b;
        g.inv[a] = (float)gi / g.L[a];
    }
    if (grid_out) {
        for (int a = 0; a < 3; ++a) { grid_out[a] = g.G[a]; grid_out[3 + a] = bits[a]; }
        memcpy(&grid_out[6], &cell, 4);
        grid_out[7] = D;
    }
    int64_t ncells = (int64_t)1 << (mb * D);
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* begin = (int32_t*)calloc((size_t)ncells + 1, sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) {
        int c[3];
        cell_coords_f(&g, D, x + i * D, c);
        keys[i] = morton(D, c);
        begin[keys[i] + 1]++;
    }
    for (int64_t c = 0; c < ncells; ++c) begin[c + 1] += begin[c];
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)ncells);
    memcpy(cur, begin, sizeof(int32_t) * (size_t)ncells);
    for (int64_t i = 0; i < n; ++i) sort_index[cur[keys[i]]++] = (int32_t)i;   /* stable */
    for (int64_t k = 0; k < n; ++k) sorted_keys[k] = keys[sort_index[k]];

    int64_t total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            total = 0;
            for (int64_t i = 0; i < n; ++i) { offsets[i] = (int32_t)total; total += counts[i]; }
            *nnz_out = total;
            if (total > list_capacity) break;
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const float* xi = x + i * D;
            float Hi = H[i];
            int c[3];
            cell_coords_f(&g, D, xi, c);
            /* stencil cells in offset order (x fastest), duplicates (grids with fewer
             * than three cells along a periodic axis) visited once */
            uint32_t sk[27];
            int nk = 0;
            int NS = D == 1 ? 3 : (D == 2 ? 9 : 27);
            for (int s = 0; s < NS; ++s) {
                int o[3] = {s % 3 - 1, (s / 3) % 3 - 1, (s / 9) % 3 - 1};
                int cc[3];
                int ok = 1;
                for (int a = 0; a < D; ++a) {
                    int v = c[a] + o[a];
                    if (v < 0 || v >= g.G[a]) {
                        if (g.periodic[a]) v = (v + g.G[a]) % g.G[a]; else ok = 0;
                    }
                    cc[a] = v;
                }
                if (!ok) continue;
                uint32_t kk = morton(D, cc);
                int dup = 0;
                for (int q = 0; q < nk; ++q) if (sk[q] == kk) { dup = 1; break; }
                if (dup) continue;
                sk[nk++] = kk;
            }
            int cntv = 0, icntv = 0, restv = 0;
            int32_t base = pass ? offsets[i] : 0;
            int32_t tail = (pass && inter_counts) ? base + inter_counts[i] : base;
            for (int q = 0; q < nk; ++q) {
                for (int32_t k = begin[sk[q]]; k < begin[sk[q] + 1]; ++k) {
                    int32_t j = sort_index[k];
                    const float* xj = x + (int64_t)j * D;
                    float Hm = fmaxf(Hi, H[j]);
                    float R = vs * Hm;
                    float r2 = 0.f;
                    for (int a = 0; a < D; ++a) {
                        float d = xi[a] - xj[a];
                        if (g.periodic[a]) {
                            if (d > g.halfL[a]) d = d - g.L[a];
                            else if (d < -g.halfL[a]) d = d + g.L[a];
                        }
                        r2 = a == 0 ? d * d : r2 + d * d;
                    }
                    if (r2 < R * R) {
                        int inter = inter_counts && (sqrtf(r2) / Hm < 1.0f);
                        if (pass) {
                            if (inter) list[base + icntv] = j;
                            else list[tail + restv] = j;
                        }
                        icntv += inter;
                        restv += !inter;
                        ++cntv;
                    }
                }
            }
            if (!pass) { counts[i] = cntv; if (inter_counts) inter_counts[i] = icntv; }
        }
    }
    free(keys); free(begin); free(cur);
    return 0;
}

/* ------------------------------------------------------------------ density (modules/density/density.py:16-28) */
int oracle_density(const SphParams* p, int64_t n, int mode, const real* x, const real* H, const real* m,
                   const int32_t* offs, const int32_t* cnt, const int32_t* list, real* rho) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            s += m[j] * kW_mode(&o, rsqrt_safe(dotD(d, d, D)), H[i], H[j], mode);
        }
        rho[i] = s;
    }
    return 0;
}

/* ------------------------------------------------------------------ adaptive support
 * modules/adaptiveSupport/optimalSupportMonaghan.py:52-59 (computeH/F) and :87-125 (Newton step),
 * modules/adaptiveSupport/wp_omega.py:40-60 (Omega = 1 - sum dh/drho m_j dW/dh),
 * utils/support.py:24-44 (volumeToSupportHelper). */
static real volume_to_support(real V, real nH, int D) {
    if (D == 1) return nH * V / 2;
    if (D == 2) return SQRT(nH * V / PI_R);
    return POW(nH * V / PI_R * 3 / 4, (real)1 / (real)3);
}
int oracle_adaptive_h_iter(const SphParams* p, int64_t n, const real* x, const real* H, const real* m,
                           const int32_t* offs, const int32_t* cnt, const int32_t* list, const real* hb,
                           real* rho_out, real* H_out, real* ratio) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real rs = 0, ds = 0, Hi = H[i];
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real W, dWdH;
            kWdH(&o, rsqrt_safe(dotD(d, d, D)), Hi, &W, &dWdH);
            rs += m[j] * W;
            ds += m[j] * dWdH;
        }
        real rho = rs;
        real safe_rho = isfinite(rho) ? (rho > (real)1e-12 ? rho : (real)1e-12) : 1;
        real F = Hi - volume_to_support(m[i] / safe_rho, o.target_neighbors, D);
        real dh_drho = -Hi / (rho * (real)D);
        real omega = 1 - dh_drho * ds;
        if (!isfinite(omega)) omega = 0;
        real step = F / (omega + (real)1e-6);
        if (!isfinite(step)) step = 0;
        real hn = Hi - step;
        if (!isfinite(hn)) hn = Hi;
        real lo = hb[0] * (real)0.25, hi = hb[1] * 4;
        hn = hn < lo ? lo : (hn > hi ? hi : hn);
        rho_out[i] = rho; H_out[i] = hn;
        if (ratio) ratio[i] = hn / (Hi + (real)1e-6);
    }
    return 0;
}

/* ------------------------------------------------------------------ CRK volume and coefficients
 * warpSPHCore crk_volume / crk_moments / crk_density (called via computeCRKFactors,
 * schemes/crkSPH.py:61), restated from Frontiere, Raskin & Owen 2017. */
/* Owen adaptive support, one iteration (modules/adaptiveSupport/optimalSupportOwen.py:70-108,
 * wp_psi0.py:46-98 gather support, owenLUT.py:6-12 lookup in FP64, the update of :27-33). */
int oracle_owen_iter(const SphParams* p, int64_t n, const real* x, const real* H, const int32_t* offs, const int32_t* cnt,
                     const int32_t* list, const double* lut_nh, const double* lut_psiH, int nlut, double target, const real* hb,
                     real* psi0_out, real* psiH_out, real* H_out, real* ratio_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real hi = H[i];
        real hsW = (real)1 / POW(hi, -(real)D), hsG = (real)1 / POW(hi, -(real)(D + 1));
        real sW = 0, sG = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), hi, &W, g);
            sW += hsW * W;
            sG += hsG * rsqrt_safe(dotD(g, g, D));
        }
        real psi0 = POW(sW, (real)1 / (real)D), psiH = POW(sG, (real)1 / (real)D);
        double xv = (double)psiH;
        int cntle = 0;                                   /* searchsorted(right=True) */
        while (cntle < nlut && lut_psiH[cntle] <= xv) ++cntle;
        int il = cntle - 1;
        il = il < 0 ? 0 : (il > nlut - 2 ? nlut - 2 : il);
        double alpha = (xv - lut_psiH[il]) / (lut_psiH[il + 1] - lut_psiH[il]);
        alpha = alpha < 0 ? 0 : (alpha > 1 ? 1 : alpha);
        real nh = (real)(lut_nh[il] * (1 - alpha) + lut_nh[il + 1] * alpha);
        real sv = (real)target / nh;
        real a = sv >= 1 ? (real)0.4 * (1 + POW(sv, (real)-3)) : (real)0.4 * (1 + POW(sv, (real)2));
        real hn = (1 - a + a * sv) * hi;
        real lo = hb[0] * (real)0.25, up = hb[1] * (real)4;
        hn = hn < lo ? lo : (hn > up ? up : hn);
        if (psi0_out) psi0_out[i] = psi0;
        if (psiH_out) psiH_out[i] = psiH;
        H_out[i] = hn;
        if (ratio_out) ratio_out[i] = hn / hi;
    }
    return 0;
}

int oracle_crk_volume(const SphParams* p, int64_t n, const real* x, const real* H, const int32_t* offs, const int32_t* cnt,
                      const int32_t* list, real* V) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            s += kW(&o, rsqrt_safe(dotD(d, d, D)), H[j]);
        }
        V[i] = 1 / s;
    }
    return 0;
}

static double inv_sym(int D, const double* a, double* r) {
    if (D == 1) { r[0] = 1.0 / a[0]; return a[0]; }
    if (D == 2) {
        double det = a[0] * a[3] - a[1] * a[2], id = 1.0 / det;
        r[0] = a[3] * id; r[3] = a[0] * id; r[1] = -a[1] * id; r[2] = -a[2] * id;
        return det;
    }
    double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    double det = a[0] * c00 + a[1] * c01 + a[2] * c02, id = 1.0 / det;
    r[0] = c00 * id; r[1] = (a[2] * a[7] - a[1] * a[8]) * id; r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    r[3] = c01 * id; r[4] = (a[0] * a[8] - a[2] * a[6]) * id; r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    r[6] = c02 * id; r[7] = (a[1] * a[6] - a[0] * a[7]) * id; r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return det;
}

int oracle_crk_factors(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* V,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list,
                       real* Aout, real* Bout, real* gAout, real* gBout, real* rho_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real m0 = 0, s0 = 0, m1[3] = {0}, s1[3] = {0}, m2[9] = {0}, dm0[3] = {0}, dm1[9] = {0}, dm2[27] = {0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], gW[3], W;
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[j], &W, gW);
            if (W == 0) continue;
            real Vj = V[j], VW = Vj * W;
            m0 += VW; s0 += m[j] * W;
            for (int a = 0; a < D; ++a) {
                m1[a] += VW * d[a];
                s1[a] += m[j] * W * d[a];
                dm0[a] += Vj * gW[a];
                for (int c = 0; c < D; ++c) {
                    m2[a * D + c] += VW * d[a] * d[c];
                    dm1[a * D + c] += Vj * (d[a] * gW[c] + (a == c ? W : 0));
                }
            }
            for (int a = 0; a < D; ++a)
                for (int c = a; c < D; ++c)
                    for (int g2 = 0; g2 < D; ++g2)
                        dm2[(a * D + c) * D + g2] += Vj * (d[a] * d[c] * gW[g2] + ((a == g2 ? d[c] : 0) + (c == g2 ? d[a] : 0)) * W);
        }
        double M2[9], Mi[9], tr = 0;
        for (int a = 0; a < D; ++a) { for (int c = 0; c < D; ++c) M2[a * D + c] = (double)(a <= c ? m2[a * D + c] : m2[c * D + a]); tr += M2[a * D + a]; }
        double det = inv_sym(D, M2, Mi);
        double sc = tr / D, sD = sc;
        for (int a = 1; a < D; ++a) sD *= sc;
        int ok = isfinite(det) && fabs(det) > 1e-10 * fabs(sD) && m0 > 0;
        double A, Bv[3], gA[3], gB[9];
        if (ok) {
            double mb = (double)m0;
            for (int a = 0; a < D; ++a) { double t = 0; for (int c = 0; c < D; ++c) t -= Mi[a * D + c] * (double)m1[c]; Bv[a] = t; }
            for (int a = 0; a < D; ++a) mb += (double)m1[a] * Bv[a];
            A = 1.0 / mb;
            for (int g2 = 0; g2 < D; ++g2) {
                double rhs[3];
                for (int a = 0; a < D; ++a) {
                    double t = (double)dm1[a * D + g2];
                    for (int c = 0; c < D; ++c) t += (double)(a <= c ? dm2[(a * D + c) * D + g2] : dm2[(c * D + a) * D + g2]) * Bv[c];
                    rhs[a] = t;
                }
                for (int a = 0; a < D; ++a) { double t = 0; for (int c = 0; c < D; ++c) t -= Mi[a * D + c] * rhs[c]; gB[a * D + g2] = t; }
            }
            for (int g2 = 0; g2 < D; ++g2) {
                double t = (double)dm0[g2];
                for (int a = 0; a < D; ++a) t += (double)dm1[a * D + g2] * Bv[a] + (double)m1[a] * gB[a * D + g2];
                gA[g2] = -A * A * t;
            }
        } else {
            double m0d = (double)m0;
            A = 1.0 / m0d;
            for (int a = 0; a < D; ++a) { Bv[a] = 0; gA[a] = -(double)dm0[a] / (m0d * m0d); for (int c = 0; c < D; ++c) gB[a * D + c] = 0; }
        }
        double rho = (double)s0;
        for (int a = 0; a < D; ++a) rho += Bv[a] * (double)s1[a];
        rho *= A;
        Aout[i] = (real)A;
        for (int a = 0; a < D; ++a) {
            Bout[i * D + a] = (real)Bv[a]; gAout[i * D + a] = (real)gA[a];
            for (int c = 0; c < D; ++c) gBout[i * D * D + a * D + c] = (real)gB[a * D + c];
        }
        if (rho_out) rho_out[i] = (real)rho;
    }
    return 0;
}

/* ------------------------------------------------------------------ EOS (modules/eos/idealGas.py:16-36, u and rho given) */
int oracle_eos_ideal_gas(const SphParams* p, int64_t n, const real* u, const real* rho, real* A, real* P, real* c) {
    real g = (real)p->gamma;
    for (int64_t i = 0; i < n; ++i) {
        if (c) c[i] = SQRT(FABS(u[i]) * g * (g - 1));
        if (P) P[i] = (g - 1) * rho[i] * u[i];
        if (A) A[i] = u[i] * (g - 1) * POW(rho[i], 1 - g);
    }
    return 0;
}

/* ------------------------------------------------------------------ velocity gradient, Cullen div, v_sig
 * schemes/crkSPH.py:158-172 (CRK difference gradient, scatter, then .mT),
 * modules/shockCapturing/CullenDehnen2010.py:246-257 (divergence, super-symmetric),
 * modules/shockCapturing/wp_vsig.py:55-90 (signal velocity max-reduction). */
int oracle_grad_v(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                  const real* V, const real* A, const real* B, const real* gA, const real* gB, const real* v, const real* c,
                  const int32_t* offs, const int32_t* cnt, const int32_t* list,
                  real* DvDx, real* drhodt, real* div_out, real* vsig_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real G[9] = {0}, div = 0, vsig = 0;
        const real* vi = v + i * D;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], gW[3], W, gR[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            const real* vj = v + (int64_t)j * D;
            kWG(&o, d, r, H[j], &W, gW);
            if (W != 0) {
                crk_grad(D, d, W, gW, A[i], B + i * D, gA + i * D, gB + i * D * D, gR);
                for (int a = 0; a < D; ++a) {
                    real dv = V[j] * (vj[a] - vi[a]);
                    for (int g2 = 0; g2 < D; ++g2) G[a * D + g2] += dv * gR[g2];
                }
            }
            if (div_out) {
                real Hs = wmax(H[i], H[j]);
                if (r < Hs) {
                    real W2, g2v[3];
                    kWG(&o, d, r, Hs, &W2, g2v);
                    real vol = m[j] / rho[j], s = 0;
                    for (int a = 0; a < D; ++a) s += (vj[a] - vi[a]) * g2v[a];
                    div += vol * s;
                }
                if (r < o.vs * Hs) {
                    real mu = 0;
                    for (int a = 0; a < D; ++a) mu += (vi[a] - vj[a]) * d[a];
                    mu = mu / (r + (real)1e-14 * H[i]);
                    real vsv = (real)0.5 * (c[i] + c[j]) - mu;
                    if (mu > 0) vsv = 0;
                    vsig = wmax(vsig, vsv);
                }
            }
        }
        for (int q = 0; q < D * D; ++q) DvDx[i * D * D + q] = G[q];
        if (drhodt) { real tr = 0; for (int a = 0; a < D; ++a) tr += G[a * D + a]; drhodt[i] = -tr * rho[i]; }
        if (div_out) { div_out[i] = div; if (vsig_out) vsig_out[i] = FABS(vsig); }
    }
    return 0;
}

/* ------------------------------------------------------------------ Cullen & Dehnen switch
 * modules/shockCapturing/CullenDehnen2010.py:121-164 (R), :166-191 (Xi), :281-314 (alpha update). */
int oracle_switch_cullen(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                         const real* div, const real* div_prev, const real* vsig, const real* alpha0_prev, real dt,
                         const int32_t* offs, const int32_t* cnt, const int32_t* list, real* alpha_out, real* R_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0, Hi = H[i];
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real W = kW(&o, rsqrt_safe(dotD(d, d, D)), Hi);
            if (W == 0) continue;
            real sg = div[j] > 0 ? 1 : (div[j] < 0 ? -1 : 0);
            s += m[j] / rho[j] * (rho[j] * sg) * W;
        }
        real R = 1 / rho[i] * s;
        real omr = 1 - R, omr2 = omr * omr;
        real nom = o.beta_xi * (omr2 * omr2) * div[i];
        real Xi = o.limit_xi ? (nom * nom + (real)1e-14 * Hi) / (nom * nom + 0 + (real)1e-14 * Hi)
                             : (nom * nom) / (nom * nom + 0 + (real)1e-14 * Hi);
        real ddiv = (div[i] - div_prev[i]) / dt;
        real Ai = Xi * (-ddiv > 0 ? -ddiv : 0);
        real vs = vsig[i];
        real scaling = Hi * Hi * Ai / (vs * vs + Hi * Hi * Ai + (real)1e-14 * Hi);
        real al = o.alpha_max * scaling;
        al = al < o.alpha_min ? o.alpha_min : (al > o.alpha_max ? o.alpha_max : al);
        real a0 = alpha0_prev[i];
        real tau = Hi * (1 / o.kxi) / (2 * (real)0.05 * vs);
        real adot = (al - a0) / tau;
        a0 = al > a0 ? al : a0;
        a0 = al < a0 ? a0 + adot * dt : a0;
        a0 = a0 < o.alpha_min ? o.alpha_min : (a0 > o.alpha_max ? o.alpha_max : a0);
        alpha_out[i] = a0;
        if (R_out) R_out[i] = R;
    }
    return 0;
}

/* Signal velocity over the Verlet set (modules/shockCapturing/wp_vsig.py:11-90): max_j of
 * c_bar - mu_ij for approaching pairs with r < verletScale * max(H_i, H_j), absolute value. */
int oracle_vsig(const SphParams* p, int64_t n, const real* x, const real* H, const real* v, const real* c,
                const int32_t* offs, const int32_t* cnt, const int32_t* list, real* vsig_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real vsig = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            if (!(r < o.vs * wmax(H[i], H[j]))) continue;
            real mu = 0;
            for (int a = 0; a < D; ++a) mu += (v[i * D + a] - v[(int64_t)j * D + a]) * d[a];
            mu = mu / (r + (real)1e-14 * H[i]);
            real vsv = (real)0.5 * (c[i] + c[j]) - mu;
            if (mu > 0) vsv = 0;
            vsig = wmax(vsig, vsv);
        }
        vsig_out[i] = FABS(vsig);
    }
    return 0;
}

/* CRKSPH moment matrix of the velocity-gradient correction (common.py:10-25 negating
 * wp_computeM.py:55-86): M_i = -sum_j m_j x_ij (x) grad W(r_ij, H_i), gather support,
 * row-major D x D per particle. */
int oracle_moment_matrix(const SphParams* p, int64_t n, const real* x, const real* H, const real* m,
                         const int32_t* offs, const int32_t* cnt, const int32_t* list, real* M_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real M[9] = {0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], &W, g);
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) M[a * D + b] += m[j] * d[a] * g[b];
        }
        for (int a = 0; a < D * D; ++a) M_out[i * D * D + a] = -M[a];
    }
    return 0;
}

/* Cullen-Hopkins switch (modules/shockCapturing/CullenHopkins.py:7-149).  The velocity
 * gradient is warpSPHCore's difference gradient with gather support, restated as
 * sum_j m_j/rho_j (v_j - v_i) (x) grad W(r_ij, H_i).  With correctVelocityGradient the
 * caller passes Minv = pinv(M) (row-major D x D per particle) and the gradient becomes
 * Minv V before its trace and shear are taken (common.py:76-78); NULL leaves it as is. */
int oracle_switch_hopkins_terms(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                                const real* v, const real* alpha0, const int32_t* offs, const int32_t* cnt,
                                const int32_t* list, const real* Minv, real* div_out, real* shear2_out, real* alpha_out,
                                real* R_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real G[9] = {0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], &W, g);
            if (W == 0) continue;
            real Vj = m[j] / rho[j];
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) G[a * D + b] += Vj * (v[(int64_t)j * D + a] - v[i * D + a]) * g[b];
        }
        if (Minv) {
            const real* Mi = Minv + i * D * D;
            real C[9] = {0};
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b)
                    for (int c = 0; c < D; ++c) C[a * D + b] += Mi[a * D + c] * G[c * D + b];
            for (int a = 0; a < D * D; ++a) G[a] = C[a];
        }
        real tr = 0, s2 = 0;
        for (int a = 0; a < D; ++a) tr += G[a * D + a];
        for (int a = 0; a < D; ++a)
            for (int b = 0; b < D; ++b) {
                real sv = (G[a * D + b] + G[b * D + a]) / 2 - (a == b ? tr / (real)D : 0);
                s2 += sv * sv;
            }
        div_out[i] = tr;
        shear2_out[i] = s2;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0, Hi = H[i];
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real W = kW(&o, rsqrt_safe(dotD(d, d, D)), Hi);
            if (W == 0) continue;
            real sg = div_out[j] > 0 ? 1 : (div_out[j] < 0 ? -1 : 0);
            s += m[j] / rho[j] * (rho[j] * sg) * W;
        }
        real R = 1 / rho[i] * s;
        real omr = 1 - R, omr2 = omr * omr;
        real nom = o.beta_xi * (omr2 * omr2) * div_out[i];
        real Xi = o.limit_xi ? (nom * nom + (real)1e-14 * Hi) / (nom * nom + shear2_out[i] + (real)1e-14 * Hi)
                             : (nom * nom) / (nom * nom + shear2_out[i] + (real)1e-14 * Hi);
        real al = Xi * alpha0[i];
        alpha_out[i] = al < o.alpha_min ? o.alpha_min : al;
        if (R_out) R_out[i] = R;
    }
    return 0;
}

/* Free-surface detection, colour-field scheme (modules/surfaceDetection/colorFieldCompute.py,
 * colorFieldDetection.py, util/wp_numNeighbors.py, util/wp_sum.py, wp_dilate.py).  The
 * super-symmetric tests are W(r_ij, max(H_i, H_j)) > 0 as in the reference pair bodies. */
int oracle_surface_color_field(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                               const int32_t* offs, const int32_t* cnt, const int32_t* list, real* c_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real W = kW(&o, rsqrt_safe(dotD(d, d, D)), H[i]);
            if (W == 0) continue;
            s += m[j] / rho[j] * W;
        }
        c_out[i] = s;
    }
    return 0;
}

int oracle_surface_detect(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                          const real* c, const int32_t* offs, const int32_t* cnt, const int32_t* list, real limit,
                          real normal_sign, real* fs_out, real* normals_out, real* nn_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real gc[3] = {0, 0, 0}, nn = 0, cs = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            kWG(&o, d, r, H[i], &W, g);
            if (W != 0)
                for (int a = 0; a < D; ++a) gc[a] += m[j] / rho[j] * (c[j] - c[i]) * g[a];
            if (kW(&o, r, H[i] > H[j] ? H[i] : H[j]) > 0) { nn += 1; cs += c[j]; }
        }
        fs_out[i] = (c[i] < cs / nn && nn < limit) ? 1 : 0;
        nn_out[i] = nn;
        real nrm = SQRT(dotD(gc, gc, D));
        if (nrm < (real)1e-12) nrm = (real)1e-12;
        for (int a = 0; a < D; ++a) normals_out[i * D + a] = normal_sign * (gc[a] / nrm);
    }
    return 0;
}

int oracle_surface_dilate(const SphParams* p, int64_t n, const real* x, const real* H, const real* fs, const int32_t* offs,
                          const int32_t* cnt, const int32_t* list, real* out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            if (kW(&o, rsqrt_safe(dotD(d, d, D)), H[i] > H[j] ? H[i] : H[j]) > 0) s += fs[j];
        }
        out[i] = s;
    }
    return 0;
}

/* Barecasco detection (modules/surfaceDetection/wp_barecasco.py:36-113, 120-236, 338-355;
 * barecascoDetection.py:22-43): cover vector over the pairs with W(r, max(H_i, H_j)) > 0,
 * Warp's normalize (zero for a zero vector), the cone count, mask = count < 0.5. */
int oracle_surface_barecasco(const SphParams* p, int64_t n, const real* x, const real* H, const int32_t* offs, const int32_t* cnt,
                             const int32_t* list, real threshold, real* fs_out, real* normals_out, real* count_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real c[3] = {0, 0, 0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            if (!(kW(&o, r, H[i] > H[j] ? H[i] : H[j]) > 0)) continue;
            for (int a = 0; a < D; ++a) c[a] += d[a] / (r + (real)1e-14 * H[i]);
        }
        real l = SQRT(dotD(c, c, D));
        real ch[3] = {0, 0, 0};
        for (int a = 0; a < D; ++a) ch[a] = l > 0 ? c[a] / l : 0;
        int degenerate = SQRT(dotD(ch, ch, D)) <= (real)0.5;
        real count = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            if (!(kW(&o, r, H[i] > H[j] ? H[i] : H[j]) > 0)) continue;
            real den = r + (real)1e-14 * H[i], dt = 0;
            for (int a = 0; a < D; ++a) dt += -(d[a] / den) * ch[a];
            if (dt > 1) dt = 1;
            if (dt < -1) dt = -1;
            real angle = ACOS(dt);
            if ((angle <= threshold / 2 && j != i) || degenerate) count += 1;
        }
        fs_out[i] = count < (real)0.5 ? 1 : 0;
        count_out[i] = count;
        for (int a = 0; a < D; ++a) normals_out[i * D + a] = ch[a];
    }
    return 0;
}

/* Maronne detection (modules/surfaceDetection/wp_maronne.py:57-161) with given normals. */
int oracle_surface_maronne(const SphParams* p, int64_t n, const real* x, const real* H, const real* normals, const int32_t* offs,
                           const int32_t* cnt, const int32_t* list, real* fs_out, real* count_out) {
    OP o = op_from(p);
    int D = o.dim;
    real xk = (real)o.kxi;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const real* ni = normals + i * D;
        real T[3] = {0, 0, 0}, tau[3] = {0, 0, 0};
        for (int a = 0; a < D; ++a) T[a] = x[i * D + a] + ni[a] * H[i] / xk;
        if (D == 2) { tau[0] = -ni[1]; tau[1] = ni[0]; }
        if (D == 3) { tau[0] = ni[1] * ni[2]; tau[1] = -ni[0] * ni[2]; tau[2] = ni[0] * ni[1]; }
        int long_normal = rsqrt_safe(dotD(ni, ni, D)) > (real)0.5;
        real count = 0, s2 = SQRT((real)2);
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], dt[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real rij = rsqrt_safe(dotD(d, d, D)), hij = H[j];
            if (rij >= hij) continue;
            dist_vec(&o, x + (int64_t)j * D, T, dt);
            real rjt = rsqrt_safe(dotD(dt, dt, D)), lim = hij / xk;
            int A = rij >= s2 * hij / xk && rjt <= lim && j != i;
            int B = rij < s2 * hij / xk && FABS(dotD(ni, dt, D)) + FABS(dotD(tau, dt, D)) < lim && j != i;
            if ((A || B) && long_normal) count += 1;
        }
        fs_out[i] = count < (real)0.5 ? 1 : 0;
        count_out[i] = count;
    }
    return 0;
}

/* Colour-field-gradient detection (colorFieldGradientDetection.py:18-56). */
int oracle_surface_color_gradient(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                                  const real* c, const int32_t* offs, const int32_t* cnt, const int32_t* list, real threshold,
                                  real* fs_out, real* normals_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real gc[3] = {0, 0, 0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], &W, g);
            if (W == 0) continue;
            for (int a = 0; a < D; ++a) gc[a] += m[j] / rho[j] * (c[j] - c[i]) * g[a];
        }
        real l = SQRT(dotD(gc, gc, D));
        fs_out[i] = l > threshold * H[i] / (real)o.kxi ? 1 : 0;
        real den = l < (real)1e-12 ? (real)1e-12 : l;
        for (int a = 0; a < D; ++a) normals_out[i * D + a] = -(gc[a] / den);
    }
    return 0;
}

/* The moment matrix of the renormalisation, M_i = sum_j V_j (x_j - x_i) (x) grad_i W(r,
 * max(H_i, H_j)) (M_out row-major D x D per particle); the caller inverts it. */
int oracle_surface_moments(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                           const int32_t* offs, const int32_t* cnt, const int32_t* list, real* M_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[i] > H[j] ? H[i] : H[j], &W, g);
            if (W == 0) continue;
            real Vj = m[j] / rho[j];
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) M[a * D + b] += Vj * (-d[a]) * g[b];
        }
        for (int a = 0; a < D * D; ++a) M_out[i * D * D + a] = M[a];
    }
    return 0;
}

/* Normals from the renormalised gradients: mode 0 (lambdaGrad.py) sum_j V_j (lambda_j -
 * lambda_i) grad W(r, H_j), mode 1 (maronneNormals.py) sum_j V_j grad W(r, H_j); g = L_i times
 * the sum, normals = -g / max(|g|, 1e-12). */
int oracle_surface_renorm_normals(const SphParams* p, int64_t n, int mode, const real* x, const real* H, const real* m,
                                  const real* rho, const real* L, const real* lam, const int32_t* offs, const int32_t* cnt,
                                  const int32_t* list, real* normals_out, real* grad_out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s[3] = {0, 0, 0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), H[j], &W, g);
            if (W == 0) continue;
            real Vj = m[j] / rho[j];
            real w = mode == 0 ? Vj * (lam[j] - lam[i]) : Vj;
            for (int a = 0; a < D; ++a) s[a] += w * g[a];
        }
        real v[3] = {0, 0, 0};
        for (int a = 0; a < D; ++a)
            for (int b = 0; b < D; ++b) v[a] += L[i * D * D + a * D + b] * s[b];
        real l = SQRT(dotD(v, v, D));
        if (l < (real)1e-12) l = (real)1e-12;
        for (int a = 0; a < D; ++a) {
            normals_out[i * D + a] = -(v[a] / l);
            if (grad_out) grad_out[i * D + a] = v[a];
        }
    }
    return 0;
}

int oracle_switch_hopkins_update(const SphParams* p, int64_t n, const real* x, const real* H, const real* v, const real* c,
                                 const real* div, const real* div_prev, const real* alpha0, real dt,
                                 const int32_t* offs, const int32_t* cnt, const int32_t* list, real* alpha0_out,
                                 real* vsig_out) {
    OP o = op_from(p);
    real* vs = (real*)malloc(sizeof(real) * (size_t)(n > 0 ? n : 1));
    oracle_vsig(p, n, x, H, v, c, offs, cnt, list, vs);
    real f_kern = 1 / o.kxi;
    for (int64_t i = 0; i < n; ++i) {
        real ddiv = (div[i] - div_prev[i]) / dt;
        real ad = FABS(ddiv);
        real fh = f_kern * H[i];
        real at = o.alpha_max * ad / (ad + o.beta_c * (c[i] * c[i]) / (fh * fh) + (real)1e-14);
        if (ddiv > 0 || div[i] > 0) at = 0;
        real nxt = at + (alpha0[i] - at) * EXP(-o.beta_d * dt * vs[i] / (2 * f_kern * H[i]));
        alpha0_out[i] = at >= alpha0[i] ? at : nxt;
        if (vsig_out) vsig_out[i] = vs[i];
    }
    free(vs);
    return 0;
}

/* Balsara (commented formula at schemes/crkSPH.py:132-133) */
int oracle_switch_balsara(const SphParams* p, int64_t n, const real* DvDx, const real* c, real* alpha) {
    int D = p->dim;
    for (int64_t i = 0; i < n; ++i) {
        const real* G = DvDx + i * D * D;
        real dv = 0, curl2 = 0;
        for (int a = 0; a < D; ++a) dv += G[a * D + a];
        if (D == 2) { real w = G[2] - G[1]; curl2 = w * w; }
        if (D == 3) { real w0 = G[7] - G[5], w1 = G[2] - G[6], w2 = G[3] - G[1]; curl2 = w0 * w0 + w1 * w1 + w2 * w2; }
        real ad = FABS(dv);
        real b = ad / (ad + SQRT(curl2) + (real)1e-4 * c[i]);
        alpha[i] = b < 0 ? 0 : (b > 1 ? 1 : b);
    }
    return 0;
}

/* ------------------------------------------------------------------ CRK accel / dudt
 * modules/crk/limiter.py:10-16 (limiterVL), :27-86 (computeVanLeer), :89-128 (crkLimiter);
 * modules/crk/accel.py:65-250 (computeCrkSPHAccel_Func_i);
 * modules/crk/dudt.py:62-229 (computeCrkSPHdudt_Func_i). */
static real limiter_vl(real x) {
    if (x <= 0) return 0;
    real vL = 2 / (1 + x);
    return x * vL * vL;
}
static real sgn_pos(real x) { return x >= 0 ? 1 : -1; }
static real van_leer(int D, const real* xij_, const real* Gi, const real* Gj) {
    real h[3], ci[3], cj[3];
    for (int a = 0; a < D; ++a) h[a] = (real)0.5 * xij_[a];
    for (int a = 0; a < D; ++a) {
        ci[a] = Gi[a * D] * h[0]; cj[a] = Gj[a * D] * h[0];
        for (int b = 1; b < D; ++b) { ci[a] += Gi[a * D + b] * h[b]; cj[a] += Gj[a * D + b] * h[b]; }
    }
    real gi = dotD(ci, h, D), gj = dotD(cj, h, D);
    real ri = gi / (sgn_pos(gj) * FABS(gj));
    real rj = gj / (sgn_pos(gi) * FABS(gi));
    if (ri != ri) ri = 1;
    if (rj != rj) rj = 1;
    return limiter_vl(wmin(ri, rj));
}
static real crk_limiter(int D, const real* xij, real hi, real hj, real eta_crit, real eta_fold) {
    real ni = 0, nj = 0;
    for (int a = 0; a < D; ++a) { real ei = xij[a] / hi, ej = xij[a] / hj; ni += ei * ei; nj += ej * ej; }
    real eta = wmin(rsqrt_safe(ni), rsqrt_safe(nj));
    real f = 1;
    if (eta < eta_crit) { real t = (eta - eta_crit) / eta_fold; f = EXP(-(t * t)); }
    return f;
}
static void kahan_add(real* s, real* c, real x, int comp) {
    if (!comp) { *s += x; return; }
    real t = *s + x;
    if (FABS(*s) >= FABS(x)) *c += (*s - t) + x; else *c += (x - t) + *s;
    *s = t;
}

int oracle_crk_accel_dudt(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                          const real* V, const real* A, const real* B, const real* gA, const real* gB, const real* v,
                          const real* c, const real* Pr, const real* DvDx,
                          const int32_t* offs, const int32_t* cnt, const int32_t* list,
                          real* dvdt, real* dudt, real* ap, real* av) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        const real *xi = x + i * D, *vi = v + i * D, *Gi = DvDx + i * D * D;
        real Hi = H[i], mi = m[i], rhoi = rho[i], Vi = V[i], ci = c[i], Pi = Pr[i];
        real smooth_i = Hi / o.kscale;
        real acc[3] = {0, 0, 0}, accc[3] = {0, 0, 0}, du = 0, duc = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, xi, x + (int64_t)j * D, d);
            real r2 = dotD(d, d, D);
            real Hj = H[j], Hm = wmax(Hi, Hj);
            if (!(r2 < Hm * Hm)) {
                if (ap) for (int a = 0; a < D; ++a) ap[(int64_t)k * D + a] = 0;
                if (av) for (int a = 0; a < D; ++a) av[(int64_t)k * D + a] = 0;
                continue;
            }
            real r = rsqrt_safe(r2);
            const real *vj = v + (int64_t)j * D, *Gj = DvDx + (int64_t)j * D * D;
            real rhoj = rho[j], Vj = V[j], cj = c[j], Pj = Pr[j];
            real factor = 1;
            if (o.crk_lim) factor = crk_limiter(D, d, Hi, Hj, o.eta_crit, o.eta_fold);
            real phi = 0;
            if (o.vl) phi = van_leer(D, d, Gi, Gj) * factor;
            if (o.vl_off) phi = 0;
            if (o.vl_on) phi = 1;
            phi = wmax(wmin(phi, 1), 0);
            real Gix[3], Gjx[3];
            for (int a = 0; a < D; ++a) {
                Gix[a] = Gi[a * D] * d[0]; Gjx[a] = Gj[a * D] * d[0];
                for (int b = 1; b < D; ++b) { Gix[a] += Gi[a * D + b] * d[b]; Gjx[a] += Gj[a * D + b] * d[b]; }
            }
            real hp = phi / 2, vdi[3], vdja[3], vdjd[3];
            for (int a = 0; a < D; ++a) {
                vdi[a] = vi[a] - hp * Gix[a];
                vdja[a] = vj[a] + hp * Gjx[a];
                vdjd[a] = vj[a] + hp * (-Gjx[a]);
            }
            real Wi, gWi[3], gri[3], Wj, gWj[3], grj[3], xji[3], gij[3];
            kWG(&o, d, r, Hj, &Wi, gWi);
            crk_grad(D, d, Wi, gWi, A[i], B + i * D, gA + i * D, gB + i * D * D, gri);
            for (int a = 0; a < D; ++a) xji[a] = -d[a];
            kWG(&o, xji, r, Hi, &Wj, gWj);
            crk_grad(D, xji, Wj, gWj, A[j], B + (int64_t)j * D, gA + (int64_t)j * D, gB + (int64_t)j * D * D, grj);
            for (int a = 0; a < D; ++a) gij[a] = (real)0.5 * (gri[a] - grj[a]);
            real smooth_j = Hj / o.kscale;
            real ee_i = 0, ee_j = 0, mia = 0, mja = 0, mid = 0, mjd = 0;
            for (int a = 0; a < D; ++a) {
                real ei = d[a] / smooth_i, ej = d[a] / smooth_j;
                ee_i += ei * ei; ee_j += ej * ej;
                real da = vdi[a] - vdja[a], dd = vdi[a] - vdjd[a];
                mia += da * ei; mja += da * ej; mid += dd * ei; mjd += dd * ej;
            }
            real den_i = ee_i + (real)1.0e-7 * smooth_i * smooth_i, den_j = ee_j + (real)1.0e-7 * smooth_j * smooth_j;
            mia = wmin(0, mia / den_i); mja = wmin(0, mja / den_j);
            mid = wmin(0, mid / den_i); mjd = wmin(0, mjd / den_j);
            real Qia = rhoi * (-o.C_l * ci * mia + o.C_q * mia * mia), Qja = rhoj * (-o.C_l * cj * mja + o.C_q * mja * mja);
            real Qid = rhoi * (-o.C_l * ci * mid + o.C_q * mid * mid), Qjd = rhoj * (-o.C_l * cj * mjd + o.C_q * mjd * mjd);
            real dotu = 0;
            for (int a = 0; a < D; ++a) {
                real pt = -(Pi + Pj) * gij[a] * Vi * Vj / mi;
                real vt = -(Qia + Qja) * Vj * 1 * gij[a] * Vi / mi;
                if (ap) ap[(int64_t)k * D + a] = pt;
                if (av) av[(int64_t)k * D + a] = vt;
                kahan_add(&acc[a], &accc[a], pt + vt, o.kahan);
                dotu += (vi[a] - vj[a]) * gij[a];
            }
            real pTerm = Pj * dotu * Vi * Vj / mi;
            real vTerm = (real)0.5 * (Qid + Qjd) * 1 * dotu * Vi * Vj / mi;
            kahan_add(&du, &duc, pTerm + vTerm, o.kahan);
        }
        if (dvdt) for (int a = 0; a < D; ++a) dvdt[i * D + a] = acc[a] + accc[a];
        if (dudt) dudt[i] = du + duc;
    }
    return 0;
}

/* ------------------------------------------------------------------ energy partition (modules/compSPH/balance.py:62-154) */
static real sgn0(real x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
int oracle_compsph_balance(const SphParams* p, int64_t n, const real* m, const real* rho, const real* Pr, const real* u,
                           const real* v, const real* dvdt, real dt, const int32_t* offs, const int32_t* cnt,
                           const int32_t* list, const real* ap, const real* av, real* fout) {
    OP o = op_from(p);
    int D = o.dim;
    real hdt = (real)0.5 * dt;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real vi[3];
        for (int a = 0; a < D; ++a) vi[a] = v[i * D + a] + hdt * dvdt[i * D + a];
        real mi = m[i], rhoi = rho[i], Pi = Pr[i], ui = u[i];
        real si = o.energy_scheme == SPH_ENERGY_CRK ? Pi / POW(rhoi, o.gamma) : 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real mj = m[j], rhoj = rho[j], Pj = Pr[j], uj = u[j];
            real dE = 0;
            for (int a = 0; a < D; ++a)
                dE += ((v[(int64_t)j * D + a] + hdt * dvdt[(int64_t)j * D + a]) - vi[a]) * (ap[(int64_t)k * D + a] + av[(int64_t)k * D + a]);
            dE = mi * dE * dt;
            real uji = uj - ui, f = (real)0.5;
            int sch = o.energy_scheme;
            if (sch == SPH_ENERGY_EQUALWORK) f = (real)0.5;
            else if (sch == SPH_ENERGY_PDV) f = (Pi / (rhoi * rhoi)) / (Pi / (rhoi * rhoi) + Pj / (rhoj * rhoj));
            else if (sch == SPH_ENERGY_DIMINISHING) { real un = FABS(uji); f = (real)0.5 * (1 + (uji * sgn0(dE)) / (un + 1 / (1 + un))); }
            else if (sch == SPH_ENERGY_MONOTONIC || sch == SPH_ENERGY_HYBRID) {
                real Aq = dE / (uji + (real)1.0e-14);
                real Bq = Aq >= 0 ? Aq / mi : Aq / mj;
                real t1 = wmax(0, sgn0(Bq));
                real t2 = mi / (dE + (real)1.0e-14) * ((dE + mi * ui + mj * uj) / (mi + mj) - ui);
                real fm = FABS(Bq) <= 1 ? t1 : t2;
                if (sch == SPH_ENERGY_MONOTONIC) f = fm;
                else {
                    real un = FABS(uji);
                    real fsm = (real)0.5 * (1 + (uji * sgn0(dE)) / (un + 1 / (1 + un)));
                    real chi = FABS(uji) / (FABS(ui) + FABS(uj) + (real)1.0e-14);
                    f = chi * fm + (1 - chi) * fsm;
                }
            } else if (sch == SPH_ENERGY_CRK) {
                real sj = Pj / POW(rhoj, o.gamma);
                real smin = wmin(FABS(si), FABS(sj)), smax = wmax(FABS(si), FABS(sj));
                int mA = FABS(si - sj) == 0;
                int mB = (dE >= 0 && si >= sj) || (dE < 0 && si < sj);
                int mC = (dE >= 0 && si < sj) || (dE < 0 && si >= sj);
                f = (real)0.5;
                if (mA) f = (real)0.5;
                if (!mA && mB) f = smin / (smin + smax + (real)1.0e-14);
                if (!mA && !mB && mC) f = smax / (smin + smax + (real)1.0e-14);
                f = wmax(0, wmin(1, f));
            }
            fout[k] = f;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ CFL (modules/timestep/compressible.py:18-61) */
real oracle_cfl_dt(const SphParams* p, int64_t n, const real* H, const real* u, real dt_prev, int has_prev) {
    OP o = op_from(p);
    real hmin = H[0], best = 0;
    for (int64_t i = 1; i < n; ++i) hmin = H[i] < hmin ? H[i] : hmin;
    for (int64_t i = 0; i < n; ++i) {
        real cs = SQRT(FABS(u[i]) * o.gamma * (o.gamma - 1));
        real dt = o.cfl * hmin / (cs * o.kxi);
        if (i == 0 || dt < best) best = dt;
    }
    best = best < o.min_dt ? o.min_dt : (best > o.max_dt ? o.max_dt : best);
    if (has_prev && best > dt_prev) best = best < o.dt_growth * dt_prev ? best : o.dt_growth * dt_prev;
    return best;
}

/* ------------------------------------------------------------------ compatible energy
 * modules/compSPH/multistep.py:52-94 and systems/compSPH.py:100-111. */
int oracle_finalize_compatible_energy(const SphParams* p, int64_t n, int ns, const double* w, real dt, const real* v0,
                                      const real* u0, const real* const* dvdt_s, const int32_t* const* offs_s,
                                      const int32_t* const* cnt_s, const int32_t* const* list_s, const real* const* f_s,
                                      const real* const* ap_s, const real* const* av_s, real* u_out, real* du_out) {
    int D = p->dim;
    int pdv = p->energy_scheme == SPH_ENERGY_PDV;
    real* vh = (real*)malloc(sizeof(real) * (size_t)(n * D > 0 ? n * D : 1));
    for (int64_t q = 0; q < n * D; ++q) {
        real fa = 0;
        for (int s = 0; s < ns; ++s) fa += (real)w[s] * dvdt_s[s][q];
        vh[q] = v0[q] + (real)0.5 * fa * dt;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real du = 0;
        for (int s = 0; s < ns; ++s) {
            real acc = 0, ws = (real)w[s];
            for (int32_t k = offs_s[s][i]; k < offs_s[s][i] + cnt_s[s][i]; ++k) {
                int32_t j = list_s[s][k];
                real d1 = 0, d2 = 0;
                for (int a = 0; a < D; ++a) {
                    real vji = vh[(int64_t)j * D + a] - vh[i * D + a];
                    d1 += vji * ap_s[s][(int64_t)k * D + a];
                    d2 += vji * av_s[s][(int64_t)k * D + a];
                }
                real fk = f_s[s][k];
                acc += pdv ? (ws * fk * d1 + ws * (real)0.5 * d2) : (ws * fk * (d1 + d2));
            }
            du += acc;
        }
        if (du_out) du_out[i] = du;
        u_out[i] = u0[i] + du * dt;
    }
    free(vh);
    return 0;
}

/* ------------------------------------------------------------------ incompressible (DFSPH)
 * The generic warpSPHCore operations these modules call are restated with the
 * standard SPH forms (parity with the reference unpinned for those operators):
 *   Divergence, Difference, consistentDivergence=False:  sum_j V_j (q_j - q_i) . gradW_ij
 *   Gradient, Symmetric:  rho_i sum_j m_j (q_i/rho_i^2 + q_j/rho_j^2) gradW_ij
 * with V_j = m_j/rho_j and gradW_ij = grad_i W(x_i - x_j, H) (H_j for scatter, H_i
 * for gather support). */
static void kWG_mode(const OP* o, const real* x, real r, real Hi, real Hj, int mode, real* W, real* g) {
    if (mode == SPH_SUPPORT_GATHER) kWG(o, x, r, Hi, W, g);
    else kWG(o, x, r, Hj, W, g);
}

/* modules/momentum/incompressible.py:9-34 with v* = v + dt*dvdt (divergenceFree.py:32) */
int oracle_incompressible_divergence(const SphParams* p, int64_t n, double rho0, const real* x, const real* H, const real* m,
                                     const real* rho, const real* v, const real* dvdt, real dt, const int32_t* offs,
                                     const int32_t* cnt, const int32_t* list, real* div) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real vi[3], s = 0;
        for (int a = 0; a < D; ++a) vi[a] = dvdt ? v[i * D + a] + dt * dvdt[i * D + a] : v[i * D + a];
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG_mode(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], H[j], SPH_SUPPORT_SCATTER, &W, g);
            real Vj = m[j] / rho[j], t = 0;
            for (int a = 0; a < D; ++a) {
                real vj = dvdt ? v[(int64_t)j * D + a] + dt * dvdt[(int64_t)j * D + a] : v[(int64_t)j * D + a];
                t += (vj - vi[a]) * g[a];
            }
            s += Vj * t;
        }
        div[i] = -(real)rho0 * s;
    }
    return 0;
}

/* modules/incompressible/wp_alpha.py:35-118 (gather support, areaI = m_i/rho_i) and
 * :294-313 (the returned value is -alpha) */
int oracle_dfsph_alpha(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list, real* alpha) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real sA[3] = {0, 0, 0}, sB = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG_mode(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], H[j], SPH_SUPPORT_GATHER, &W, g);
            real Vj = m[j] / rho[j];
            for (int a = 0; a < D; ++a) sA[a] += Vj * g[a];
            sB += Vj * Vj / m[j] * dotD(g, g, D);
        }
        real Ai = m[i] / rho[i];
        alpha[i] = -(Ai / m[i] * dotD(sA, sA, D) + Ai * sB);
    }
    return 0;
}

/* modules/pressure/iisph.py:7-24 (scatter support) */
int oracle_pressure_accel_iisph(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                                const real* pr, const int32_t* offs, const int32_t* cnt, const int32_t* list, real* acc) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s[3] = {0, 0, 0};
        real qi = pr[i] / (rho[i] * rho[i]);
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG_mode(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], H[j], SPH_SUPPORT_SCATTER, &W, g);
            real c = m[j] * (qi + pr[j] / (rho[j] * rho[j]));
            for (int a = 0; a < D; ++a) s[a] += c * g[a];
        }
        for (int a = 0; a < D; ++a) acc[i * D + a] = -(rho[i] * s[a]) / rho[i];
    }
    return 0;
}

/* modules/incompressible/drift.py:38-57 */
int oracle_pressure_shift_iisph(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                                const real* acc, const int32_t* offs, const int32_t* cnt, const int32_t* list, real* shift) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real s = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, g[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG_mode(&o, d, rsqrt_safe(dotD(d, d, D)), H[i], H[j], SPH_SUPPORT_SCATTER, &W, g);
            real t = 0;
            for (int a = 0; a < D; ++a) t += (acc[(int64_t)j * D + a] - acc[i * D + a]) * g[a];
            s += m[j] / rho[j] * t;
        }
        shift[i] = -s;
    }
    return 0;
}

/* The two relaxed Jacobi solves:
 *   mode 0: solveDivergenceFree (modules/incompressible/divergenceFree.py:23-139)
 *   mode 1: solveIncompressible (modules/incompressible/incompressible.py:21-143)
 * hist[it*4 + {0,1,2,3}] = error, min p, max p, mean p (after the update of iteration it). */
int oracle_jacobi_solve(const SphParams* p, int mode, const SphJacobiConfig* cfg, int64_t n, const real* x, const real* H,
                        const real* m, const real* rho, const real* v, const real* dvdt, const real* p_init, real dt,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list, real* p_out, real* acc_out,
                        double* hist, int* iters) {
    int D = p->dim;
    size_t nn = (size_t)(n > 0 ? n : 1);
    real* src = (real*)malloc(sizeof(real) * nn);
    real* diag = (real*)malloc(sizeof(real) * nn);
    real* pa = (real*)malloc(sizeof(real) * nn);
    real* sh = (real*)malloc(sizeof(real) * nn);
    real* acc = (real*)malloc(sizeof(real) * nn * D);
    real dtf = mode == 0 ? dt : dt * dt;
    real omega = (real)cfg->relaxation, tol = (real)cfg->tolerance;
    oracle_incompressible_divergence(p, n, cfg->rest_density, x, H, m, rho, v, dvdt, dt, offs, cnt, list, src);
    oracle_dfsph_alpha(p, n, x, H, m, rho, offs, cnt, list, diag);
    for (int64_t i = 0; i < n; ++i) {
        if (mode == 0) {
            src[i] = -src[i];                                   /* divergenceFree.py:54 */
            diag[i] = dt * diag[i];                             /* :62 */
            p_out[i] = cfg->init_mode ? p_init[i] : p_init[i] * (real)0.75;   /* :72 */
        } else {
            real rs = rho[i] + dt * src[i];                     /* incompressible.py:54-56 */
            rs = rs < (real)0.9 ? (real)0.9 : rs;
            src[i] = (real)cfg->rest_density - rs;              /* :59 */
            real a = dt * dt * diag[i];                         /* :68 */
            diag[i] = a > (real)-1e-6 ? (real)-1e-6 : a;        /* :76 */
            p_out[i] = cfg->init_mode ? p_init[i] : (real)0;    /* :79 */
        }
    }
    int it = 0;
    for (it = 0; it < cfg->max_iterations; ++it) {
        for (int64_t i = 0; i < n; ++i) pa[i] = p_out[i];
        oracle_pressure_accel_iisph(p, n, x, H, m, rho, pa, offs, cnt, list, acc);
        oracle_pressure_shift_iisph(p, n, x, H, m, rho, acc, offs, cnt, list, sh);
        double esum = 0, psum = 0;
        for (int64_t i = 0; i < n; ++i) {
            real r = src[i] - dtf * sh[i];
            real pb = pa[i] + omega * r / diag[i];
            if (mode == 1) {
                pb = pb < 0 ? 0 : pb;                           /* incompressible.py:108 */
                real e = -r < -tol ? -tol : -r;                 /* :111 */
                esum += (double)e;
            } else {
                esum += fabs((double)r);                        /* divergenceFree.py:112 */
            }
            p_out[i] = pb;
            psum += (double)pb;
        }
        real mu = mode == 0 && n > 0 ? (real)(psum / (double)n) : 0;
        real pmin = 0, pmax = 0;
        double msum = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (mode == 0) p_out[i] = p_out[i] - mu;            /* divergenceFree.py:104 */
            if (i == 0 || p_out[i] < pmin) pmin = p_out[i];
            if (i == 0 || p_out[i] > pmax) pmax = p_out[i];
            msum += (double)p_out[i];
        }
        double err = n > 0 ? esum / (double)n : 0;
        hist[it * 4 + 0] = err;
        hist[it * 4 + 1] = pmin;
        hist[it * 4 + 2] = pmax;
        hist[it * 4 + 3] = n > 0 ? msum / (double)n : 0;
        if (it >= cfg->min_iterations && err < cfg->tolerance) { ++it; break; }
    }
    *iters = it < cfg->max_iterations ? it : cfg->max_iterations;
    oracle_pressure_accel_iisph(p, n, x, H, m, rho, p_out, offs, cnt, list, acc_out);
    free(src); free(diag); free(pa); free(sh); free(acc);
    return 0;
}

/* ------------------------------------------------------------------ weakly compressible delta-SPH
 * modules/eos/weaklyCompressible.py:4-44; the renormalised density gradient of
 * modules/density/gradRhoL.py:33-56 with L = (sum_j V_j gradW (x) (x_j - x_i))^-1
 * (warpSPHCore's renormalisation, restated); modules/momentum/inconsistent.py:16-31;
 * modules/deltaSPH/wp_densityDelta.py:14-118 with densityDiffusion.py:17-35;
 * modules/pressure/wp_surfaceAware.py:10-64, :207; modules/deltaSPH/wp_viscosityDelta.py:14-108.
 * Kernel support max(H_i, H_j) (super-symmetric). */
static real wc_eos(const SphWcParams* w, real rho) {
    real r0 = (real)w->rest_density, c = (real)w->sound_speed, g = (real)w->polytropic_exponent, k = (real)w->kappa;
    switch (w->eos) {
        case SPH_EOS_STIFF_TAIT: return r0 * c * c / g * (POW(rho / r0, g) - 1);
        case SPH_EOS_TAIT: return k * (rho - r0);
        case SPH_EOS_ISOTHERMAL: return c * c * (rho - r0);
        case SPH_EOS_POLYTROPIC: return k * POW(rho, g);
        default: return k / g * (POW(rho / r0, g) - 1);
    }
}

int oracle_deltasph_rhs(const SphParams* p, const SphWcParams* w, int64_t n, const real* x, const real* H, const real* m,
                        const real* rho, const real* v, const int32_t* smask, const int32_t* offs, const int32_t* cnt,
                        const int32_t* list, real* gL, real* Pr, real* dvdt, real* drhodt) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real M[3][3] = {{0}}, g[3] = {0, 0, 0};
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, gw[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), wmax(H[i], H[j]), &W, gw);
            real Vj = m[j] / rho[j], dr = rho[j] - rho[i];
            for (int a = 0; a < D; ++a) {
                g[a] += Vj * dr * gw[a];
                for (int c = 0; c < D; ++c) M[a][c] += Vj * gw[a] * (-d[c]);
            }
        }
        real r[3] = {g[0], g[1], g[2]};
        if (D == 1) {
            if (FABS(M[0][0]) > (real)1e-6) r[0] = g[0] / M[0][0];
        } else if (D == 2) {
            real det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
            if (FABS(det) > (real)1e-6) {
                real id = 1 / det;
                r[0] = id * (M[1][1] * g[0] - M[0][1] * g[1]);
                r[1] = id * (-M[1][0] * g[0] + M[0][0] * g[1]);
            }
        } else {
            double a[9], inv[9];
            for (int q = 0; q < 9; ++q) a[q] = (double)M[q / 3][q % 3];
            double det = inv_sym(3, a, inv);   /* general 3x3 inverse */
            if (fabs(det) > 1e-6)
                for (int q = 0; q < 3; ++q) r[q] = (real)(inv[q * 3 + 0] * g[0] + inv[q * 3 + 1] * g[1] + inv[q * 3 + 2] * g[2]);
        }
        for (int a = 0; a < D; ++a) gL[i * D + a] = r[a];
        Pr[i] = wc_eos(w, rho[i]);
    }
    real xi = o.kxi;
    real visc_nu = (real)2 * (real)(D + 2) * (real)w->viscosity_nu;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real cont = 0, dd = 0, pf[3] = {0, 0, 0}, vs[3] = {0, 0, 0};
        real Hi = H[i], rhoi = rho[i], Pi = Pr[i], eps = (real)1.0e-14 * Hi;
        int surf_i = smask != NULL && smask[i] == 1;   /* wp_surfaceAware.py:89-92: mask_i == 1 */
        real factor = w->inviscid ? (real)w->inviscid_alpha * (real)w->sound_speed * Hi / xi : visc_nu;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, gw[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r2 = dotD(d, d, D), rr = rsqrt_safe(r2);
            kWG(&o, d, rr, wmax(Hi, H[j]), &W, gw);
            real rj = rho[j], Vj = m[j] / rj;
            real t = 0;
            for (int a = 0; a < D; ++a) t += (v[(int64_t)j * D + a] - v[i * D + a]) * gw[a];
            cont += Vj * t;
            real inv = 1 / (rr + eps), s = (real)2 * (rj - rhoi) * inv * inv, pd = 0;
            for (int a = 0; a < D; ++a) {
                real psi;
                if (w->density_scheme == SPH_DENSITY_DIFFUSION_DELTA) psi = (gL[i * D + a] + gL[(int64_t)j * D + a]) - s * d[a];
                else if (w->density_scheme == SPH_DENSITY_DIFFUSION_DENSITY_ONLY) psi = -(s * d[a]);
                else psi = gL[i * D + a] + gL[(int64_t)j * D + a];
                pd += psi * gw[a];
            }
            dd += Vj * pd;
            real Pj = Pr[j], pij;
            switch (w->pressure_term) {
                case SPH_PRESSURE_CONSERVATIVE: pij = Pj - Pi; break;
                case SPH_PRESSURE_NONCONSERVATIVE: pij = Pj + Pi; break;
                case SPH_PRESSURE_ANTUONO: pij = (Pi >= 0 || Pj >= 0 || surf_i) ? Pj + Pi : Pj - Pi; break;
                case SPH_PRESSURE_I: pij = Pi; break;
                case SPH_PRESSURE_J: pij = Pj; break;
                default: pij = (Pj / (rj * rj) + Pi / (rhoi * rhoi)) * rj; break;
            }
            for (int a = 0; a < D; ++a) pf[a] += Vj * pij * gw[a];
            real vx = 0;
            for (int a = 0; a < D; ++a) vx += (v[i * D + a] - v[(int64_t)j * D + a]) * d[a];
            real mu = vx / (r2 + eps * Hi);
            mu = mu > 0 ? 0 : mu;
            real ww = Vj * mu * factor / ((rj + rhoi) / 2);
            for (int a = 0; a < D; ++a) vs[a] += ww * gw[a];
        }
        drhodt[i] = -rhoi * cont + (real)w->density_delta * Hi / xi * (real)w->sound_speed * dd;
        /* the pressure force is divided by the particle's own density (wp_surfaceAware.py:207-218) */
        for (int a = 0; a < D; ++a) dvdt[i * D + a] = -pf[a] / rhoi + vs[a];
    }
    return 0;
}

/* delta-plus shift: modules/shifting/delta.py:6-47 (the scaling -CFL Ma 2 h^2, Ma from the
 * finite max |v| / c0, 0.1 below 1e-6) with the pair sum of sample/wp_deltaShift.py:57-126
 * under the gather support: sum_j (1 + R (W_ij / W0)^nexp) m_j / (2 (rho_i + rho_j)) gradW_ij,
 * W0 = eval_k(q0) C_d / H_i^d at q0 = ((m_j / rho0)^(1/d) / xi) / H_i.  Zero for kinds != 0
 * (modules/shifting/wrapper.py:100). */
int oracle_delta_shift(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho, const real* v,
                       const int32_t* kinds, const int32_t* offs, const int32_t* cnt, const int32_t* list, real cfl, real c0,
                       real R, int nexp, real rho0, real* shift) {
    OP o = op_from(p);
    int D = o.dim;
    real vmax = 0;
    int finite = 0;
    for (int64_t i = 0; i < n; ++i) {
        real s2 = 0;
        for (int a = 0; a < D; ++a) s2 += v[i * D + a] * v[i * D + a];
        real mag = SQRT(s2);
        if (isfinite(mag)) { vmax = mag > vmax ? mag : vmax; finite = 1; }
    }
    real cmax = finite ? vmax / c0 : (real)NAN;
    real Ma = cmax < (real)1e-6 ? (real)0.1 : cmax;
    real xi = o.kxi;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real acc[3] = {0, 0, 0};
        real Hi = H[i], rhoi = rho[i];
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3], W, gw[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            kWG(&o, d, rsqrt_safe(dotD(d, d, D)), Hi, &W, gw);
            real dxs = POW(m[j] / rho0, (real)1 / (real)D) / xi;
            real q0 = dxs / Hi, k0 = 0, p0;
            if (q0 < 1) kernel_kp(o.kernel, D, q0, &k0, &p0);
            real hd = D == 1 ? Hi : (D == 2 ? Hi * Hi : Hi * Hi * Hi);
            real W0 = k0 * kernel_C(o.kernel, D) / hd;
            real term = 1 + R * POW(W / W0, (real)nexp);
            real dterm = (real)0.5 * m[j] / (rhoi + rho[j]);
            real sc = term * dterm;
            for (int a = 0; a < D; ++a) acc[a] += sc * gw[a];
        }
        real h = Hi / xi;
        real scale = -cfl * Ma * (real)2 * (h * h);
        int moving = kinds == NULL || kinds[i] == 0;
        for (int a = 0; a < D; ++a) shift[i * D + a] = moving ? acc[a] * scale : 0;
    }
    return 0;
}

/* ------------------------------------------------------------------ artificial viscosity Pi_ij
 * modules/dissipation/pi.py:11-161 (computePi_actual) with util.py:6-38 (compute_mu_ij) and
 * util.py:42-134 (compute_bars).  ux = (v_i - v_j).x_ij, x_ij = x_i - x_j.  Returns Pi_ij
 * times rho_j, as the reference does (pi.py:8-9). */
static real oracle_pi(const OP* o, real r, real ux, real hi, real hj, real rhoi, real rhoj, real Pi_, real Pj_,
                      real ci, real cj, real ai, real aj, int useJ, int thermal) {
    real rho_bar = (real)1 / (real)2 * (rhoi + rhoj);
    real c_bar = (real)1 / (real)2 * (ci + cj);
    real h_bar = (real)1 / (real)2 * (hi + hj);
    real xi = o->correct_xi ? o->kxi : (real)1;
    real Cl_ = thermal ? o->Cu_l : o->C_l, Cq_ = thermal ? o->Cu_q : o->C_q;
    real C_l = (real)1 / (real)2 * (ai + aj) * Cl_;
    real C_q = (real)1 / (real)2 * (ai + aj) * Cq_;
    if (o->scale_beta) C_q = C_q * C_l;
    int term = thermal ? o->cond_term : o->visc_term;
    /* compute_mu_ij */
    real mu0 = ux / (r + (real)1e-14 * h_bar);
    real sfac = h_bar / xi / (r + (real)1e-14 * h_bar);
    real mu, sf;
    if (term == SPH_VISC_MONAGHAN1992) { mu = mu0 * sfac; sf = (real)1 * sfac; }
    else if (term == SPH_VISC_DEFAULT || term == SPH_VISC_MONAGHANGINGOLD1983 || term == SPH_VISC_DELTASPH || term > SPH_VISC_DELTASPH) {
        mu = mu0 * sfac; sf = h_bar / xi;
    } else { mu = mu0; sf = 1; }
    /* compute_bars */
    int brho = 1, bc = 1, bh = 1;
    if (term == SPH_VISC_CLEARY1998) { brho = 0; bc = 0; bh = 0; }
    else if (term == SPH_VISC_MONAGHAN1992) bc = 0;
    else if (term == SPH_VISC_DELTASPH) brho = 0;
    real rho = brho ? rho_bar : (useJ ? rhoj : rhoi);
    real c = bc ? c_bar : (useJ ? cj : ci);
    real h = bh ? h_bar : (useJ ? hj : hi);
    real v_sig = 0;
    switch (term) {
        case SPH_VISC_MONAGHANGINGOLD1983: v_sig = c; break;
        case SPH_VISC_CLEARY1998: {
            real f = (real)1 / ((real)2 * ((real)o->dim + (real)2));
            real mi_ = f * ai * C_l * hi * ci * rhoi / xi, mj_ = f * aj * C_l * hj * cj * rhoj / xi;
            v_sig = (real)19.8 * mi_ * mj_ / (rhoi * rhoj * (mi_ + mj_)) / (r + (real)1e-14 * h);
            break;
        }
        case SPH_VISC_MONAGHAN1997B:
            v_sig = rsqrt_safe(ci * ci + C_q * mu * mu) + rsqrt_safe(cj * cj + C_q * mu * mu) - mu; break;
        case SPH_VISC_DUKOWICZ: v_sig = C_l * c - (real)3 / (real)4 * C_q * mu; break;
        case SPH_VISC_PRICE2012: v_sig = C_l * c - C_q / (real)2 * mu; break;
        case SPH_VISC_PRICE2008: {
            real rb = (rhoi + rhoj) / (real)2;
            v_sig = C_l * rsqrt_safe(FABS(Pi_ - Pj_) / (rb + (real)1e-14 * h));
            break;
        }
        case SPH_VISC_WADSLEY2008: v_sig = C_l * FABS(mu); break;
        default: v_sig = C_l * c - C_q * mu; break;   /* Monaghan1992, 1997a, Price2012_98, DeltaSPH, Default */
    }
    real val = rhoj * (real)1 / rho * v_sig * sf;
    if (o->mswitch && !thermal && ux > 0) val = 0;
    return val;
}

/* Pi_ij for every Verlet entry (tests compare it with the reference's computePi_actual). */
int oracle_pi_pairs(const SphParams* p, int64_t n, const real* x, const real* H, const real* rho, const real* v, const real* c,
                    const real* alpha, const real* Pr, const int32_t* offs, const int32_t* cnt, const int32_t* list, int useJ,
                    int thermal, real* out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D)), ux = 0;
            for (int a = 0; a < D; ++a) ux += (v[i * D + a] - v[(int64_t)j * D + a]) * d[a];
            out[k] = oracle_pi(&o, r, ux, H[i], H[j], rho[i], rho[j], Pr[i], Pr[j], c ? c[i] : o.c_s, c ? c[j] : o.c_s,
                               alpha ? alpha[i] : 1, alpha ? alpha[j] : 1, useJ, thermal);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ CompSPH / Monaghan schemes
 * Omega: modules/adaptiveSupport/wp_omega.py:11-78, :140 (gather support).
 * Cullen divergence: difference divergence, super-symmetric support, V_j = m_j/rho_j
 * (CullenDehnen2010.py:246-257).  Consistent continuity (modules/momentum/consistent.py:
 * 8-35): -(rho_i/Omega_i) * (1/rho_i) sum_j m_j (v_j - v_i).gradW(max(H_i,H_j)) -- the
 * consistentDivergence operator of warpSPHCore is restated as the divergence weighted
 * by m_j/rho_i (parity unpinned for that operator). */
int oracle_compsph_prep(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                        const real* v, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                        real* omega, real* div, real* drhodt) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real Hi = H[i], dh_drho = -Hi / (rho[i] * (real)D), om = 0, sdiv = 0, scon = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            real d[3];
            dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            real W, dWdh;
            kWdH(&o, r, Hi, &W, &dWdh);
            om += dh_drho * m[j] * dWdh;
            if (div || drhodt) {
                real g[3], W2, s = 0;
                kWG(&o, d, r, wmax(Hi, H[j]), &W2, g);
                for (int a = 0; a < D; ++a) s += (v[(int64_t)j * D + a] - v[i * D + a]) * g[a];
                sdiv += m[j] / rho[j] * s;
                scon += m[j] * s;
            }
        }
        real Om = omega ? (real)1 - om : (real)1;
        if (omega) omega[i] = Om;
        if (div) div[i] = sdiv;
        if (drhodt) drhodt[i] = -(rho[i] / Om) * (scon / rho[i]);
    }
    return 0;
}

/* modules/compSPH/accel.py:60-154 and modules/compSPH/dudt.py:60-139 (see the GPU pass). */
int oracle_compsph_accel_dudt(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                              const real* v, const real* c, const real* alpha, const real* Pr, const real* omega,
                              const int32_t* offs, const int32_t* cnt, const int32_t* list,
                              real* dvdt, real* dudt, real* dEdt, real* ap, real* av) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        const real *xi = x + i * D, *vi = v + i * D;
        real Hi = H[i], rhoi = rho[i], Pi = Pr[i];
        real ci = c ? c[i] : o.c_s, ai = alpha ? alpha[i] : 1, omi = omega ? omega[i] : 1;
        real pTi = Pi / (rhoi * rhoi) / omi;
        real acc[3] = {0, 0, 0}, accc[3] = {0, 0, 0}, du = 0, duc = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            const real* vj = v + (int64_t)j * D;
            real d[3];
            dist_vec(&o, xi, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            real Hj = H[j], mj = m[j], rhoj = rho[j], Pj = Pr[j];
            real cj = c ? c[j] : o.c_s, aj = alpha ? alpha[j] : 1, omj = omega ? omega[j] : 1;
            real Vj = mj / rhoj;
            real rho_bar = (real)0.5 * (rhoi + rhoj);
            real ux = 0, uxr = 0;
            for (int a = 0; a < D; ++a) { ux += (vi[a] - vj[a]) * d[a]; uxr += (vj[a] - vi[a]) * d[a]; }
            real pi_i = oracle_pi(&o, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, ci, cj, ai, aj, 0, 0) * (rho_bar / rhoi);
            real pi_j = oracle_pi(&o, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, ci, cj, ai, aj, 1, 0) * (rho_bar / rhoj);
            real Wi, Wj, gi[3], gj[3], gw[3];
            kWG(&o, d, r, Hi, &Wi, gi);
            kWG(&o, d, r, Hj, &Wj, gj);
            for (int a = 0; a < D; ++a) gw[a] = (real)0.5 * (gi[a] + gj[a]);
            real pTj = Pj / (rhoj * rhoj) / omj;
            real mu = uxr / (r + (real)1.0e-14 * Hi);
            real dotg = 0;
            for (int a = 0; a < D; ++a) {
                real pt = -(pTi * gw[a] + pTj * gw[a]) * mj;
                real vt = -(real)0.5 * (pi_i * gw[a] + pi_j * gw[a]) * Vj * mu;
                if (ap) ap[(int64_t)k * D + a] = pt;
                if (av) av[(int64_t)k * D + a] = vt;
                kahan_add(&acc[a], &accc[a], pt + vt, o.kahan);
                dotg += (vj[a] - vi[a]) * gi[a];
            }
            real pTerm = -Vj * pTi * rhoj * dotg;
            real vTerm = -(real)0.5 * Vj * pi_i * mu * dotg;
            kahan_add(&du, &duc, pTerm + vTerm, o.kahan);
        }
        real a_[3], vdot = 0;
        for (int a = 0; a < D; ++a) { a_[a] = acc[a] + accc[a]; vdot += vi[a] * a_[a]; }
        if (dvdt) for (int a = 0; a < D; ++a) dvdt[i * D + a] = a_[a];
        if (dudt) dudt[i] = du + duc;
        if (dEdt) dEdt[i] = m[i] * vdot + m[i] * (du + duc);
    }
    return 0;
}

/* Monaghan scheme (schemes/monaghan.py:77-143), kernel-mean support.  The symmetric
 * pressure gradient with grad-h terms is the warpSPHCore operator restated as
 * rho_i sum_j m_j (P_i/(Omega_i rho_i^2) + P_j/(Omega_j rho_j^2)) gradW (parity unpinned);
 * the viscosity, conductivity and heating pair bodies are wp_diffusion.py:71-107,
 * wp_conductivity.py:59-115 and wp_dissipation.py:59-119.  out5 (nullable) receives the
 * five terms: [pressure (D), viscosity (D), PdV, conductivity, heating] per particle. */
int oracle_monaghan_rhs(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                        const real* v, const real* u, const real* c, const real* alpha, const real* Pr, const real* omega,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list,
                        real* dvdt, real* dudt, real* dEdt, real* out5) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        const real *xi = x + i * D, *vi = v + i * D;
        real Hi = H[i], rhoi = rho[i], Pi = Pr[i], ui = u[i];
        real ci = c ? c[i] : o.c_s, ai = alpha ? alpha[i] : 1, omi = omega ? omega[i] : 1;
        real pTi = Pi / (rhoi * rhoi) / omi;
        real sp[3] = {0, 0, 0}, spc[3] = {0, 0, 0}, sv[3] = {0, 0, 0}, svc[3] = {0, 0, 0};
        real pdv = 0, pdvc = 0, cond = 0, condc = 0, heat = 0, heatc = 0;
        for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
            int32_t j = list[k];
            const real* vj = v + (int64_t)j * D;
            real d[3];
            dist_vec(&o, xi, x + (int64_t)j * D, d);
            real r = rsqrt_safe(dotD(d, d, D));
            real Hj = H[j], mj = m[j], rhoj = rho[j], Pj = Pr[j];
            real cj = c ? c[j] : o.c_s, aj = alpha ? alpha[j] : 1, omj = omega ? omega[j] : 1;
            real Vj = mj / rhoj;
            real ux = 0, uxr = 0;
            for (int a = 0; a < D; ++a) { ux += (vi[a] - vj[a]) * d[a]; uxr += (vj[a] - vi[a]) * d[a]; }
            real pi_v = oracle_pi(&o, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, ci, cj, ai, aj, 0, 0);
            real pi_u = oracle_pi(&o, r, ux, Hi, Hj, rhoi, rhoj, Pi, Pj, ci, cj, ai, aj, 0, 1);
            real Wi, Wj, gi[3], gj[3], gk[3];
            kWG(&o, d, r, Hi, &Wi, gi);
            kWG(&o, d, r, Hj, &Wj, gj);
            for (int a = 0; a < D; ++a) gk[a] = (real)0.5 * (gi[a] + gj[a]);
            real pTj = Pj / (rhoj * rhoj) / omj;
            real den = r + (real)1.0e-14 * Hi;
            real mu = ux / den, mup = uxr / den;
            real dvg = 0, lap = 0;
            for (int a = 0; a < D; ++a) {
                kahan_add(&sp[a], &spc[a], mj * (pTi + pTj) * gk[a], o.kahan);
                kahan_add(&sv[a], &svc[a], Vj * pi_v * gk[a] * mu, o.kahan);
                dvg += (vj[a] - vi[a]) * gk[a];
                lap += gk[a] * (d[a] / den);
            }
            kahan_add(&pdv, &pdvc, mj * dvg, o.kahan);
            kahan_add(&cond, &condc, -(real)0.5 * Vj * pi_u * (u[j] - ui) * lap, o.kahan);
            kahan_add(&heat, &heatc, -Vj * pi_v * (mup * mup) * lap, o.kahan);
        }
        real ap_[3], av_[3], vdot = 0;
        for (int a = 0; a < D; ++a) {
            ap_[a] = -(rhoi * (sp[a] + spc[a])) / rhoi;
            av_[a] = sv[a] + svc[a];
            vdot += vi[a] * (ap_[a] + av_[a]);
        }
        real du_pdv = -(Pi / rhoi / omi) * ((pdv + pdvc) / rhoi);
        real du_cond = cond + condc, du_heat = heat + heatc;
        if (dvdt) for (int a = 0; a < D; ++a) dvdt[i * D + a] = ap_[a] + av_[a];
        if (dudt) dudt[i] = du_pdv + du_cond + du_heat;
        if (dEdt) dEdt[i] = m[i] * vdot + m[i] * (du_pdv + du_cond);
        if (out5) {
            real* q = out5 + i * (2 * D + 3);
            for (int a = 0; a < D; ++a) { q[a] = ap_[a]; q[D + a] = av_[a]; }
            q[2 * D] = du_pdv; q[2 * D + 1] = du_cond; q[2 * D + 2] = du_heat;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ helpers exported for tests */
int oracle_real_size(void) { return (int)sizeof(real); }
int oracle_kernel_eval(int kernel, int dim, int64_t n, const real* r, real H, real* W, real* dWdr, real* dWdH) {
    SphParams p;
    memset(&p, 0, sizeof(p));
    p.kernel = kernel; p.dim = dim;
    OP o = op_from(&p);
    for (int64_t i = 0; i < n; ++i) {
        real q = r[i] / H;
        if (!(q < 1)) { W[i] = 0; dWdr[i] = 0; dWdH[i] = 0; continue; }
        real k, pq; kernel_kp(kernel, dim, q, &k, &pq);
        real cH = kernel_C(kernel, dim) / ipowD(H, dim);
        W[i] = cH * k;
        dWdr[i] = -cH / H * q * pq;
        real Wd, dh; kWdH(&o, r[i], H, &Wd, &dh);
        dWdH[i] = dh;
    }
    return 0;
}

/* sizeof / offsetof probes so tests can check the ctypes mirror of SphParams */
#include <stddef.h>
int64_t oracle_params_layout(int which) {
    switch (which) {
        case 0: return (int64_t)sizeof(SphParams);
        case 1: return (int64_t)offsetof(SphParams, dim);
        case 2: return (int64_t)offsetof(SphParams, kahan);
        case 3: return (int64_t)offsetof(SphParams, target_neighbors);
        case 4: return (int64_t)offsetof(SphParams, energy_scheme);
        default: return -1;
    }
}

/* ------------------------------------------------------------------ mDBC (wall particles)
 * Liu-Liu moments at the ghost points, modules/liu/wp_mat.py:9-135 (computeLiuMatrices_Func_i)
 * under the scatter support H_j and the FluidToGhost direction (fluid neighbours only):
 *   b = sum_j V_j rho_j [W, grad W],  A = sum_j V_j [[W, -x_gj W], [grad W, -x_gj (x) grad W]],
 * nbrs = #{j : r < H_j}.  Rows of particles that are not ghosts (kind != 2) are zero.  The
 * pseudo-inverse and the density formula of density2025.py are in oracle.py. */
int oracle_liu_moments(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* rho,
                       const int32_t* kinds, const int32_t* offs, const int32_t* cnt, const int32_t* list, real* b_out,
                       real* A_out, int32_t* nbrs_out) {
    OP o = op_from(p);
    int D = o.dim, E = D + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real b[4] = {0, 0, 0, 0}, A[4][4];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 4; ++c) A[a][c] = 0;
        int nb = 0;
        if (kinds[i] == 2) {
            for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
                int32_t j = list[k];
                if (kinds[j] != 0) continue;
                real d[3], W, gw[3];
                dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
                real r = rsqrt_safe(dotD(d, d, D));
                kWG(&o, d, r, H[j], &W, gw);
                real Vj = m[j] / rho[j];
                real VQ = Vj * rho[j];
                b[0] += VQ * W;
                A[0][0] += Vj * W;
                for (int a = 0; a < D; ++a) {
                    b[a + 1] += VQ * gw[a];
                    A[a + 1][0] += Vj * gw[a];
                    A[0][a + 1] += -Vj * d[a] * W;
                    for (int c = 0; c < D; ++c) A[a + 1][c + 1] += -Vj * d[a] * gw[c];
                }
                if (r < H[j]) ++nb;
            }
        }
        for (int a = 0; a < E; ++a) {
            b_out[i * E + a] = b[a];
            for (int c = 0; c < E; ++c) A_out[(i * E + a) * E + c] = A[a][c];
        }
        nbrs_out[i] = nb;
    }
    return 0;
}

/* No-penetration shift, modules/mdbc/wp_nopenshift.py:187-307 (computeMdbcNoPenShift_Func_i)
 * and its kernel's per-axis average (:400-420): fluid query particles, wall neighbours
 * (BoundaryToFluid), gather support.  Rows that are not fluid are zero. */
int oracle_mdbc_nopen_shift(const SphParams* p, int64_t n, const real* x, const real* H, const real* m, const real* v,
                            const int32_t* kinds, const real* ghost_off, const int32_t* offs, const int32_t* cnt,
                            const int32_t* list, real* out) {
    OP o = op_from(p);
    int D = o.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        real acc[3] = {0, 0, 0}, ctr[3] = {0, 0, 0};
        if (kinds[i] == 0) {
            real dp = POW(m[i], (real)1 / (real)D);
            for (int32_t k = offs[i]; k < offs[i] + cnt[i]; ++k) {
                int32_t j = list[k];
                if (kinds[j] != 1) continue;
                real d[3];
                dist_vec(&o, x + i * D, x + (int64_t)j * D, d);
                real r = rsqrt_safe(dotD(d, d, D));
                if (!(kW(&o, r, H[i]) > 0)) continue;
                real on = 0, nj[3], normDist = 0;
                for (int a = 0; a < D; ++a) on += ghost_off[(int64_t)j * D + a] * ghost_off[(int64_t)j * D + a];
                real norm_j = rsqrt_safe(on) + (real)1e-12;
                for (int a = 0; a < D; ++a) { nj[a] = -ghost_off[(int64_t)j * D + a] / norm_j; normDist += d[a] * nj[a]; }
                int cab = (r < (real)1.25 * dp) && (FABS(normDist) < (real)0.75 * norm_j && norm_j < (real)1.75 * dp);
                for (int a = 0; a < D; ++a) {
                    real dv = v[i * D + a] - v[(int64_t)j * D + a], nrm = nj[a], dr = d[a];
                    int mask = cab && (dr * nrm < (real)0.75) && (FABS(nrm) > (real)0.001 * dp);
                    real vfc = dv * nrm;
                    real ratio = FABS(dr / nrm);
                    ratio = ratio < (real)0.25 ? (real)0.25 : (ratio > 1 ? 1 : ratio);
                    real factor = (real)-4 * ratio + 3;
                    real term = -factor * dv * nrm * nrm;
                    if (mask && vfc < 0) { acc[a] += term; ctr[a] += 1; }
                }
            }
        }
        for (int a = 0; a < D; ++a) out[i * D + a] = acc[a] / (ctr[a] + (real)1e-12);
    }
    return 0;
}
