/*
 * warpsph_b200.h -- C ABI of libwarpsph_b200.so, the sm_100a implementation of the
 * warpSPH per-step particle hot path (neighbour search, SPH pair interactions,
 * DFSPH Jacobi solves, integrator update and CFL time step).
 *
 * Conventions shared by every entry point
 *   - All array arguments are DEVICE pointers (allocated by the caller, e.g. torch).
 *     The library never allocates in these calls and never frees caller memory.
 *   - Positions and other per-particle vectors are row-major [n, dim] float arrays,
 *     per-particle matrices are row-major [n, dim, dim]; M[a][b] = d(field^a)/dx^b.
 *   - Neighbour lists are CSR: neighbor_offsets[n], num_neighbors[n] (int32) and
 *     neighbor_list[nnz] (int32, original particle indices).  Row i lists every j
 *     with |x_i - x_j| < verlet_scale * max(H_i, H_j) (i itself included), ordered
 *     by stencil cell (offsets -1, 0, +1 per axis, x fastest) and, inside a cell, by
 *     ascending position in the cell-sorted order.
 *   - `stream` is a cudaStream_t passed as void*; work is enqueued asynchronously.
 *   - Scalars that change every step (dt) are read from DEVICE memory so a step can
 *     be captured in a CUDA graph without host round trips.
 *   - Return value: SPH_OK (0) or a negative SPH_ERR_* code; sph_last_error_string()
 *     describes the last failure of the calling thread.
 *   - Every entry point accepts n == 0 and then does nothing.
 *
 * Reference interface: wi-re/warpSPH (Python + NVIDIA Warp).  Each declaration names
 * the reference function it replaces, relative to the reference's project root.
 */
#ifndef WARPSPH_B200_H
#define WARPSPH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define SPH_OK                  0
#define SPH_ERR_BAD_ARG        -1   /* null pointer, bad enum, misaligned array, n < 0 */
#define SPH_ERR_WORKSPACE      -2   /* caller workspace smaller than *_workspace_size */
#define SPH_ERR_CAPACITY       -3   /* neighbour list capacity exceeded (device flag) */
#define SPH_ERR_CUDA           -4   /* a CUDA launch failed */
#define SPH_ERR_NOT_CONVERGED  -5   /* Jacobi solve hit its iteration cap */
#define SPH_ERR_TIMEOUT        -6   /* a bounded device wait gave up */
#define SPH_ERR_NONFINITE      -7   /* NaN/Inf detected in a reduction */
#define SPH_ERR_UNSUPPORTED    -8   /* option not implemented on this path */

/* device status word bits (written by kernels into a caller-provided int32) */
#define SPH_STATUS_LIST_OVERFLOW   0x1
#define SPH_STATUS_NONFINITE       0x2
#define SPH_STATUS_NOT_CONVERGED   0x4
#define SPH_STATUS_TIMEOUT         0x8
#define SPH_STATUS_LIST_STALE      0x10

/* ---------------------------------------------------------------- enumerations */
/* Kernel functions (warpSPHCore KernelFunctions; names as used in
 * configurations/simulationConfig.py:25). */
#define SPH_KERNEL_WENDLAND2 1
#define SPH_KERNEL_WENDLAND4 2
#define SPH_KERNEL_WENDLAND6 3
/* B7: the degree-7 B-spline (eight intervals, knots at q = 1/4, 1/2, 3/4), the kernel of
 * the reference's compressible notebooks (e.g. examples/compressible/01-Sod_Shock_Tube_1D.ipynb). */
#define SPH_KERNEL_B7        4

/* Support schemes (warpSPHCore SupportScheme): h used for the pair kernel value. */
#define SPH_SUPPORT_GATHER               0   /* H_i */
#define SPH_SUPPORT_SCATTER              1   /* H_j */
#define SPH_SUPPORT_SYMMETRIC            2   /* W(r, (H_i+H_j)/2) */
#define SPH_SUPPORT_SUPERSYMMETRIC       3   /* W(r, max(H_i, H_j)) */
#define SPH_SUPPORT_KERNELMEANSYMMETRIC  4   /* (W(r,H_i) + W(r,H_j)) / 2 */

/* Energy partition schemes (enumTypes.py:5-11, same values). */
#define SPH_ENERGY_EQUALWORK   0
#define SPH_ENERGY_PDV         1
#define SPH_ENERGY_DIMINISHING 2
#define SPH_ENERGY_MONOTONIC   3
#define SPH_ENERGY_HYBRID      4
#define SPH_ENERGY_CRK         5

/* Artificial viscosity terms (configurations/moduleConfigurations/diffusionParameters.py:8-20). */
#define SPH_VISC_DEFAULT              0
#define SPH_VISC_MONAGHANGINGOLD1983  1
#define SPH_VISC_CLEARY1998           2
#define SPH_VISC_MONAGHAN1992         3
#define SPH_VISC_MONAGHAN1997A        4
#define SPH_VISC_MONAGHAN1997B        5
#define SPH_VISC_DUKOWICZ             6
#define SPH_VISC_PRICE2012_98         7
#define SPH_VISC_PRICE2012            8
#define SPH_VISC_PRICE2008            9
#define SPH_VISC_WADSLEY2008         10
#define SPH_VISC_DELTASPH            11

/* ---------------------------------------------------------------- parameters */
/* Plain-old-data parameter block.  Doubles first so the layout has no padding
 * surprises for ctypes; the GPU path rounds them to float at launch. */
typedef struct SphParams {
    /* domain (utils/domain.py:7-22 DomainDescription) */
    double domain_min[3];
    double domain_max[3];
    double verlet_scale;              /* simulationConfig.py:24 */
    /* DiffusionParameters (configurations/moduleConfigurations/diffusionParameters.py:22-37) */
    double C_l, C_q, Cu_l, Cu_q, K;
    /* CRKViscosity (configurations/crkSPH.py:16-25) */
    double eta_crit, eta_fold;
    /* compressible scheme (configurations/compressibleConfig.py:16-30) */
    double gamma;
    /* ViscositySwitchConfig (configurations/moduleConfigurations/viscositySwitchParameters.py:11-26) */
    double alpha_min, alpha_max, beta_xi;
    /* adaptive support and time step (simulationConfig.py:28-38) */
    double target_neighbors;
    double cfl, min_dt, max_dt, dt_growth;
    /* DiffusionParameters.c_s: the sound speed of the viscosity terms when no per-particle
     * sound speeds are passed (diffusionParameters.py:24) */
    double c_s;
    /* ViscositySwitchConfig.beta_c, beta_d of the Cullen-Hopkins switch
     * (viscositySwitchParameters.py:21-22) */
    double beta_c, beta_d;
    double reserved_d[5];
    /* integers */
    int32_t dim;                      /* 1, 2 or 3 */
    int32_t kernel;                   /* SPH_KERNEL_* */
    int32_t periodic[3];
    int32_t viscosity_term;           /* SPH_VISC_* */
    int32_t monaghan_switch, correct_xi, scale_beta;
    int32_t enable_crk_limiter, enable_vanleer_limiter, force_vanleer_off, force_vanleer_on;
    int32_t energy_scheme;            /* SPH_ENERGY_* */
    int32_t limit_xi;
    int32_t kahan;                    /* 1: compensated accumulation of dv/dt and du/dt */
    /* Layout of the `list` argument of the pair entry points: 1 (or 0), rows of int32
     * neighbour indices j.  A pass walks whole Verlet rows (cnt = Verlet counts) or their
     * interacting prefixes (cnt = interacting counts from sph_neighbors_build); pairwise
     * outputs/inputs (ap_ij, av_ij, f_ij) are indexed by the Verlet entry either way. */
    int32_t list_stride;
    /* DiffusionParameters.thermalConducitiyTerm (SPH_VISC_*): the signal-velocity form of
     * the artificial conductivity (diffusionParameters.py:33, pi.py:63) */
    int32_t conductivity_term;
    /* ViscositySwitchParameters.correctVelocityGradient (CullenHopkins.py:19-34): the
     * Cullen-Hopkins velocity gradient is multiplied by pinv(M) of the CRKSPH moment matrix
     * M_i = -sum_j m_j x_ij (x) grad W(r_ij, H_i) (common.py:10-25, wp_computeM.py:55-86) */
    int32_t correct_velocity_gradient;
    int32_t reserved_i[5];
} SphParams;

/* ---------------------------------------------------------------- library */
const char* sph_version(void);
const char* sph_last_error_string(void);
/* Number of CUDA kernels this library has launched in the process (all threads); a launch
 * recorded into a CUDA graph counts once, when it is recorded. */
int64_t sph_launch_count(void);
/* Of those, the launches recorded into the rebuild bodies of graph conditional nodes
 * (sph_neighbors_update during a capture): a replay runs them only when it rebuilds. */
int64_t sph_launch_count_conditional(void);
/* Kernel-function constants used by the library (normalisation C_d, kernel scale
 * H/h = 1/(2 sigma), Dehnen & Aly 2012 Table 1). Host-only, no GPU needed. */
int sph_kernel_constants(int32_t kernel, int32_t dim, double* norm_out, double* scale_out);

/* ---------------------------------------------------------------- (a) neighbour search */
/* Workspace bytes for sph_neighbors_build with `cell_capacity` dense cells. */
int sph_neighbors_workspace_size(const SphParams* p, int64_t n, int64_t cell_capacity,
                                 int64_t* bytes_out);

/* Replaces warpSPHCore buildVerletList (called at schemes/crkSPH.py:54-58,
 * schemes/compSPH.py:42-46, schemes/dfsph.py:29-33): Morton-keyed dense cell grid
 * of cell size >= verlet_scale*max(H), counting sort by (cell key, index) (atomic
 * scatter + in-cell rank), cell offset table, then count -> scan -> fill of the CSR
 * Verlet list over position/support records gathered in sorted order.
 * Outputs: sort_index[n] (original index of the k-th sorted particle),
 * sorted_keys[n] (its Morton cell key), cell_begin/cell_end[cell_capacity],
 * CSR arrays, *nnz_out (device int64).
 * Interacting prefix (inter_counts non-null): each row holds first the entries with
 * fl(sqrt(r^2))/max(H_i,H_j) < 1 -- every pair any support scheme gives a non-zero
 * kernel value -- then the rest of its Verlet entries, both parts in walk order
 * (stencil cells in offset order, candidates by sorted position); inter_counts[i] is the
 * length of the prefix and *inter_nnz_out their sum.  Without inter_counts the rows are
 * in walk order.  If the Verlet list exceeds list_capacity nothing is filled,
 * SPH_STATUS_LIST_OVERFLOW is or-ed into *status (device int32) and *nnz_out holds the
 * required size.
 * grid_out (device, 8 int32): grid dims, bits per axis, cell size as float bits, dim. */
int sph_neighbors_build(const SphParams* p, int64_t n, const float* x, const float* H,
                        void* workspace, int64_t workspace_bytes, int64_t cell_capacity,
                        int32_t* sort_index, uint32_t* sorted_keys,
                        int32_t* cell_begin, int32_t* cell_end, int32_t* grid_out,
                        int32_t* neighbor_offsets, int32_t* num_neighbors,
                        int32_t* neighbor_list, int64_t list_capacity, int64_t* nnz_out,
                        int32_t* inter_counts, int64_t* inter_nnz_out,
                        int32_t* status, void* stream);

/* Prior-list reuse (the validity check warpSPHCore buildVerletList performs before
 * rebuilding; its rule is restated here): a list built at (x0, H0) with verlet_scale vs
 * still holds every pair with |x_i - x_j| < max(H_i, H_j) at (x, H) when
 * max_k (H_k - vs H0_k) + 2 max_k |x_k - x0_k| <= 0 (a 1e-5 relative margin is kept
 * for rounding).  When that holds, every row of neighbor_list is rewritten into
 * list_out (same offsets and counts; list_out must not alias neighbor_list, which
 * earlier stages may still reference) with its interacting entries for (x, H) first,
 * in the kept order, and the rest after them in reverse kept order; inter_counts and
 * *inter_nnz_out receive the prefix lengths and their sum.  Otherwise
 * SPH_STATUS_LIST_STALE is or-ed into *status and the caller rebuilds.  With
 * list_out == NULL only the verdict is computed (the rows can be rewritten by a later
 * call, when a pass needs them).  scratch: device memory of 4 uint32 words. */
int sph_neighbors_refresh(const SphParams* p, int64_t n, const float* x, const float* H,
                          const float* x0, const float* H0,
                          const int32_t* neighbor_offsets, const int32_t* num_neighbors,
                          const int32_t* neighbor_list, int32_t* list_out, int32_t* inter_counts,
                          uint32_t* scratch, int64_t* inter_nnz_out, int32_t* status, void* stream);

/* sph_neighbors_refresh with list_out set, fused with the CRK volume of the rewritten
 * rows (computeCRKFactors, schemes/crkSPH.py:61: V_i = 1 / sum_j W(r_ij, H_j), the
 * scatter support): V_out [n] receives the volumes that sph_crk_volume gives on the
 * rewritten rows, summed in the row's original order.  The other arguments are those
 * of sph_neighbors_refresh; list_out, inter_counts and inter_nnz_out are required. */
int sph_neighbors_refresh_volume(const SphParams* p, int64_t n, const float* x, const float* H,
                                 const float* x0, const float* H0,
                                 const int32_t* neighbor_offsets, const int32_t* num_neighbors,
                                 const int32_t* neighbor_list, int32_t* list_out,
                                 int32_t* inter_counts, uint32_t* scratch, int64_t* inter_nnz_out,
                                 int32_t* status, float* V_out, void* stream);

/* Device-decided list update for a stepping loop that never reads the device: replaces
 * the host-side keep-or-rebuild decision of buildVerletList (schemes/crkSPH.py:54-58 in the
 * reference rebuilds every call).  The Verlet rows (neighbor_offsets, num_neighbors,
 * neighbor_list, nnz) are kept across calls together with the positions x0 [n, dim] and
 * supports H0 [n] they were built from.  One call checks them for (x, H) as
 * sph_neighbors_refresh does (verdict: 4 words, zeroed once at allocation) and, when a
 * particle has left the Verlet skin, rebuilds them in place on the GPU (every build launch
 * returns at once when the rows are kept) and copies x, H into x0, H0.  Initialise H0 with zeros (or anything
 * non-finite) to force the first build.  The rows are in no particular order:
 * sph_neighbors_rewrite gives the interacting prefixes.  When a rebuild needs more than
 * list_capacity entries the status word gets SPH_STATUS_LIST_OVERFLOW and every row is cut
 * to fit (the results of the walks that follow are then wrong but stay in bounds): read the
 * status word at some later point and redo the work from a saved state with a larger list.
 * Zero-fill neighbor_list once at allocation.  rebuilds (optional, one int64 on the device) is
 * incremented by every rebuild.  Called on a stream that is being captured into a CUDA graph,
 * the rebuild is recorded as the body of an IF conditional node whose condition the last block
 * of the validity check sets from the verdict (and zeroes the verdict words for the next
 * replay), so a replay that keeps the rows skips it; its body is captured on a
 * private stream per device, created by the first call outside a capture (make one before
 * capturing; without it the gated launches are recorded instead). */
int sph_neighbors_update(const SphParams* p, int64_t n, const float* x, const float* H,
                         float* x0, float* H0, void* workspace, int64_t workspace_bytes,
                         int64_t cell_capacity, int32_t* sort_index, uint32_t* sorted_keys,
                         int32_t* cell_begin, int32_t* cell_end, int32_t* grid_out,
                         int32_t* neighbor_offsets, int32_t* num_neighbors, int32_t* neighbor_list,
                         int64_t list_capacity, int64_t* nnz, uint32_t* verdict, int32_t* status,
                         int64_t* rebuilds, void* stream);

/* Rewrites the rows of a list valid for (x, H) into list_out (same offsets, capacity of the
 * input list) with the interacting entries (fl(sqrt(r^2)) / max(H_i, H_j) < 1) first, in row
 * order, and the rest after them, as sph_neighbors_refresh does, with no validity check.
 * offsets_out / counts_out [n] receive copies of the rows' offsets and lengths (so that a
 * later rebuild of the input rows leaves this list intact), inter_counts [n] the prefix
 * lengths, inter_nnz_out their sum.  With V_out the CRK volumes of the rows are computed in
 * the same pass, as in sph_neighbors_refresh_volume. */
int sph_neighbors_rewrite(const SphParams* p, int64_t n, const float* x, const float* H,
                          const int32_t* neighbor_offsets, const int32_t* num_neighbors,
                          const int32_t* neighbor_list, int32_t* list_out, int32_t* offsets_out,
                          int32_t* counts_out, int32_t* inter_counts, int64_t* inter_nnz_out,
                          float* V_out, int32_t* status, void* stream);

/* Expands CSR rows into the reference's AdjacencyList.i / .j int64 arrays
 * (io.py:8-20 field names). */
int sph_neighbors_expand(int64_t n, const int32_t* neighbor_offsets, const int32_t* num_neighbors,
                         const int32_t* neighbor_list, int64_t nnz,
                         int64_t* i_out, int64_t* j_out, void* stream);

/* ---------------------------------------------------------------- (b) pair interactions */
/* Density summation rho_i = sum_j m_j W(r_ij, h_ij) with the given support scheme.
 * Replaces warpOperation(Density) (modules/density/density.py:16-28). */
int sph_density_gather(const SphParams* p, int64_t n, int32_t support_mode,
                       const float* x, const float* H, const float* m,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list,
                       float* rho_out, void* stream);

/* One iteration of the Owen adaptive support (modules/adaptiveSupport/optimalSupportOwen.py:
 * 70-108; replaces computePsi0Warp, wp_psi0.py:173, and the table lookup and update):
 * psi0 and psi0H of wp_psi0.py:46-98 (gather support, W and |grad W| scaled by h^d and
 * h^(d+1), each sum to the power 1/d), n_h from the table (lut_psiH[nlut] ascending ->
 * lut_nh[nlut], device FP64; owenLUT.py:6-12), then H_new = (1 - a + a s) H with
 * s = target_nh / n_h and a = 0.4 (1 + s^-3) (s >= 1) or 0.4 (1 + s^2)
 * (optimalSupportOwen.py:27-33), clamped to [hbounds[0]/4, 4*hbounds[1]].  psi0_out,
 * psiH_out and ratio_out (= H_new/H) may be null.  The rows must cover every pair within
 * H_i (Verlet rows, or interacting prefixes for the current supports). */
int sph_owen_iter(const SphParams* p, int64_t n, const float* x, const float* H,
                  const int32_t* offs, const int32_t* cnt, const int32_t* list,
                  const double* lut_nh, const double* lut_psiH, int32_t nlut, double target_nh,
                  const float* hbounds, float* psi0_out, float* psiH_out, float* H_out,
                  float* ratio_out, void* stream);

/* One Monaghan Newton iteration of the adaptive support
 * (modules/adaptiveSupport/optimalSupportMonaghan.py:87-125 with the Omega kernel
 * modules/adaptiveSupport/wp_omega.py:10-60): gather density, Omega = dF/dh,
 * H_new = clamp(H - F/(Omega+1e-6), hbounds[0]/4, 4*hbounds[1]).
 * hbounds (device float[2]) holds min/max of H on entry; ratio_out[n] = H_new/(H+1e-6). */
int sph_adaptive_h_iter(const SphParams* p, int64_t n, int32_t support_mode,
                        const float* x, const float* H, const float* m,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list,
                        const float* hbounds, float* rho_out, float* H_out, float* ratio_out,
                        void* stream);

/* min and max of a device array into out2[0], out2[1] (device). */
int sph_minmax(int64_t n, const float* a, float* out2, void* stream);

/* CRK apparent volume V_i = 1 / sum_j W(r_ij, H_j)  (warpSPHCore crk_volume,
 * called through computeCRKFactors at schemes/crkSPH.py:61). */
int sph_crk_volume(const SphParams* p, int64_t n, const float* x, const float* H,
                   const int32_t* offs, const int32_t* cnt, const int32_t* list,
                   float* V_out, void* stream);

/* CRK correction coefficients A, B, gradA, gradB (Frontiere, Raskin & Owen 2017)
 * from the moments m0, m1, m2 and their gradients, solved in FP64, and the CRK
 * density rho_i = sum_j m_j A_i (1 + B_i.x_ij) W(r_ij, H_j)  (warpSPHCore
 * crk_moments / crk_density via computeCRKFactors, schemes/crkSPH.py:61). */
int sph_crk_factors(const SphParams* p, int64_t n, const float* x, const float* H,
                    const float* m, const float* V,
                    const int32_t* offs, const int32_t* cnt, const int32_t* list,
                    float* A, float* B, float* gradA, float* gradB, float* rho_out,
                    void* stream);

/* sph_crk_factors with the ideal-gas EOS of its density fused into the same pass
 * (modules/eos/idealGas.py:16-36, as sph_eos_ideal_gas computes it): from u [n] it writes
 * entropy_out, P_out and c_out [n] (each optional), gamma from p. */
int sph_crk_factors_eos(const SphParams* p, int64_t n, const float* x, const float* H,
                        const float* m, const float* V, const int32_t* offs, const int32_t* cnt,
                        const int32_t* list, float* A, float* B, float* gradA, float* gradB,
                        float* rho_out, const float* u, float* entropy_out, float* P_out,
                        float* c_out, void* stream);

/* Ideal-gas EOS (modules/eos/idealGas.py:6-38 with u and rho given). */
int sph_eos_ideal_gas(const SphParams* p, int64_t n, const float* u, const float* rho,
                      float* A_out, float* P_out, float* c_out, void* stream);

/* CRK velocity gradient DvDx[i][a][b] = sum_j V_j (v_j^a - v_i^a) dW^R_ij/dx^b
 * (scatter support, difference form; schemes/crkSPH.py:158-172 incl. the .mT),
 * drhodt = -tr(DvDx) rho.  When div_out/vsig_out are non-null the same pass also
 * computes the Cullen-Dehnen divergence (super-symmetric, m_j/rho_j volumes;
 * modules/shockCapturing/CullenDehnen2010.py:246-257) and the signal velocity
 * max_j (c_bar - mu_ij) (modules/shockCapturing/wp_vsig.py:11-90). */
int sph_grad_v(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
               const float* rho, const float* V, const float* A, const float* B,
               const float* gradA, const float* gradB, const float* v, const float* c,
               const int32_t* offs, const int32_t* cnt, const int32_t* list,
               float* DvDx_out, float* drhodt_out, float* div_out, float* vsig_out,
               void* stream);

/* Cullen & Dehnen 2010 switch (modules/shockCapturing/CullenDehnen2010.py:218-331):
 * R pass (gather interpolation of m_j sgn(div_j)), Xi limiter, A_i, alpha_loc,
 * and the alpha0 relaxation with tau = h/(2*0.05*v_sig*xi).  div_prev is the
 * state's previous divergence, alpha0_prev the state's alpha0s.  When vsig is
 * NULL the signal velocity max_j (c_bar - mu_ij) (modules/shockCapturing/wp_vsig.py:11-90)
 * is computed in the same pass from v and c over the Verlet set -- `list` must then
 * be the Verlet list (stride 1) -- and written to vsig_out when non-null.
 * Outputs the new alphas (the reference returns alpha0s as alphas, crkSPH.py:195-200). */
int sph_switch_cullen(const SphParams* p, int64_t n, const float* x, const float* H,
                      const float* m, const float* rho, const float* div, const float* div_prev,
                      const float* vsig, const float* v, const float* c,
                      const float* alpha0_prev, const float* dt,
                      const int32_t* offs, const int32_t* cnt, const int32_t* list,
                      float* alpha_out, float* R_out, float* vsig_out, void* stream);

/* Cullen-Hopkins switch, first part (modules/shockCapturing/CullenHopkins.py:7-45,
 * computeHopkinsTerms without the optional velocity-gradient correction): the gather
 * difference velocity gradient, its divergence (div_out) and tr(S S^T) of its traceless
 * symmetric part (shear2_out), then R (gather, CullenDehnen2010.py:121-164), Xi with the
 * shear term (:166-191) and alpha_out = max(Xi alpha0, alpha_min).  The rows must cover
 * the pairs within H_i.  R_out may be null. */
int sph_switch_hopkins_terms(const SphParams* p, int64_t n, const float* x, const float* H,
                             const float* m, const float* rho, const float* v, const float* alpha0,
                             const int32_t* offs, const int32_t* cnt, const int32_t* list,
                             float* div_out, float* shear2_out, float* alpha_out, float* R_out,
                             void* stream);
/* Cullen-Hopkins switch, second part (computeHopkinsUpdate, CullenHopkins.py:48-149):
 * v_sig over the Verlet rows (pass whole rows), d(div)/dt = (div - div_prev)/dt,
 * alpha_tmp = alpha_max |d div/dt| / (|d div/dt| + beta_c c^2 / (h/xi)^2 + 1e-14), zero
 * where d div/dt > 0 or div > 0, and alpha0_out = alpha_tmp where alpha_tmp >= alpha0,
 * else alpha_tmp + (alpha0 - alpha_tmp) exp(-beta_d dt v_sig / (2 h/xi)).  dt is a
 * device float; vsig_out may be null. */
int sph_switch_hopkins_update(const SphParams* p, int64_t n, const float* x, const float* H,
                              const float* v, const float* c, const float* div, const float* div_prev,
                              const float* alpha0, const float* dt,
                              const int32_t* offs, const int32_t* cnt, const int32_t* list,
                              float* alpha0_out, float* vsig_out, void* stream);

/* Balsara 1995 switch alpha = clamp(|div v| / (|div v| + |curl v| + 1e-4 c), 0, 1)
 * with CRK difference-form divergence and curl (formula restated from the comment
 * at schemes/crkSPH.py:132-133; the reference dispatcher rejects it,
 * modules/shockCapturing/wrapper.py:25-32). DvDx from sph_grad_v. */
int sph_switch_balsara(const SphParams* p, int64_t n, const float* DvDx, const float* c,
                       float* alpha_out, void* stream);

/* CRKSPH momentum and energy RHS in one pair pass:
 * modules/crk/accel.py:15-250 (dv/dt and the pairwise ap_ij, av_ij [nnz, dim]) and
 * modules/crk/dudt.py:15-229 (du/dt), with dEdt [n] = m v.dv/dt + m du/dt
 * (schemes/crkSPH.py:330).  Any of dvdt_out, dudt_out, dEdt_out, ap_ij, av_ij may be
 * null.  With p->kahan the per-particle sums are Neumaier-compensated.  Walking the
 * interacting prefixes (cnt = interacting counts), pass verlet_cnt = the Verlet counts
 * and the rest of each row of ap_ij / av_ij is written as zeros; with verlet_cnt NULL
 * only the walked entries are written. */
int sph_crk_accel_dudt(const SphParams* p, int64_t n, const float* x, const float* H,
                       const float* m, const float* rho, const float* V,
                       const float* A, const float* B, const float* gradA, const float* gradB,
                       const float* v, const float* c, const float* P, const float* DvDx,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list,
                       const int32_t* verlet_cnt, float* dvdt_out, float* dudt_out,
                       float* dEdt_out, float* ap_ij, float* av_ij, void* stream);
/* The same pass over packed particle records: a first launch copies the fields the pass
 * reads into records [n, R] (R = sph_crk_record_floats(dim) floats per particle: 12, 24
 * and 36 in 1D, 2D and 3D; 16-byte aligned, caller-owned scratch), and the pair launch
 * gathers each neighbour as R/4 128-bit loads from that one record.  Outputs and
 * arguments otherwise as sph_crk_accel_dudt. */
int sph_crk_record_floats(int32_t dim);
int sph_crk_accel_dudt_packed(const SphParams* p, int64_t n, const float* x, const float* H,
                              const float* m, const float* rho, const float* V,
                              const float* A, const float* B, const float* gradA, const float* gradB,
                              const float* v, const float* c, const float* P, const float* DvDx,
                              const int32_t* offs, const int32_t* cnt, const int32_t* list,
                              const int32_t* verlet_cnt, float* dvdt_out, float* dudt_out,
                              float* dEdt_out, float* ap_ij, float* av_ij, float* records,
                              void* stream);
/* Same pass, separate names for callers that bind the reference's two wrappers
 * computeCrkSPHAccelWarp (modules/crk/accel.py:391) and computeCrkSPHdudtWarp
 * (modules/crk/dudt.py:364). */
int sph_crk_accel(const SphParams* p, int64_t n, const float* x, const float* H,
                  const float* m, const float* rho, const float* V,
                  const float* A, const float* B, const float* gradA, const float* gradB,
                  const float* v, const float* c, const float* P, const float* DvDx,
                  const int32_t* offs, const int32_t* cnt, const int32_t* list,
                  const int32_t* verlet_cnt, float* dvdt_out, float* ap_ij, float* av_ij,
                  void* stream);
int sph_crk_dudt(const SphParams* p, int64_t n, const float* x, const float* H,
                 const float* m, const float* rho, const float* V,
                 const float* A, const float* B, const float* gradA, const float* gradB,
                 const float* v, const float* c, const float* P, const float* DvDx,
                 const int32_t* offs, const int32_t* cnt, const int32_t* list,
                 float* dudt_out, void* stream);

/* ---------------------------------------------------------------- CompSPH / Monaghan schemes */
/* One walk of each row for three of the reference's passes (schemes/compSPH.py:89-97,
 * :105-110 and :162-169; schemes/monaghan.py:59-101):
 *   omega_out  grad-h Omega_i = 1 - sum_j (-H_i/(rho_i d)) m_j dW/dH(r_ij, H_i), gather
 *              support -- replaces computeOmegaWarp (modules/adaptiveSupport/wp_omega.py:175);
 *   div_out    difference divergence sum_j m_j/rho_j (v_j - v_i).grad W(r_ij, max(H_i,H_j)) of
 *              the Cullen switch (modules/shockCapturing/CullenDehnen2010.py:246-257);
 *   drhodt_out consistent continuity -(1/Omega_i) sum_j m_j (v_j - v_i).grad W(r_ij, max(H_i,H_j))
 *              -- replaces computeMomentumConsistent_warp (modules/momentum/consistent.py:8-35);
 *              Omega = 1 when omega_out is null (no grad-h corrections).
 * Any output may be null; v may be null when only omega_out is requested. */
int sph_compsph_prep(const SphParams* p, int64_t n, const float* x, const float* H,
                     const float* m, const float* rho, const float* v,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list,
                     float* omega_out, float* div_out, float* drhodt_out, void* stream);
/* Omega alone, for callers that bind computeOmegaWarp (wp_omega.py:175). */
int sph_grad_h_omega(const SphParams* p, int64_t n, const float* x, const float* H,
                     const float* m, const float* rho,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list,
                     float* omega_out, void* stream);

/* CompSPH momentum and energy right-hand sides in one pass -- replaces
 * computeCompSPHAccelWarp (modules/compSPH/accel.py:284) and computeCompSPHdudtWarp
 * (modules/compSPH/dudt.py:224): per pair the kernel-mean gradient, grad-h pressure
 * terms P/(rho^2 Omega), and the artificial viscosity Pi of computePi_actual
 * (modules/dissipation/pi.py:11-161, the p->viscosity_term form) scaled by rho_bar/rho;
 * du/dt with the gather gradient.  c, alpha and omega may be null (c_s, 1 and 1, as the
 * reference does without sound speeds, switch or grad-h state).  Outputs:
 * dvdt [n*dim], dudt [n], dEdt [n] = m v.dvdt + m dudt (schemes/compSPH.py:170), pairwise
 * pressure / viscous accelerations ap_ij, av_ij [nnz*dim] by Verlet entry; any may be null.
 * verlet_cnt as for sph_crk_accel_dudt (zeros for the rest of each walked row). */
int sph_compsph_accel_dudt(const SphParams* p, int64_t n, const float* x, const float* H,
                           const float* m, const float* rho, const float* v, const float* c,
                           const float* alpha, const float* P, const float* omega,
                           const int32_t* offs, const int32_t* cnt, const int32_t* list,
                           const int32_t* verlet_cnt, float* dvdt_out, float* dudt_out,
                           float* dEdt_out, float* ap_ij, float* av_ij, void* stream);
/* The same pass over packed particle records: a first launch copies the fields the pass
 * reads into records [n, R] (R = sph_compsph_record_floats(dim) floats per particle: 12, 12
 * and 16 in 1D, 2D and 3D; 16-byte aligned, caller-owned scratch; null c, alpha, omega take
 * their defaults there), and the pair launch gathers each neighbour from that one record.
 * Outputs and arguments otherwise as sph_compsph_accel_dudt. */
int sph_compsph_record_floats(int32_t dim);
int sph_compsph_accel_dudt_packed(const SphParams* p, int64_t n, const float* x, const float* H,
                                  const float* m, const float* rho, const float* v, const float* c,
                                  const float* alpha, const float* P, const float* omega,
                                  const int32_t* offs, const int32_t* cnt, const int32_t* list,
                                  const int32_t* verlet_cnt, float* dvdt_out, float* dudt_out,
                                  float* dEdt_out, float* ap_ij, float* av_ij, float* records, void* stream);
/* The same pass under the reference's two wrapper names. */
int sph_compsph_accel(const SphParams* p, int64_t n, const float* x, const float* H,
                      const float* m, const float* rho, const float* v, const float* c,
                      const float* alpha, const float* P, const float* omega,
                      const int32_t* offs, const int32_t* cnt, const int32_t* list,
                      const int32_t* verlet_cnt, float* dvdt_out, float* ap_ij, float* av_ij,
                      void* stream);
int sph_compsph_dudt(const SphParams* p, int64_t n, const float* x, const float* H,
                     const float* m, const float* rho, const float* v, const float* c,
                     const float* alpha, const float* P, const float* omega,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list,
                     float* dudt_out, void* stream);

/* Monaghan-scheme right-hand side (schemes/monaghan.py:77-143) in one pass with the
 * kernel-mean support: symmetric grad-h pressure force (computePressureForceSymmetric,
 * modules/pressure/symmetricForce.py:7), PdV work (computeDudtMonaghan,
 * modules/internalEnergy/dudt.py:7), artificial viscosity (computeViscosityWarp,
 * modules/dissipation/wp_diffusion.py:246), conductivity with p->conductivity_term and
 * Cu_l / Cu_q (computeConductivityWarp, wp_conductivity.py:246) and viscous heating
 * (computeThermalDissipationWarp, wp_dissipation.py:249).  Outputs (any may be null):
 * dvdt = pressure + viscosity, dudt = PdV + conductivity + heating, dEdt = m v.dvdt +
 * m (PdV + conductivity) (monaghan.py:143), and each term on its own. */
int sph_monaghan_rhs(const SphParams* p, int64_t n, const float* x, const float* H,
                     const float* m, const float* rho, const float* v, const float* u,
                     const float* c, const float* alpha, const float* P, const float* omega,
                     const int32_t* offs, const int32_t* cnt, const int32_t* list,
                     float* dvdt_out, float* dudt_out, float* dEdt_out,
                     float* dvdt_pressure, float* dvdt_viscosity, float* dudt_pdv,
                     float* dudt_conductivity, float* dudt_heating, void* stream);

/* Pairwise energy-partition fraction f_ij (modules/compSPH/balance.py:17-154) for
 * the six energy schemes, evaluated at v_half = v + dt/2 dvdt (schemes/crkSPH.py:341-363).
 * scratch: device memory of n*(dim+1) floats (half-step velocities and P/rho^gamma).
 * f_ij is written for every entry of `list` (pass the Verlet list to fill all of it).
 * inter_counts (may be null): per row, the length of the interacting prefix of a list
 * whose rows hold their interacting entries first (sph_neighbors_build / refresh); the
 * entries after it have ap_ij = av_ij = 0, and their pair arrays are not read. */
int sph_compsph_balance(const SphParams* p, int64_t n, const float* m, const float* rho,
                        const float* P, const float* u, const float* v, const float* dvdt,
                        const float* dt, const int32_t* offs, const int32_t* cnt,
                        const int32_t* list, const int32_t* inter_counts,
                        const float* ap_ij, const float* av_ij,
                        float* scratch, float* f_ij_out, void* stream);

/* sph_compsph_balance without a scratch argument: no counterpart in the reference,
 * which allocates its temporaries through torch.  For callers that cannot allocate
 * device memory on the step path (an FFI host with no caching allocator, or a timed
 * loop where cudaMalloc/cudaFree would synchronise the device).  The scratch is a
 * fixed per-device array of SPH_BALANCE_NOALLOC_MAX_FLOATS floats, so n*(dim+1) must
 * not exceed it (SPH_ERR_BAD_ARG otherwise).  The array (16 MiB) is held on every
 * device that loads the library until the process exits.  The first call on a device,
 * and the first after its context was replaced (cudaDeviceReset), resolves the array's
 * address; make it before any stream capture.  Calls in flight at the same time on one
 * device share the array and race: serialise them on one stream. */
#define SPH_BALANCE_NOALLOC_MAX_FLOATS (1 << 22)
int sph_compsph_balance_noalloc(const SphParams* p, int64_t n, const float* m, const float* rho,
                                const float* P, const float* u, const float* v, const float* dvdt,
                                const float* dt, const int32_t* offs, const int32_t* cnt,
                                const int32_t* list, const float* ap_ij, const float* av_ij,
                                float* f_ij_out, void* stream);

/* ---------------------------------------------------------------- mDBC wall particles */
/* Particle kinds: 0 fluid, 1 wall (boundary), 2 ghost point of a wall particle (the
 * reference's kinds, initializers/weaklyCompressible.py:145 and
 * rigidBody/ghostParticles.py:71).  ghost_indices: a wall particle's ghost and a ghost's
 * wall particle (-1 for fluid); ghost_offsets [n, dim]: x_wall - x_ghost for a wall
 * particle, its negative for the ghost. */

/* computeMdbcDensity (modules/mdbc/density2025.py:20-85) with interpolateLiuLiu
 * (modules/liu/interp.py:9-37) and the moment sums of computeLiuMatrices_Func_i
 * (modules/liu/wp_mat.py:9-135): rho_out = rho, except for each wall particle, whose
 * density comes from the Liu-Liu interpolation of the fluid densities at its ghost point
 * (scatter support H_j; the FP64 pseudo-inverse of the (dim+1)^2 moment matrix when more
 * than 4 fluid neighbours lie inside their supports), projected back to the wall by the
 * first-order term (more than 9 neighbours) or else the hydrostatic Shepard estimate
 * max(rho0, rho0 + (c_s^2 (rho_sh - rho0) + rho0 (n.g)(r.n)) / c_s^2).  The rows are Verlet
 * rows of a list built over every particle, ghosts included.  gravity [3] (nullable = none)
 * is the acceleration vector.  ghost_neighbors_out [n] (nullable) gets the ghosts'
 * neighbour counts.  rho_out may alias rho. */
int sph_mdbc_density(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                     const float* rho, const int32_t* kinds, const int32_t* ghost_indices,
                     const float* ghost_offsets, const int32_t* offs, const int32_t* cnt,
                     const int32_t* list, double rest_density, double sound_speed,
                     const double* gravity, float* rho_out, int32_t* ghost_neighbors_out,
                     void* stream);

/* computeMdbcNoPenShift (modules/mdbc/wp_nopenshift.py:187-307, :400-420, :493-511): for
 * each fluid particle the wall neighbours under the gather support, the wall normal from
 * the wall particle's ghost offset, and per axis the no-penetration terms of the pairs
 * that qualify, averaged over their count; shift_out [n, dim] (zero for non-fluid). */
int sph_mdbc_nopen_shift(const SphParams* p, int64_t n, const float* x, const float* H,
                         const float* m, const float* v, const int32_t* kinds,
                         const float* ghost_offsets, const int32_t* offs, const int32_t* cnt,
                         const int32_t* list, float* shift_out, void* stream);

/* ---------------------------------------------------------------- (c) incompressible (DFSPH) */
/* Relaxed Jacobi solver settings (configurations/moduleConfigurations/solver.py:8-28
 * RelaxedJacobiSolverConfig) plus the rest density (fluidProperties.restDensity). */
typedef struct SphJacobiConfig {
    double rest_density;              /* rho0 */
    double tolerance;                 /* divergence-free default 2.5e-3, density 5e-4 */
    double relaxation;                /* omega: 0.3 for both default solvers */
    int32_t min_iterations;           /* 2 */
    int32_t max_iterations;           /* divergence-free 32, density 64 */
    /* 0: the reference's initial pressure (divergence-free: 0.75 * p_init,
     *    divergenceFree.py:72; density: 0, incompressible.py:79);
     * 1: p_init is used as given (a learned warm start). */
    int32_t init_mode;
    /* wait limit of each grid barrier in microseconds (0: 2 s).  A barrier that runs out
     * sets SPH_STATUS_TIMEOUT and every block of the solve returns; the outputs then hold
     * the last completed iteration's values. */
    int32_t barrier_timeout_us;
    int32_t reserved_i[2];
} SphJacobiConfig;

/* DFSPH diagonal, the value computeAlpha returns (modules/incompressible/wp_alpha.py:35-118,
 * :294-313): alpha_out_i = -( (V_i/m_i) |sum_j V_j gradW_ij|^2 + V_i sum_j V_j^2/m_j |gradW_ij|^2 )
 * with V = m/rho and the gather kernel gradient gradW(x_i - x_j, H_i). */
int sph_dfsph_alpha(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                    const float* rho, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                    float* alpha_out, void* stream);

/* computeMomentumIncompressible (modules/momentum/incompressible.py:9-34) of the
 * predicted velocity v* = v + dt*dvdt (dvdt may be null: v* = v):
 * div_out_i = -rho0 * sum_j V_j (v*_j - v*_i) . gradW(x_ij, H_j). */
int sph_incompressible_divergence(const SphParams* p, int64_t n, double rest_density,
                                  const float* x, const float* H, const float* m, const float* rho,
                                  const float* v, const float* dvdt, const float* dt,
                                  const int32_t* offs, const int32_t* cnt, const int32_t* list,
                                  float* div_out, void* stream);

/* computePressureAccelIISPH (modules/pressure/iisph.py:7-24), scatter support:
 * a_i = -(rho_i sum_j m_j (p_i/rho_i^2 + p_j/rho_j^2) gradW(x_ij, H_j)) / rho_i. */
int sph_pressure_accel_iisph(const SphParams* p, int64_t n, const float* x, const float* H,
                             const float* m, const float* rho, const float* pressure,
                             const int32_t* offs, const int32_t* cnt, const int32_t* list,
                             float* accel_out, void* stream);

/* computePressureShiftIISPH (modules/incompressible/drift.py:38-57):
 * s_i = -sum_j V_j (a_j - a_i) . gradW(x_ij, H_j). */
int sph_pressure_shift_iisph(const SphParams* p, int64_t n, const float* x, const float* H,
                             const float* m, const float* rho, const float* accel,
                             const int32_t* offs, const int32_t* cnt, const int32_t* list,
                             float* shift_out, void* stream);

/* Workspace bytes of sph_dfsph_div_solve / sph_dfsph_density_solve. */
int64_t sph_dfsph_workspace_size(int64_t n, int32_t dim);

/* solveDivergenceFree (modules/incompressible/divergenceFree.py:23-139) as ONE
 * persistent cooperative kernel: source = -div(v + dt dvdt) (above, times -1),
 * diag = dt*alpha, p0 from p_init (init_mode), then per iteration
 * a = pressure_accel(p), r = source - dt*pressure_shift(a), p += omega r/diag,
 * p -= mean(p), error = mean|r|, stop when it >= min_iterations and error < tolerance.
 * The final pressure acceleration is computed from the last pressure.
 * Outputs: p_out [n], accel_out [n*dim], history [max_iterations*4] floats
 * (per iteration: error, min p, max p, mean p after the gauge, as the reference's
 * `errors` and `pressures` lists), *iterations (device int32) and *status (device
 * int32; SPH_STATUS_NOT_CONVERGED when the cap was hit, SPH_STATUS_NONFINITE,
 * SPH_STATUS_TIMEOUT if a grid barrier gave up).  No host synchronisation inside. */
int sph_dfsph_div_solve(const SphParams* p, const SphJacobiConfig* cfg, int64_t n,
                        const float* x, const float* H, const float* m, const float* rho,
                        const float* v, const float* dvdt, const float* p_init, const float* dt,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list,
                        void* workspace, int64_t workspace_bytes,
                        float* p_out, float* accel_out, float* history, int32_t* iterations,
                        int32_t* status, void* stream);

/* solveIncompressible (modules/incompressible/incompressible.py:21-143), same
 * structure: rho* = max(rho + dt*div, 0.9), source = rho0 - rho*,
 * diag = min(dt^2 alpha, -1e-6), p0 = 0 (init_mode 0), per iteration
 * r = source - dt^2*pressure_shift(a), p = max(p + omega r/diag, 0),
 * error = mean(max(-r, -tolerance)). */
int sph_dfsph_density_solve(const SphParams* p, const SphJacobiConfig* cfg, int64_t n,
                            const float* x, const float* H, const float* m, const float* rho,
                            const float* v, const float* dvdt, const float* p_init, const float* dt,
                            const int32_t* offs, const int32_t* cnt, const int32_t* list,
                            void* workspace, int64_t workspace_bytes,
                            float* p_out, float* accel_out, float* history, int32_t* iterations,
                            int32_t* status, void* stream);

/* ---------------------------------------------------------------- weakly compressible (delta-SPH) */
/* EOS (modules/eos/weaklyCompressible.py:4-44), density diffusion terms
 * (enumTypes.py:53-58, DensityDiffusionScheme) and pressure terms (enumTypes.py:60-66). */
#define SPH_EOS_STIFF_TAIT   0
#define SPH_EOS_TAIT         1
#define SPH_EOS_ISOTHERMAL   2
#define SPH_EOS_POLYTROPIC   3
#define SPH_EOS_MURNAGHAN    4
#define SPH_DENSITY_DIFFUSION_DELTA         0
#define SPH_DENSITY_DIFFUSION_DENSITY_ONLY  2
#define SPH_DENSITY_DIFFUSION_DELTA_ONLY    3
#define SPH_PRESSURE_CONSERVATIVE     0
#define SPH_PRESSURE_NONCONSERVATIVE  1
#define SPH_PRESSURE_ANTUONO          2
#define SPH_PRESSURE_I                3
#define SPH_PRESSURE_J                4
#define SPH_PRESSURE_SYMMETRIC        5

/* fluidProperties (configurations/moduleConfigurations/fluidProperties.py:9-19) and
 * WeaklyCompressibleDiffusionParams (weaklyCompressibleDiffusionParams.py:10-17). */
typedef struct SphWcParams {
    double rest_density;          /* rho0 */
    double sound_speed;           /* fixedSoundSpeed c0 */
    double polytropic_exponent;   /* 7 */
    double kappa;
    double density_delta;         /* delta, 0.1 */
    double viscosity_nu;          /* viscidNu, 1e-3 */
    double inviscid_alpha;        /* 0.01 */
    int32_t inviscid;             /* 1: alpha c0 H / xi; 0: 2 (d + 2) nu */
    int32_t density_scheme;       /* SPH_DENSITY_DIFFUSION_* */
    int32_t pressure_term;        /* SPH_PRESSURE_* (the reference default is Antuono) */
    int32_t eos;                  /* SPH_EOS_* */
    int32_t reserved_i[4];
} SphWcParams;

/* One delta-SPH right-hand side (schemes/deltaSPH.py:97-171 for a fluid with no
 * boundaries or forcing): pass A computes the renormalised density gradient
 * (modules/density/gradRhoL.py) and the EOS pressure into scratch [n*(dim+1)] floats;
 * pass B writes dvdt [n, dim] = pressure force -sum_j V_j p_ij gradW_ij / rho_i
 * (modules/pressure/wp_surfaceAware.py:207-218) + velocity diffusion (wp_viscosityDelta.py)
 * and drhodt [n] = continuity (modules/momentum/inconsistent.py) + density diffusion
 * (modules/deltaSPH/densityDiffusion.py).  Kernel support max(H_i, H_j).
 * surface_mask [n] int32 (nullable = no free surface): the state's surfaceIndicators;
 * the Antuono term takes P_j + P_i for a particle whose indicator is 1
 * (wp_surfaceAware.py:89-92). */
int sph_deltasph_rhs(const SphParams* p, const SphWcParams* wc, int64_t n, const float* x,
                     const float* H, const float* m, const float* rho, const float* v,
                     const int32_t* surface_mask, const int32_t* offs, const int32_t* cnt,
                     const int32_t* list, float* scratch, float* dvdt_out, float* drhodt_out,
                     void* stream);

/* Batched ensemble of independent periodic boxes (no counterpart in the reference, which
 * runs one simulation per process).  Particles of every box share one set of arrays;
 * box_of[n] gives each particle's box.  Box b has a grid of box_grid[b]^dim cells over
 * the periodic domain of `p` (cell size L / box_grid[b] >= verlet_scale * max H of the
 * box, box_grid[b] >= 3), whose keys start at box_cell_base[b]; total_cells is the sum
 * of box_grid[b]^dim.  The Verlet rows (same row rule and order conventions as
 * sph_neighbors_build, per box) never pair particles of different boxes. */
int64_t sph_ensemble_neighbors_workspace_size(int64_t n, int64_t total_cells);
int sph_ensemble_neighbors_build(const SphParams* p, int64_t n, int32_t nbox, const int32_t* box_of,
                                 const int32_t* box_grid, const int32_t* box_cell_base,
                                 int64_t total_cells, const float* x, const float* H,
                                 void* workspace, int64_t workspace_bytes,
                                 int32_t* offs, int32_t* cnt, int32_t* list, int64_t list_capacity,
                                 int64_t* nnz_out, int32_t* status, void* stream);

/* One Heun RK2 step of every box in ONE cooperative persistent launch: delta-SPH
 * right-hand side (sph_deltasph_rhs) at y0 and y1 = y0 + dt k1, then
 * y = y0 + dt/2 (k1 + k2) for x (wrapped into the periodic domain), v and rho; dt is
 * box_dt[box_of[i]].  x, v, rho are updated in place.  *disp_max receives the largest
 * |x - x_build| / H since x_build (ordered-float encoding, atomicMax: zero it after a
 * rebuild); the rows stay valid while 2 disp_max < verlet_scale - 1.  lanes (4, 8, 16)
 * and block (128, 256) select the tile shape (the autotuner's choice).  workspace:
 * sph_ensemble_step_workspace_size(n, dim) bytes, 256-byte aligned. */
int64_t sph_ensemble_step_workspace_size(int64_t n, int32_t dim);
int sph_ensemble_step(const SphParams* p, const SphWcParams* wc, int64_t n, const int32_t* box_of,
                      const float* box_dt, const float* H, const float* m, float* x, float* v,
                      float* rho, const float* x_build, const int32_t* offs, const int32_t* cnt,
                      const int32_t* list, void* workspace, int64_t workspace_bytes,
                      int32_t lanes, int32_t block, uint32_t* disp_max, int32_t* status, void* stream);

/* weaklyCompressibleEOS (modules/eos/weaklyCompressible.py:21-44). */
int sph_wc_eos(const SphWcParams* wc, int64_t n, const float* rho, float* P_out, void* stream);

/* Velocity diffusion and continuity of the DFSPH step (schemes/dfsph.py:100-109:
 * computeVelocityDiffusion, modules/deltaSPH/velocityDissipation.py:18-36 with
 * wp_viscosityDelta.py:14-108, and computeMomentum, modules/momentum/inconsistent.py:16-31),
 * one pass, super-symmetric support max(H_i, H_j): dvdt_out [n, dim] = the delta-SPH
 * velocity diffusion, drhodt_out [n] = -rho_i sum_j V_j (v_j - v_i).gradW_ij.  Bit for
 * bit the dvdt / drhodt of sph_deltasph_rhs with zero pressure and density_delta = 0. */
int sph_wc_visc_continuity(const SphParams* p, const SphWcParams* wc, int64_t n, const float* x,
                           const float* H, const float* m, const float* rho, const float* v,
                           const int32_t* offs, const int32_t* cnt, const int32_t* list,
                           float* dvdt_out, float* drhodt_out, void* stream);

/* One delta-plus shift (modules/shifting/delta.py:6-47 with sample/wp_deltaShift.py:57-126,
 * gather support H_i): shift_out [n, dim] = -cfl Ma 2 (H_i / xi)^2 sum_j
 * (1 + R (W_ij / W0_j)^nexp) m_j / (2 (rho_i + rho_j)) gradW_ij, with W0_j the kernel at
 * (m_j / rho0)^(1/dim) / xi, Ma = max_i |v_i| / c0 over the finite magnitudes (0.1 when
 * below 1e-6) and zero shift for kinds[i] != 0 (kinds may be null: all fluid).
 * scratch: 2 device words (the max reduction).  The reference passes R = 0.25,
 * nexp = 4 and rho0 = 1. */
int sph_delta_shift(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                    const float* rho, const float* v, const int32_t* kinds,
                    const int32_t* offs, const int32_t* cnt, const int32_t* list,
                    float cfl, float c0, float R, int32_t nexp, float rho0,
                    uint32_t* scratch, float* shift_out, void* stream);

/* ---------------------------------------------------------------- free-surface detection
 * detectFreeSurface with the colour-field scheme (modules/surfaceDetection/wrapper.py:84-149).
 * Rows are the interacting prefixes (every pair with r < max(H_i, H_j)).
 *
 * Colour field (colorFieldCompute.py:11-45, first half): color_out[i] =
 * sum_j m_j/rho_j W(r_ij, H_i). */
int sph_surface_color_field(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                            const float* rho, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                            float* color_out, void* stream);

/* detectFreeSurfaceColorField (colorFieldDetection.py:16-73) in one pass, with the gradient
 * of colorFieldCompute.py:33-44 and the counts and sums of util/wp_numNeighbors.py and
 * util/wp_sum.py (pairs with W(r_ij, max(H_i, H_j)) > 0, self included):
 *   fs_out[i] = 1 if color[i] < S_i / N_i and N_i < neighbor_limit, else 0
 *     (neighbor_limit = targetNeighbors * colorFieldThreshold);
 *   normals_out [n, dim] (may be null) = normal_sign * grad c_i / max(|grad c_i|, 1e-12),
 *     with grad c_i = sum_j m_j/rho_j (c_j - c_i) grad W(r_ij, H_i).  normal_sign is -1 for
 *     NormalSource.ColorFieldGrad (wrapper.py:54-61) and +1 for the scheme's own normals;
 *   num_neighbors_out (may be null) = N_i. */
int sph_surface_detect_color_field(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                                   const float* rho, const float* color, const int32_t* offs, const int32_t* cnt,
                                   const int32_t* list, float neighbor_limit, float normal_sign, float* fs_out,
                                   float* normals_out, float* num_neighbors_out, void* stream);

/* One dilation iteration (wp_dilate.py:14-89): fs_out[i] = sum_j fs_in[j] over the pairs
 * with W(r_ij, max(H_i, H_j)) > 0.  The reference keeps the sum (a count, not a 0/1 mask);
 * so does this.  fs_in and fs_out must not alias. */
int sph_surface_dilate(const SphParams* p, int64_t n, const float* x, const float* H, const float* fs_in,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list, float* fs_out, void* stream);
/* Barecasco detection (wp_barecasco.py:36-453, barecascoDetection.py:22-43): the cover
 * vector c_i = sum_j x_ij / (r_ij + 1e-14 H_i) over the pairs with W(r, max(H_i, H_j)) > 0,
 * normals_out = c_i / |c_i| (0 for c_i = 0), count_out = the pairs with W > 0 whose
 * acos(-n_ij . c^_i) <= threshold / 2 (j != i), or every pair when |c^_i| <= 0.5; fs_out =
 * 1 where the count is below 0.5.  normals_out and count_out may be null. */
int sph_surface_barecasco(const SphParams* p, int64_t n, const float* x, const float* H,
                          const int32_t* offs, const int32_t* cnt, const int32_t* list, float threshold,
                          float* fs_out, float* normals_out, float* count_out, void* stream);
/* Maronne detection (wp_maronne.py:57-332, maronneDetection.py:20-80) with the given
 * normals [n, dim]: fs_out = 1 where no neighbour j != i with r_ij < H_j lies in the
 * circle of radius H_j / xi around T_i = x_i + n_i H_i / xi (r_ij >= sqrt(2) H_j / xi) or in
 * the square |n_i.(x_j - T_i)| + |tau_i.(x_j - T_i)| < H_j / xi (r_ij < sqrt(2) H_j / xi),
 * for |n_i| > 0.5; xi = p's kernel xi.  count_out (may be null) gets the count. */
int sph_surface_maronne(const SphParams* p, int64_t n, const float* x, const float* H, const float* normals,
                        const int32_t* offs, const int32_t* cnt, const int32_t* list, float* fs_out,
                        float* count_out, void* stream);
/* Colour-field-gradient detection (colorFieldGradientDetection.py:18-56): the gather
 * difference gradient g_i of the colour field, fs_out = [|g_i| > threshold H_i / xi] and
 * normals_out = -g_i / max(|g_i|, 1e-12) (may be null). */
int sph_surface_detect_color_gradient(const SphParams* p, int64_t n, const float* x, const float* H,
                                      const float* m, const float* rho, const float* color,
                                      const int32_t* offs, const int32_t* cnt, const int32_t* list,
                                      float threshold, float* fs_out, float* normals_out, void* stream);
/* Renormalisation matrices, standing in for warpSPHCore's computeRenormalizationMatrices
 * (called at surfaceDetection/wrapper.py:21-33): M_i = sum_j V_j (x_j - x_i) (x)
 * grad_i W(r_ij, max(H_i, H_j)), V_j = m_j / rho_j; L_out [n, dim, dim] = pinv(M_i) (FP64,
 * cutoff dim * FLT_EPSILON * sigma_max), lambda_out [n] = the smallest |eigenvalue| of M_i.
 * Either output may be null, not both. */
int sph_surface_renormalization(const SphParams* p, int64_t n, const float* x, const float* H,
                                const float* m, const float* rho, const int32_t* offs, const int32_t* cnt,
                                const int32_t* list, float* L_out, float* lambda_out, void* stream);
/* Normals from the renormalised gradients, normals_out = -g_i / max(|g_i|, 1e-12) with
 * g_i = L_i sum_j V_j q_ij grad W(r_ij, H_j) (scatter support): mode 0, the lambda gradient
 * of lambdaGrad.py:46-83 (q_ij = lambda_j - lambda_i); mode 1, Maronne's normals of
 * maronneNormals.py:16-62 (q_ij = 1; lambdas may be null).  grad_out (may be null) gets g. */
int sph_surface_renormalized_normals(const SphParams* p, int64_t n, int32_t mode, const float* x,
                                     const float* H, const float* m, const float* rho, const float* L,
                                     const float* lambdas, const int32_t* offs, const int32_t* cnt,
                                     const int32_t* list, float* normals_out, float* grad_out, void* stream);

/* ---------------------------------------------------------------- learned warm start
 * No counterpart in the reference: a per-particle MLP predicts the initial pressure of
 * the Jacobi solves (replacing 0.75 p_prev at divergenceFree.py:72 and 0 at
 * incompressible.py:79); the solve then iterates to the same tolerance (init_mode 1).
 * Network: 8 -> 64 -> 64 -> 64 -> 1, ReLU; FP32 master parameters
 *   W1[64][8] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4[1]
 * BF16 weights and activations into the tensor cores, FP32 accumulation. */
#define SPH_MLP_PARAM_COUNT 8961
int64_t sph_mlp_param_count(void);

/* Input features of the solve `mode` (0 divergence-free, 1 density) for the state:
 * feats_out [n][8] (16-byte aligned): p_jac/P, smoothed p_jac/P, p_prev/P, smoothed
 * p_prev/P, 100 (rho/rho0 - 1), Shepard deficit, relative neighbour count, relative
 * diagonal, with p_jac = source/diagonal of that solve and P = mean |p_jac|
 * (scale_out[0]).  workspace: sph_dfsph_workspace_size(n) bytes, 256-byte aligned. */
int sph_dfsph_features(const SphParams* p, const SphJacobiConfig* cfg, int32_t mode, int64_t n,
                       const float* x, const float* H, const float* m, const float* rho,
                       const float* v, const float* dvdt, const float* p_prev, const float* dt,
                       const int32_t* offs, const int32_t* cnt, const int32_t* list,
                       void* workspace, int64_t workspace_bytes,
                       float* feats_out, float* scale_out, void* stream);

/* out[i] = MLP(feats[i]) * (*scale) (scale may be null: 1). */
int sph_mlp_forward(const float* params, int64_t n, const float* feats, const float* scale,
                    float* out, void* stream);

/* The same network on the Blackwell tensor cores (tcgen05.mma kind::f16, accumulators in
 * TMEM): 128 samples per CTA tile, the same BF16 rounding points as sph_mlp_forward.
 * feats must be 16-byte aligned.  If a tensor-core chain does not complete within about
 * a second the kernel gives up: the samples it had not finished get NaN and
 * SPH_STATUS_TIMEOUT is or-ed into *status (device int32; may be null). */
int sph_mlp_forward_tc(const float* params, int64_t n, const float* feats, const float* scale,
                       float* out, int32_t* status, void* stream);

/* Gradient of the mean squared error (1/n) sum_i (MLP(feats_i) - target_i)^2 with
 * respect to the parameters: grad [SPH_MLP_PARAM_COUNT] is overwritten, *loss receives
 * sum_i (MLP(feats_i) - target_i)^2 (device double). */
int sph_mlp_grad(const float* params, int64_t n, const float* feats, const float* target,
                 float* grad, double* loss, void* stream);
/* The same gradient with every GEMM on tcgen05 (one CTA per SM, the weight gradients
 * accumulated in tensor memory; feats 16-byte aligned).  Rounding points as sph_mlp_grad,
 * except that the bias gradients are summed from the BF16 dZ.  A tensor-core wait that
 * runs out ors SPH_STATUS_TIMEOUT into *status (may be null) and leaves grad incomplete. */
int sph_mlp_grad_tc(const float* params, int64_t n, const float* feats, const float* target,
                    float* grad, double* loss, int32_t* status, void* stream);

/* One Adam step (Kingma & Ba 2015, bias-corrected; step counts from 1). */
int sph_mlp_adam(float* params, const float* grad, float* m1, float* m2, int64_t count,
                 float lr, float beta1, float beta2, float eps, int64_t step, void* stream);

/* ---------------------------------------------------------------- (d) integrator and dt */
/* CFL time step (modules/timestep/compressible.py:12-61): dt = min_i cfl*min(H)/(c_i xi),
 * clamped to [min_dt, max_dt] and, when dt_prev != null, to <= dt_growth*dt_prev.
 * c is computed from u by the ideal-gas EOS.  dt_out is device memory of at least
 * 4 floats: dt_out[0] receives dt, dt_out[1..2] are reduction scratch. */
int sph_cfl_dt(const SphParams* p, int64_t n, const float* H, const float* u, const float* rho,
               const float* dt_prev, float* dt_out, void* stream);

/* Runge-Kutta stage combination y = y0 + dt * sum_k w_k K_k for `nk` derivative
 * arrays (each [count] floats), optional periodic wrap of positions into the domain
 * when wrap_dim > 0 (count = n*wrap_dim).  Weights are host doubles, dt is device. */
int sph_rk_combine(const SphParams* p, int64_t count, const float* y0, int32_t nk,
                   const float* const* k_ptrs, const double* weights, const float* dt,
                   int32_t wrap_dim, float* y_out, void* stream);

/* sph_rk_combine over up to 4 fields in one launch (the stage update of positions,
 * velocities and energies together): field f has counts[f] floats y0s[f] -> y_outs[f],
 * wrap_dims[f] as wrap_dim above, and derivatives k_ptrs[f * nk + q]; the weights are
 * shared.  Each element is computed as sph_rk_combine computes it. */
int sph_rk_combine_fields(const SphParams* p, int32_t nfields, const int64_t* counts,
                          const float* const* y0s, float* const* y_outs, const int32_t* wrap_dims,
                          int32_t nk, const float* const* k_ptrs, const double* weights,
                          const float* dt, void* stream);

/* Compatible-energy finalize (systems/compSPH.py:100-111 and
 * modules/compSPH/multistep.py:52-94): v_half = v0 + dt/2 sum_s b_s dvdt_s,
 * du_i = sum_s b_s sum_j f_ij^s (v_half_j - v_half_i).(ap_ij^s + av_ij^s)
 * (PdV: f_ij ap + 1/2 av), u = u0 + du*dt.  Per-stage arrays are passed as arrays
 * of device pointers (host arrays of length nstages).  du_out must hold
 * n*(1+dim) floats: du in the first n, the half-step velocity as scratch after it. */
int sph_finalize_compatible_energy(const SphParams* p, int64_t n, int32_t nstages,
                                   const double* weights, const float* dt,
                                   const float* v0, const float* u0,
                                   const float* const* dvdt_s,
                                   const int32_t* const* offs_s, const int32_t* const* cnt_s,
                                   const int32_t* const* list_s,
                                   const float* const* f_ij_s, const float* const* ap_ij_s,
                                   const float* const* av_ij_s,
                                   float* u_out, float* du_out, void* stream);

/* Mass, momentum, kinetic, internal and total energy sums in FP64 (device double[6+dim]):
 * [M, KE, IE, E, px, py, pz]; used for conservation checks. */
int sph_conservation_sums(const SphParams* p, int64_t n, const float* m, const float* v,
                          const float* u, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WARPSPH_B200_H */
