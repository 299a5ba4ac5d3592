// Modified dynamic boundary conditions (mDBC) of the DFSPH step with wall particles
// (kind 1) and their ghost points (kind 2):
//
//   sph_mdbc_density   modules/mdbc/density2025.py:20-85 with the Liu-Liu interpolation of
//                      modules/liu/interp.py:9-37 and the moment sums of
//                      modules/liu/wp_mat.py:9-135: for each ghost g the fluid neighbours j
//                      (kind 0) under the scatter support H_j give
//                        b = sum_j V_j rho_j [W, grad W],
//                        A = sum_j V_j [[W, -x_gj W], [grad W, -x_gj (x) grad W]]
//                      (V_j = m_j / rho_j, x_gj = x_g - x_j), res = pinv(A) b when more
//                      than 4 neighbours lie inside H_j (else 0), and the wall particle
//                      b(g) gets
//                        rho_b = max(rho0, rho0 + (c_s^2 (rho_sh - rho0) + rho0 (n.g)(r.n)) / c_s^2)
//                      with the Shepard value rho_sh = b0 / A00 (rho0 when A00 = 0 or at most
//                      one neighbour), r = x_b - x_g and n = r / |r|; with more than 9
//                      neighbours it gets the first-order projection res0 - r . res[1:]
//                      instead.  Every other density is copied.
//   sph_mdbc_nopen_shift  modules/mdbc/wp_nopenshift.py:187-307, :400-420: for each fluid
//                      particle the wall neighbours (kind 1) under the gather support, with
//                      the wall normal -o_j / (|o_j| + 1e-12) from the wall particle's ghost
//                      offset o_j; per axis the no-penetration terms of the qualifying pairs
//                      averaged over their count.
//
// The density pass walks the Verlet rows of a list built over every particle (ghosts
// included); the shift walks any list whose rows cover the fluid and wall particles.
#include <cuda_runtime.h>
#include <cfloat>
#include "sph_pair_common.cuh"
#include "sph_pinv.cuh"

namespace wsph {

struct MdbcArgs {
    float rho0, cs2;
    float g[3];
};

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_mdbc_density(int n, DevParams P, MdbcArgs M, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
               const float* __restrict__ rho, const int32_t* __restrict__ kinds, const int32_t* __restrict__ ghost_idx,
               const float* __restrict__ ghost_off, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
               const int32_t* __restrict__ list, float* __restrict__ rho_out, int32_t* __restrict__ nbr_out) {
    constexpr int E = D + 1;
    Grp<G> g(n);
    const bool ghost = g.valid && kinds[g.i] == 2;
    float b[E], A[E][E];
    #pragma unroll
    for (int a = 0; a < E; ++a) {
        b[a] = 0.f;
        #pragma unroll
        for (int c = 0; c < E; ++c) A[a][c] = 0.f;
    }
    float nb = 0.f;
    if (ghost) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const int be = offs[i], e = be + cnt[i];
        for (int q = be + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            if (__ldg(kinds + j) != 0) continue;                     // FluidToGhost: fluid neighbours only
            const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            const float hj = __ldg(H + j);
            float W; Vec<D> gW;
            kernelWG<KF, D>(xij, r, hj, W, gW);                        // scatter support H_j
            const float rj = __ldg(rho + j);
            const float Vj = __ldg(m + j) / rj;
            const float VQ = Vj * rj;
            b[0] += VQ * W;
            A[0][0] += Vj * W;
            #pragma unroll
            for (int d = 0; d < D; ++d) {
                b[d + 1] += VQ * gW.v[d];
                A[d + 1][0] += Vj * gW.v[d];
                A[0][d + 1] += -Vj * xij.v[d] * W;
                #pragma unroll
                for (int dd = 0; dd < D; ++dd) A[d + 1][dd + 1] += -Vj * xij.v[d] * gW.v[dd];
            }
            if (r < hj) nb += 1.f;
        }
    }
    #pragma unroll
    for (int a = 0; a < E; ++a) {
        b[a] = gsum<G>(b[a]);
        #pragma unroll
        for (int c = 0; c < E; ++c) A[a][c] = gsum<G>(A[a][c]);
    }
    nb = gsum<G>(nb);
    if (!ghost || g.lane != 0) return;
    const int i = g.i;
    const int nbrs = (int)nb;
    // res = pinv(A) b for more than 4 neighbours (interp.py:30-33)
    double res[E];
    #pragma unroll
    for (int a = 0; a < E; ++a) res[a] = 0.0;
    if (nbrs > 4) {
        double Ad[E][E], Pd[E][E];
        #pragma unroll
        for (int a = 0; a < E; ++a)
            #pragma unroll
            for (int c = 0; c < E; ++c) Ad[a][c] = (double)A[a][c];
        pinv_jacobi<E>(Ad, Pd, (double)E * (double)FLT_EPSILON);
        #pragma unroll
        for (int a = 0; a < E; ++a) {
            double s = 0.0;
            #pragma unroll
            for (int c = 0; c < E; ++c) s += Pd[a][c] * (double)b[c];
            res[a] = s;
        }
    }
    // density2025.py:39-83
    const float rho0 = M.rho0;
    const float shep = A[0][0] > 0.f ? b[0] / A[0][0] : rho0;
    const float rho_g = nbrs > 1 ? shep : rho0;
    const float P_g = M.cs2 * (rho_g - rho0);
    Vec<D> rel;
    float rn = 0.f;
    #pragma unroll
    for (int d = 0; d < D; ++d) { rel.v[d] = -ghost_off[(size_t)i * D + d]; rn += rel.v[d] * rel.v[d]; }
    const float inv = 1.f / fmaxf(sqrtf(rn), 1e-12f);                 // torch.nn.functional.normalize
    float dotg = 0.f, dot2 = 0.f, drho = 0.f;
    #pragma unroll
    for (int d = 0; d < D; ++d) {
        const float nd = rel.v[d] * inv;
        dotg += nd * M.g[d];
        dot2 += rel.v[d] * nd;
        drho += rel.v[d] * (float)res[d + 1];
    }
    const float P_b = P_g + rho0 * (dotg * dot2);
    float rho_b = rho0 + P_b / M.cs2;
    rho_b = fmaxf(rho_b, rho0);
    const float rho_proj = (float)res[0] + -drho;
    const int bidx = ghost_idx[i];
    if (bidx >= 0 && bidx < n) rho_out[bidx] = nbrs > 9 ? rho_proj : rho_b;
    if (nbr_out) nbr_out[i] = nbrs;
}

template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_mdbc_nopen(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
             const float* __restrict__ v, const int32_t* __restrict__ kinds, const float* __restrict__ ghost_off,
             const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
             float* __restrict__ shift_out) {
    Grp<G> g(n);
    const bool fluid = g.valid && kinds[g.i] == 0;
    Vec<D> acc = vzero<D>();
    float ctr[D];
    #pragma unroll
    for (int d = 0; d < D; ++d) ctr[d] = 0.f;
    if (fluid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i), vi = load_vec<D>(v, i);
        const float Hi = H[i];
        const float dp = powf(m[i], 1.f / (float)D);               // mi^(1/dim)
        const int be = offs[i], e = be + cnt[i];
        for (int q = be + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            if (__ldg(kinds + j) != 1) continue;                     // BoundaryToFluid: wall neighbours only
            const Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            const float w = kernelW<KF, D>(r, Hi);                   // gather support
            if (!(w > 0.f)) continue;
            Vec<D> o;
            float on = 0.f;
            #pragma unroll
            for (int d = 0; d < D; ++d) { o.v[d] = ghost_off[(size_t)j * D + d]; on += o.v[d] * o.v[d]; }
            const float norm_j = safe_sqrt(on) + 1e-12f;
            float normDist = 0.f;
            Vec<D> nj;
            #pragma unroll
            for (int d = 0; d < D; ++d) { nj.v[d] = -o.v[d] / norm_j; normDist += xij.v[d] * nj.v[d]; }
            const bool ca = r < 1.25f * dp;
            const bool cb = fabsf(normDist) < 0.75f * norm_j && norm_j < 1.75f * dp;
            const bool cab = ca && cb;
            const Vec<D> vj = load_vec<D>(v, j);
            #pragma unroll
            for (int d = 0; d < D; ++d) {
                const float dv = vi.v[d] - vj.v[d];
                const float nrm = nj.v[d];
                const float dr = xij.v[d];
                const bool mask = cab && (dr * nrm < 0.75f) && (fabsf(nrm) > 0.001f * dp);
                const float vfc = dv * nrm;
                const float ratio = fminf(fmaxf(fabsf(dr / nrm), 0.25f), 1.f);
                const float factor = -4.f * ratio + 3.f;
                const float term = -factor * dv * nrm * nrm;
                if (mask && vfc < 0.f) { acc.v[d] += term; ctr[d] += 1.f; }
            }
        }
    }
    #pragma unroll
    for (int d = 0; d < D; ++d) { acc.v[d] = gsum<G>(acc.v[d]); ctr[d] = gsum<G>(ctr[d]); }
    if (!g.valid || g.lane != 0) return;
    Vec<D> out;
    #pragma unroll
    for (int d = 0; d < D; ++d) out.v[d] = acc.v[d] / (ctr[d] + 1e-12f);
    store_vec<D>(shift_out, g.i, out);
}

}  // namespace wsph

using namespace wsph;

extern "C" {

int sph_mdbc_density(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                     const int32_t* kinds, const int32_t* ghost_indices, const float* ghost_offsets, const int32_t* offs,
                     const int32_t* cnt, const int32_t* list, double rest_density, double sound_speed, const double* gravity,
                     float* rho_out, int32_t* ghost_neighbors_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(kinds); WSPH_CHECK_PTR(ghost_indices);
    WSPH_CHECK_PTR(ghost_offsets); WSPH_CHECK_PTR(rho_out); CHECK_CSR();
    if (!(rest_density > 0.0) || !(sound_speed > 0.0)) return set_error(SPH_ERR_BAD_ARG, "sph_mdbc_density: rho0 and c_s must be > 0");
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, ghost_offsets, "ghost_offsets"))) return rc;
    MdbcArgs M;
    M.rho0 = (float)rest_density;
    M.cs2 = (float)(sound_speed * sound_speed);
    for (int d = 0; d < 3; ++d) M.g[d] = gravity ? (float)gravity[d] : 0.f;
    if (rho_out != rho) {
        cudaError_t e = cudaMemcpyAsync(rho_out, rho, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_mdbc_density: copy: %s", cudaGetErrorString(e));
    }
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_mdbc_density<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, M, x, H, m, rho, kinds, ghost_indices, ghost_offsets, offs, cnt, list, rho_out, ghost_neighbors_out)));
    return check_launch("sph_mdbc_density");
}

int sph_mdbc_nopen_shift(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* v,
                         const int32_t* kinds, const float* ghost_offsets, const int32_t* offs, const int32_t* cnt,
                         const int32_t* list, float* shift_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(v); WSPH_CHECK_PTR(kinds); WSPH_CHECK_PTR(ghost_offsets);
    WSPH_CHECK_PTR(shift_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, v, "v")) || (rc = check_align_vec(P, ghost_offsets, "ghost_offsets")) ||
        (rc = check_align_vec(P, shift_out, "shift_out")))
        return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_mdbc_nopen<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
        (int)n, P, x, H, m, v, kinds, ghost_offsets, offs, cnt, list, shift_out)));
    return check_launch("sph_mdbc_nopen_shift");
}

}  // extern "C"
