// Moore-Penrose inverse of small dense matrices in FP64 (the Cullen-Hopkins velocity
// gradient correction and the Liu-Liu interpolation of the mDBC wall density).
#pragma once
#include <cuda_runtime.h>

namespace wsph {

// Moore-Penrose inverse of a D x D matrix in FP64 by one-sided (Hestenes) Jacobi: column
// rotations make A V = U orthogonal-columned, sigma_k = |U_k|, and
// pinv(A) = sum_k v_k U_k^T / sigma_k^2 over sigma_k > rtol * sigma_max.  With
// rtol = D * FLT_EPSILON this is torch.linalg.pinv's default cutoff for a float32 input
// (CullenHopkins.py:27, liu/interp.py:31).  The sweep count is bounded; D <= 4 converges in a few
// sweeps.  With smin_out the smallest singular value is written there (for a symmetric A, its
// smallest |eigenvalue|).
template <int D>
__device__ __forceinline__ void pinv_jacobi(const double (&A)[D][D], double (&P)[D][D], double rtol, double* smin_out = nullptr) {
    double U[D][D], V[D][D];
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) { U[a][b] = A[a][b]; V[a][b] = a == b ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 16; ++sweep) {
        bool rotated = false;
        #pragma unroll
        for (int p = 0; p < D - 1; ++p)
            #pragma unroll
            for (int q = p + 1; q < D; ++q) {
                double al = 0.0, be = 0.0, ga = 0.0;
                #pragma unroll
                for (int r = 0; r < D; ++r) { al += U[r][p] * U[r][p]; be += U[r][q] * U[r][q]; ga += U[r][p] * U[r][q]; }
                if (!(fabs(ga) > 1e-15 * sqrt(al * be))) continue;
                rotated = true;
                const double zeta = (be - al) / (2.0 * ga);
                const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
                #pragma unroll
                for (int r = 0; r < D; ++r) {
                    const double up = U[r][p], uq = U[r][q];
                    U[r][p] = c * up - sn * uq; U[r][q] = sn * up + c * uq;
                    const double vp = V[r][p], vq = V[r][q];
                    V[r][p] = c * vp - sn * vq; V[r][q] = sn * vp + c * vq;
                }
            }
        if (!rotated) break;
    }
    double s2[D], smax = 0.0;
    #pragma unroll
    for (int k = 0; k < D; ++k) {
        s2[k] = 0.0;
        #pragma unroll
        for (int r = 0; r < D; ++r) s2[k] += U[r][k] * U[r][k];
        smax = fmax(smax, sqrt(s2[k]));
    }
    if (smin_out) {
        double smin = sqrt(s2[0]);
        #pragma unroll
        for (int k = 1; k < D; ++k) smin = fmin(smin, sqrt(s2[k]));
        *smin_out = smin;
    }
    const double cut = rtol * smax;
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) P[a][b] = 0.0;
    #pragma unroll
    for (int k = 0; k < D; ++k) {
        if (!(sqrt(s2[k]) > cut)) continue;
        const double inv = 1.0 / s2[k];
        #pragma unroll
        for (int a = 0; a < D; ++a)
            #pragma unroll
            for (int b = 0; b < D; ++b) P[a][b] += V[a][k] * U[b][k] * inv;
    }
}

}  // namespace wsph
