// Free-surface detection passes (modules/surfaceDetection): the colour field and its gather
// difference gradient (colorFieldCompute.py:11-45), the colour-field detection
// (colorFieldDetection.py:16-73) with the neighbour counts and sums of util/wp_numNeighbors.py
// and util/wp_sum.py under super-symmetric support, and the mask dilation (dilation.py,
// wp_dilate.py:14-89).  Each pass walks the interacting prefixes of the Verlet rows, which
// hold every pair with r < max(H_i, H_j).
//
// The Barecasco scheme (wp_barecasco.py:36-453), the Maronne scheme (wp_maronne.py:57-332,
// maronneDetection.py), the colour-field-gradient scheme (colorFieldGradientDetection.py)
// and the normal sources built on the renormalisation matrix (lambdaGrad.py,
// maronneNormals.py) are here too.  The renormalisation matrix and its eigenvalues come
// from warpSPHCore's computeRenormalizationMatrices, which the reference imports from its
// absent sibling package; they are restated as M_i = sum_j V_j (x_j - x_i) (x) grad_i W_ij
// under super-symmetric support (the moment matrix that is the identity for an interior
// particle), L_i = pinv(M_i) in FP64 and lambda_i = the smallest |eigenvalue| of the
// symmetric M_i (its smallest singular value).
#include <cuda_runtime.h>
#include "sph_pair_common.cuh"
#include "sph_pinv.cuh"

using namespace wsph;

namespace {

// c_i = sum_j m_j/rho_j W(r_ij, H_i): the gather interpolation of ones.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_color_field(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
              const float* __restrict__ rho, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
              const int32_t* __restrict__ list, float* __restrict__ c_out) {
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        const float invHi = 1.f / H[i];
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float W = kW_inv<KF, D>(safe_sqrt(dot<D>(xij, xij)), invHi);
            if (W == 0.f) continue;
            s += __ldg(m + j) / __ldg(rho + j) * W;
        }
    }
    s = gsum<G>(s);
    if (g.valid && g.lane == 0) c_out[g.i] = s;
}

// One pass over the rows: grad c_i = sum_j m_j/rho_j (c_j - c_i) grad W(r_ij, H_i) (gather),
// the count N_i and sum S_i of c_j over the pairs with W(r_ij, max(H_i, H_j)) > 0, the mask
// fs_i = [c_i < S_i / N_i and N_i < limit] and the normal sign * grad c_i / max(|grad c_i|, 1e-12).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_color_detect(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
               const float* __restrict__ rho, const float* __restrict__ c, const int32_t* __restrict__ offs,
               const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float limit, float normal_sign,
               float* __restrict__ fs_out, float* __restrict__ normals_out, float* __restrict__ nn_out) {
    Grp<G> g(n);
    Vec<D> gc = vzero<D>();
    float nn = 0.f, cs = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i], invHi = 1.f / Hi, ci = c[i];
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, r, invHi, W, gW);
            const float cj = __ldg(c + j);
            if (W != 0.f) {
                const float dq = __ldg(m + j) / __ldg(rho + j) * (cj - ci);
                #pragma unroll
                for (int a = 0; a < D; ++a) gc.v[a] += dq * gW.v[a];
            }
            if (kW_inv<KF, D>(r, 1.f / wmax(Hi, __ldg(H + j))) > 0.f) { nn += 1.f; cs += cj; }
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) gc.v[a] = gsum<G>(gc.v[a]);
    nn = gsum<G>(nn);
    cs = gsum<G>(cs);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    fs_out[i] = (c[i] < cs / nn && nn < limit) ? 1.f : 0.f;
    if (nn_out) nn_out[i] = nn;
    if (normals_out) {
        const float den = fmaxf(sqrtf(dot<D>(gc, gc)), 1e-12f);
        #pragma unroll
        for (int a = 0; a < D; ++a) normals_out[(size_t)i * D + a] = normal_sign * (gc.v[a] / den);
    }
}

// out_i = sum_j fs_j over the pairs with W(r_ij, max(H_i, H_j)) > 0 (the self pair included).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_dilate(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ fs,
         const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
         float* __restrict__ out) {
    Grp<G> g(n);
    float s = 0.f;
    if (g.valid) {
        const int i = g.i;
        Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i];
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            if (kW_inv<KF, D>(safe_sqrt(dot<D>(xij, xij)), 1.f / wmax(Hi, __ldg(H + j))) > 0.f) s += __ldg(fs + j);
        }
    }
    s = gsum<G>(s);
    if (g.valid && g.lane == 0) out[g.i] = s;
}


// Warp's normalize: v / |v|, or the zero vector when |v| = 0.
template <int D> __device__ __forceinline__ Vec<D> wnormalize(const Vec<D>& v) {
    const float l = sqrtf(dot<D>(v, v));
    Vec<D> r;
    #pragma unroll
    for (int a = 0; a < D; ++a) r.v[a] = l > 0.f ? v.v[a] / l : 0.f;
    return r;
}
// torch.nn.functional.normalize: v / max(|v|, 1e-12).
template <int D> __device__ __forceinline__ Vec<D> tnormalize(const Vec<D>& v) {
    const float l = fmaxf(sqrtf(dot<D>(v, v)), 1e-12f);
    Vec<D> r;
    #pragma unroll
    for (int a = 0; a < D; ++a) r.v[a] = v.v[a] / l;
    return r;
}

// Barecasco (wp_barecasco.py:36-113, 120-236, 338-355): the cover vector
// c_i = sum_j n_ij over the pairs with W(r_ij, max(H_i, H_j)) > 0, n_ij = x_ij / (r_ij +
// 1e-14 H_i); its normalisation c^_i; then the count of the pairs with W > 0 for which
// (acos(-n_ij . c^_i) <= theta / 2 and j != i) or |c^_i| <= 0.5.  The mask is count < 0.5
// (barecascoDetection.py:40).  Both walks run in the same group.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_barecasco(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const int32_t* __restrict__ offs,
            const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float theta, float* __restrict__ fs_out,
            float* __restrict__ normals_out, float* __restrict__ count_out) {
    Grp<G> g(n);
    Vec<D> cv = vzero<D>();
    Vec<D> xi = vzero<D>();
    float Hi = 1.f;
    int b = 0, e = 0;
    if (g.valid) {
        const int i = g.i;
        xi = load_vec<D>(x, i);
        Hi = H[i];
        b = offs[i]; e = b + cnt[i];
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            if (!(kW_inv<KF, D>(r, 1.f / wmax(Hi, __ldg(H + j))) > 0.f)) continue;
            const float den = r + 1.0e-14f * Hi;
            #pragma unroll
            for (int a = 0; a < D; ++a) cv.v[a] += xij.v[a] / den;
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) cv.v[a] = gsum<G>(cv.v[a]);
    const Vec<D> ch = wnormalize<D>(cv);
    const bool degenerate = sqrtf(dot<D>(ch, ch)) <= 0.5f;
    const float half = theta / 2.f;
    float count = 0.f;
    if (g.valid) {
        const int i = g.i;
        for (int q = b + g.lane; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            const float r = safe_sqrt(dot<D>(xij, xij));
            if (!(kW_inv<KF, D>(r, 1.f / wmax(Hi, __ldg(H + j))) > 0.f)) continue;
            const float den = r + 1.0e-14f * Hi;
            float d = 0.f;
            #pragma unroll
            for (int a = 0; a < D; ++a) d += -(xij.v[a] / den) * ch.v[a];
            const float angle = acosf(fminf(fmaxf(d, -1.f), 1.f));
            if ((angle <= half && j != i) || degenerate) count += 1.f;
        }
    }
    count = gsum<G>(count);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    fs_out[i] = count < 0.5f ? 1.f : 0.f;
    if (count_out) count_out[i] = count;
    if (normals_out) store_vec<D>(normals_out, i, ch);
}

// Maronne (wp_maronne.py:57-161, maronneDetection.py): with T_i = x_i + n_i H_i / xi and
// the tangent tau_i ((-n1, n0) in 2D, (n1 n2, -n0 n2, n0 n1) in 3D), the count of the
// neighbours j != i with r_ij < H_j and either r_ij >= sqrt(2) H_j / xi and |x_j - T_i| <=
// H_j / xi, or r_ij < sqrt(2) H_j / xi and |n_i . (x_j - T_i)| + |tau_i . (x_j - T_i)| <
// H_j / xi, for a normal of length above 0.5.  The mask is count < 0.5.
template <int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_maronne(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ normals,
          const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt, const int32_t* __restrict__ list,
          float* __restrict__ fs_out, float* __restrict__ count_out) {
    Grp<G> g(n);
    float count = 0.f;
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i), ni = load_vec<D>(normals, i);
        const float Hi = H[i], xi_k = P.kxi;
        Vec<D> T, tau = vzero<D>();
        #pragma unroll
        for (int a = 0; a < D; ++a) T.v[a] = xi.v[a] + ni.v[a] * Hi / xi_k;
        if constexpr (D == 2) { tau.v[0] = -ni.v[1]; tau.v[1] = ni.v[0]; }
        if constexpr (D == 3) { tau.v[0] = ni.v[1] * ni.v[2]; tau.v[1] = -ni.v[0] * ni.v[2]; tau.v[2] = ni.v[0] * ni.v[1]; }
        const bool long_normal = safe_sqrt(dot<D>(ni, ni)) > 0.5f;
        const float s2 = sqrtf(2.f);
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            const Vec<D> xj = load_vec<D>(x, j);
            const Vec<D> xij = dist_vec<D>(xi, xj, P.dom);
            const float rij = safe_sqrt(dot<D>(xij, xij));
            const float hij = __ldg(H + j);
            if (rij >= hij) continue;
            const Vec<D> xjt = dist_vec<D>(xj, T, P.dom);
            const float rjt = safe_sqrt(dot<D>(xjt, xjt));
            const float lim = hij / xi_k;
            const bool condA = rij >= s2 * hij / xi_k && rjt <= lim && j != i;
            const bool condB = rij < s2 * hij / xi_k && fabsf(dot<D>(ni, xjt)) + fabsf(dot<D>(tau, xjt)) < lim && j != i;
            if ((condA || condB) && long_normal) count += 1.f;
        }
    }
    count = gsum<G>(count);
    if (!g.valid || g.lane != 0) return;
    fs_out[g.i] = count < 0.5f ? 1.f : 0.f;
    if (count_out) count_out[g.i] = count;
}

// The colour-field-gradient scheme (colorFieldGradientDetection.py:18-56): the gather
// difference gradient of the colour field, the mask |grad c_i| > threshold H_i / xi and
// the normal -grad c_i / max(|grad c_i|, 1e-12).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_color_grad_detect(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                    const float* __restrict__ rho, const float* __restrict__ c, const int32_t* __restrict__ offs,
                    const int32_t* __restrict__ cnt, const int32_t* __restrict__ list, float threshold,
                    float* __restrict__ fs_out, float* __restrict__ normals_out) {
    Grp<G> g(n);
    Vec<D> gc = vzero<D>();
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float invHi = 1.f / H[i], ci = c[i];
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, safe_sqrt(dot<D>(xij, xij)), invHi, W, gW);
            if (W == 0.f) continue;
            const float dq = __ldg(m + j) / __ldg(rho + j) * (__ldg(c + j) - ci);
            #pragma unroll
            for (int a = 0; a < D; ++a) gc.v[a] += dq * gW.v[a];
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) gc.v[a] = gsum<G>(gc.v[a]);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    fs_out[i] = sqrtf(dot<D>(gc, gc)) > threshold * H[i] / P.kxi ? 1.f : 0.f;
    if (normals_out) {
        Vec<D> nn = tnormalize<D>(gc);
        #pragma unroll
        for (int a = 0; a < D; ++a) nn.v[a] = -nn.v[a];
        store_vec<D>(normals_out, i, nn);
    }
}

// M_i = sum_j V_j (x_j - x_i) (x) grad_i W(r_ij, max(H_i, H_j)), V_j = m_j / rho_j; L_i =
// pinv(M_i) (FP64, torch's default cutoff for FP32); lambda_i = min |eig(M_i)|, the smallest
// singular value of the symmetric M_i.
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_renormalization(int n, DevParams P, const float* __restrict__ x, const float* __restrict__ H, const float* __restrict__ m,
                  const float* __restrict__ rho, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                  const int32_t* __restrict__ list, float* __restrict__ L_out, float* __restrict__ lambda_out) {
    Grp<G> g(n);
    float M[D][D];
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) M[a][b] = 0.f;
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float Hi = H[i];
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, safe_sqrt(dot<D>(xij, xij)), 1.f / wmax(Hi, __ldg(H + j)), W, gW);
            if (W == 0.f) continue;
            const float Vj = __ldg(m + j) / __ldg(rho + j);
            #pragma unroll
            for (int a = 0; a < D; ++a)
                #pragma unroll
                for (int b = 0; b < D; ++b) M[a][b] += Vj * (-xij.v[a]) * gW.v[b];
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) M[a][b] = gsum<G>(M[a][b]);
    if (!g.valid || g.lane != 0) return;
    double A[D][D], Pm[D][D];
    #pragma unroll
    for (int a = 0; a < D; ++a)
        #pragma unroll
        for (int b = 0; b < D; ++b) A[a][b] = (double)M[a][b];
    double smin = 0.0;
    pinv_jacobi<D>(A, Pm, (double)D * 1.1920928955078125e-07, &smin);
    const int i = g.i;
    if (L_out) {
        #pragma unroll
        for (int a = 0; a < D; ++a)
            #pragma unroll
            for (int b = 0; b < D; ++b) L_out[(size_t)i * D * D + a * D + b] = (float)Pm[a][b];
    }
    if (lambda_out) lambda_out[i] = (float)smin;
}

// Normals from the renormalised gradients, n_i = -normalize(L_i g_i) with torch's
// normalise: mode 0 (lambdaGrad.py:46-83) g_i = sum_j V_j (lambda_j - lambda_i) grad W(r_ij, H_j)
// (the difference gradient under scatter support); mode 1 (maronneNormals.py:16-62) g_i =
// sum_j V_j grad W(r_ij, H_j) (the naive gradient of ones).
template <int KF, int D, int G>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_renorm_normals(int n, DevParams P, int mode, const float* __restrict__ x, const float* __restrict__ H,
                 const float* __restrict__ m, const float* __restrict__ rho, const float* __restrict__ L,
                 const float* __restrict__ lam, const int32_t* __restrict__ offs, const int32_t* __restrict__ cnt,
                 const int32_t* __restrict__ list, float* __restrict__ normals_out, float* __restrict__ grad_out) {
    Grp<G> g(n);
    Vec<D> gs = vzero<D>();
    if (g.valid) {
        const int i = g.i;
        const Vec<D> xi = load_vec<D>(x, i);
        const float li = mode == 0 ? lam[i] : 0.f;
        for (int q = offs[i] + g.lane, e = offs[i] + cnt[i]; q < e; q += G) {
            int j, k; entry(list, q, j, k);
            Vec<D> xij = dist_vec<D>(xi, load_vec<D>(x, j), P.dom);
            float W; Vec<D> gW;
            kWG_inv<KF, D>(xij, safe_sqrt(dot<D>(xij, xij)), 1.f / __ldg(H + j), W, gW);
            if (W == 0.f) continue;
            const float Vj = __ldg(m + j) / __ldg(rho + j);
            const float w = mode == 0 ? Vj * (__ldg(lam + j) - li) : Vj;
            #pragma unroll
            for (int a = 0; a < D; ++a) gs.v[a] += w * gW.v[a];
        }
    }
    #pragma unroll
    for (int a = 0; a < D; ++a) gs.v[a] = gsum<G>(gs.v[a]);
    if (!g.valid || g.lane != 0) return;
    const int i = g.i;
    const Mat<D> Li = load_mat<D>(L, i);
    const Vec<D> v = matvec<D>(Li, gs);
    if (grad_out) store_vec<D>(grad_out, i, v);
    Vec<D> nn = tnormalize<D>(v);
    #pragma unroll
    for (int a = 0; a < D; ++a) nn.v[a] = -nn.v[a];
    store_vec<D>(normals_out, i, nn);
}

}  // namespace

extern "C" {

int sph_surface_color_field(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                            const int32_t* offs, const int32_t* cnt, const int32_t* list, float* color_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(color_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_color_field<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, m, rho, offs, cnt,
                                                                                                      list, color_out)));
    return check_launch("sph_surface_color_field");
}

int sph_surface_detect_color_field(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                                   const float* color, const int32_t* offs, const int32_t* cnt, const int32_t* list,
                                   float neighbor_limit, float normal_sign, float* fs_out, float* normals_out,
                                   float* num_neighbors_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(color); WSPH_CHECK_PTR(fs_out);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_color_detect<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, m, rho, color, offs,
                                                                                                       cnt, list, neighbor_limit, normal_sign,
                                                                                                       fs_out, normals_out, num_neighbors_out)));
    return check_launch("sph_surface_detect_color_field");
}

int sph_surface_dilate(const SphParams* p, int64_t n, const float* x, const float* H, const float* fs_in, const int32_t* offs,
                       const int32_t* cnt, const int32_t* list, float* fs_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(fs_in); WSPH_CHECK_PTR(fs_out); CHECK_CSR();
    if (fs_in == fs_out) return set_error(SPH_ERR_BAD_ARG, "sph_surface_dilate: fs_in and fs_out must not alias");
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_dilate<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, fs_in, offs, cnt, list,
                                                                                                 fs_out)));
    return check_launch("sph_surface_dilate");
}

int sph_surface_barecasco(const SphParams* p, int64_t n, const float* x, const float* H, const int32_t* offs, const int32_t* cnt,
                          const int32_t* list, float threshold, float* fs_out, float* normals_out, float* count_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(fs_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, normals_out, "normals_out"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_barecasco<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, offs, cnt, list,
                                                                                                    threshold, fs_out, normals_out,
                                                                                                    count_out)));
    return check_launch("sph_surface_barecasco");
}

int sph_surface_maronne(const SphParams* p, int64_t n, const float* x, const float* H, const float* normals, const int32_t* offs,
                        const int32_t* cnt, const int32_t* list, float* fs_out, float* count_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(normals); WSPH_CHECK_PTR(fs_out); CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, normals, "normals"))) return rc;
    count_launch();
    WSPH_DISPATCH_DS(*p, (k_maronne<D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, normals, offs, cnt, list,
                                                                                            fs_out, count_out)));
    return check_launch("sph_surface_maronne");
}

int sph_surface_detect_color_gradient(const SphParams* p, int64_t n, const float* x, const float* H, const float* m,
                                      const float* rho, const float* color, const int32_t* offs, const int32_t* cnt,
                                      const int32_t* list, float threshold, float* fs_out, float* normals_out, void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(color); WSPH_CHECK_PTR(fs_out);
    CHECK_CSR();
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, normals_out, "normals_out"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_color_grad_detect<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
                              (int)n, P, x, H, m, rho, color, offs, cnt, list, threshold, fs_out, normals_out)));
    return check_launch("sph_surface_detect_color_gradient");
}

int sph_surface_renormalization(const SphParams* p, int64_t n, const float* x, const float* H, const float* m, const float* rho,
                                const int32_t* offs, const int32_t* cnt, const int32_t* list, float* L_out, float* lambda_out,
                                void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); CHECK_CSR();
    if (!L_out && !lambda_out) return set_error(SPH_ERR_BAD_ARG, "sph_surface_renormalization: no output");
    if ((rc = check_align_vec(P, x, "x"))) return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_renormalization<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>((int)n, P, x, H, m, rho, offs,
                                                                                                          cnt, list, L_out, lambda_out)));
    return check_launch("sph_surface_renormalization");
}

int sph_surface_renormalized_normals(const SphParams* p, int64_t n, int32_t mode, const float* x, const float* H, const float* m,
                                     const float* rho, const float* L, const float* lambdas, const int32_t* offs,
                                     const int32_t* cnt, const int32_t* list, float* normals_out, float* grad_out,
                                     void* stream) {
    PAIR_PRELUDE();
    WSPH_CHECK_PTR(x); WSPH_CHECK_PTR(H); WSPH_CHECK_PTR(m); WSPH_CHECK_PTR(rho); WSPH_CHECK_PTR(L); WSPH_CHECK_PTR(normals_out);
    CHECK_CSR();
    if (mode != 0 && mode != 1) return set_error(SPH_ERR_BAD_ARG, "sph_surface_renormalized_normals: mode must be 0 or 1");
    if (mode == 0) WSPH_CHECK_PTR(lambdas);
    if ((rc = check_align_vec(P, x, "x")) || (rc = check_align_vec(P, normals_out, "normals_out")) ||
        (rc = check_align_vec(P, grad_out, "grad_out")))
        return rc;
    count_launch();
    WSPH_DISPATCH_KDS(*p, (k_renorm_normals<KF, D, G_LIGHT><<<grid_g<G_LIGHT>(n), PAIR_BLOCK, 0, s>>>(
                              (int)n, P, mode, x, H, m, rho, L, lambdas, offs, cnt, list, normals_out, grad_out)));
    return check_launch("sph_surface_renormalized_normals");
}

}  // extern "C"
