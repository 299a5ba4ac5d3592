// Free-surface detection passes (modules/surfaceDetection): the colour field and its gather
// difference gradient (colorFieldCompute.py:11-45), the colour-field detection
// (colorFieldDetection.py:16-73) with the neighbour counts and sums of util/wp_numNeighbors.py
// and util/wp_sum.py under super-symmetric support, and the mask dilation (dilation.py,
// wp_dilate.py:14-89).  Each pass walks the interacting prefixes of the Verlet rows, which
// hold every pair with r < max(H_i, H_j).
#include <cuda_runtime.h>
#include "sph_pair_common.cuh"

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

}  // extern "C"
