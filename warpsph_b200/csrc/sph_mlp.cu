// Learned warm start for the DFSPH pressure solves: a per-particle MLP
//   8 features -> 64 -> 64 -> 64 -> 1, ReLU hidden layers,
// with FP32 master parameters, BF16 weights and activations into the tensor cores and
// FP32 accumulation.  No counterpart in the reference: it replaces the initial pressure
// guess of modules/incompressible/divergenceFree.py:72 (0.75 p_prev) and
// modules/incompressible/incompressible.py:79 (0).
//
// Tensor-core tiles: mma.sync m16n8k16 (BF16 x BF16 -> FP32).  One warp owns 16 samples;
// a hidden layer is 8 n-tiles x (K/16) k-steps.  The FP32 accumulator fragment of one
// layer maps onto the BF16 A fragment of the next without leaving registers:
//   A(k-block kb) = { C(n-tile 2kb)[0:2], C(2kb)[2:4], C(2kb+1)[0:2], C(2kb+1)[2:4] }.
// The weight-gradient GEMMs dW_l = dZ_l^T H_{l-1} contract over the 16 samples of the warp;
// their operands are staged transposed in per-warp shared memory.
//
// Parameter vector (FP32, SPH_MLP_PARAM_COUNT floats):
//   W1[64][8] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4[1]
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <mutex>
#include "sph_common.cuh"
#include "sph_tcgen05.cuh"

namespace wsph {

constexpr int MLP_IN = 8, MLP_H = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + MLP_H * MLP_IN, OFF_W2 = OFF_B1 + MLP_H, OFF_B2 = OFF_W2 + MLP_H * MLP_H,
              OFF_W3 = OFF_B2 + MLP_H, OFF_B3 = OFF_W3 + MLP_H * MLP_H, OFF_W4 = OFF_B3 + MLP_H, OFF_B4 = OFF_W4 + MLP_H,
              MLP_NPARAM = OFF_B4 + 1;
static_assert(MLP_NPARAM == SPH_MLP_PARAM_COUNT, "parameter layout");
constexpr int MLP_WARPS = 4;
constexpr int MLP_THREADS = 32 * MLP_WARPS;
constexpr int K1 = 16;   // layer-1 K padded to one mma k-step

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// Weights staged in shared memory as BF16.  W1s is [64][16] (K zero padded); WT are the
// transposes used by the backward data GEMMs.
struct MlpSmemW {
    __nv_bfloat16 W1[MLP_H * K1];
    __nv_bfloat16 W2[MLP_H * MLP_H];
    __nv_bfloat16 W3[MLP_H * MLP_H];
    float b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_H];
    float b4;
};

__device__ void stage_weights(const float* __restrict__ prm, MlpSmemW& s, __nv_bfloat16* W2T, __nv_bfloat16* W3T) {
    for (int t = threadIdx.x; t < MLP_H * K1; t += blockDim.x) {
        const int nrow = t / K1, k = t % K1;
        s.W1[t] = __float2bfloat16_rn(k < MLP_IN ? prm[OFF_W1 + nrow * MLP_IN + k] : 0.f);
    }
    for (int t = threadIdx.x; t < MLP_H * MLP_H; t += blockDim.x) {
        const int r = t / MLP_H, c = t % MLP_H;
        const __nv_bfloat16 w2 = __float2bfloat16_rn(prm[OFF_W2 + t]), w3 = __float2bfloat16_rn(prm[OFF_W3 + t]);
        s.W2[t] = w2;
        s.W3[t] = w3;
        if (W2T) { W2T[c * MLP_H + r] = w2; W3T[c * MLP_H + r] = w3; }
    }
    for (int t = threadIdx.x; t < MLP_H; t += blockDim.x) {
        s.b1[t] = prm[OFF_B1 + t]; s.b2[t] = prm[OFF_B2 + t]; s.b3[t] = prm[OFF_B3 + t]; s.w4[t] = prm[OFF_W4 + t];
    }
    if (threadIdx.x == 0) s.b4 = prm[OFF_B4];
}

// One hidden layer with K = 64: C[nt] = A x W^T (W row-major [64 out][64 in]) + bias, ReLU.
__device__ __forceinline__ void hidden_layer(const uint32_t (&A)[4][4], const __nv_bfloat16* W, const float* bias, int g, int t,
                                             float (&h)[8][4]) {
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16* wr = W + (nt * 8 + g) * MLP_H + 2 * t;
        #pragma unroll
        for (int ks = 0; ks < 4; ++ks) mma_bf16(c, A[ks][0], A[ks][1], A[ks][2], A[ks][3], lds32(wr + ks * 16), lds32(wr + ks * 16 + 8));
        const float bb0 = bias[nt * 8 + 2 * t], bb1 = bias[nt * 8 + 2 * t + 1];
        h[nt][0] = fmaxf(c[0] + bb0, 0.f); h[nt][1] = fmaxf(c[1] + bb1, 0.f);
        h[nt][2] = fmaxf(c[2] + bb0, 0.f); h[nt][3] = fmaxf(c[3] + bb1, 0.f);
    }
}
__device__ __forceinline__ void c_to_a(const float (&h)[8][4], uint32_t (&A)[4][4]) {
    #pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
        A[kb][0] = pack_bf16(h[2 * kb][0], h[2 * kb][1]);
        A[kb][1] = pack_bf16(h[2 * kb][2], h[2 * kb][3]);
        A[kb][2] = pack_bf16(h[2 * kb + 1][0], h[2 * kb + 1][1]);
        A[kb][3] = pack_bf16(h[2 * kb + 1][2], h[2 * kb + 1][3]);
    }
}
__device__ __forceinline__ void layer1(const float* __restrict__ feats, int64_t n, int64_t r0, int g, int t, const MlpSmemW& s,
                                       uint32_t (&A0)[4], float (&h1)[8][4]) {
    const int64_t ra = r0 + g, rb = r0 + g + 8;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
    if (ra < n) { x0 = feats[ra * MLP_IN + 2 * t]; x1 = feats[ra * MLP_IN + 2 * t + 1]; }
    if (rb < n) { x2 = feats[rb * MLP_IN + 2 * t]; x3 = feats[rb * MLP_IN + 2 * t + 1]; }
    A0[0] = pack_bf16(x0, x1); A0[1] = pack_bf16(x2, x3); A0[2] = 0u; A0[3] = 0u;
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16* wr = s.W1 + (nt * 8 + g) * K1 + 2 * t;
        mma_bf16(c, A0[0], A0[1], A0[2], A0[3], lds32(wr), lds32(wr + 8));
        const float bb0 = s.b1[nt * 8 + 2 * t], bb1 = s.b1[nt * 8 + 2 * t + 1];
        h1[nt][0] = fmaxf(c[0] + bb0, 0.f); h1[nt][1] = fmaxf(c[1] + bb1, 0.f);
        h1[nt][2] = fmaxf(c[2] + bb0, 0.f); h1[nt][3] = fmaxf(c[3] + bb1, 0.f);
    }
}
// y for rows g (out[0]) and g+8 (out[1]) of the warp tile, valid in lanes with t == 0.
__device__ __forceinline__ void output_layer(const float (&h3)[8][4], const MlpSmemW& s, int t, float& ya, float& yb) {
    float pa = 0.f, pb = 0.f;
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float w0 = s.w4[nt * 8 + 2 * t], w1 = s.w4[nt * 8 + 2 * t + 1];
        pa += h3[nt][0] * w0 + h3[nt][1] * w1;
        pb += h3[nt][2] * w0 + h3[nt][3] * w1;
    }
    pa += __shfl_xor_sync(0xffffffffu, pa, 1); pa += __shfl_xor_sync(0xffffffffu, pa, 2);
    pb += __shfl_xor_sync(0xffffffffu, pb, 1); pb += __shfl_xor_sync(0xffffffffu, pb, 2);
    ya = pa + s.b4;
    yb = pb + s.b4;
}

// ---------------------------------------------------------------- inference
__global__ void __launch_bounds__(MLP_THREADS)
k_mlp_forward(const float* __restrict__ prm, int64_t n, const float* __restrict__ feats, const float* __restrict__ scale,
              float* __restrict__ out) {
    __shared__ MlpSmemW s;
    stage_weights(prm, s, nullptr, nullptr);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const float sc = scale ? *scale : 1.f;
    for (int64_t r0 = ((int64_t)blockIdx.x * MLP_WARPS + warp) * 16; r0 < n; r0 += (int64_t)gridDim.x * MLP_WARPS * 16) {
        uint32_t A0[4], A[4][4];
        float h[8][4];
        layer1(feats, n, r0, g, t, s, A0, h);
        c_to_a(h, A);
        hidden_layer(A, s.W2, s.b2, g, t, h);
        c_to_a(h, A);
        hidden_layer(A, s.W3, s.b3, g, t, h);
        float ya, yb;
        output_layer(h, s, t, ya, yb);
        if (t == 0) {
            if (r0 + g < n) out[r0 + g] = ya * sc;
            if (r0 + g + 8 < n) out[r0 + g + 8] = yb * sc;
        }
    }
}

// ---------------------------------------------------------------- training: forward + backward
// Per warp: transposed BF16 copies of the layer inputs and of dZ for the weight GEMMs.
struct MlpWarpScratch {
    __nv_bfloat16 xT[K1 * 16];        // [k][r]
    __nv_bfloat16 h1T[MLP_H * 16];    // [c][r]
    __nv_bfloat16 h2T[MLP_H * 16];
    __nv_bfloat16 dzT[MLP_H * 16];
};
struct MlpSmemTrain {
    MlpSmemW w;
    __nv_bfloat16 W2T[MLP_H * MLP_H];
    __nv_bfloat16 W3T[MLP_H * MLP_H];
    float grad[MLP_NPARAM];
    MlpWarpScratch ws[MLP_WARPS];
    double loss[MLP_WARPS];
};

// Writes the fragment h (rows g, g+8; cols nt*8+2t, +1) transposed into dstT[c][r] as BF16.
__device__ __forceinline__ void store_T(const float (&h)[8][4], __nv_bfloat16* dstT, int g, int t) {
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * t;
        dstT[c * 16 + g] = __float2bfloat16_rn(h[nt][0]);
        dstT[(c + 1) * 16 + g] = __float2bfloat16_rn(h[nt][1]);
        dstT[c * 16 + g + 8] = __float2bfloat16_rn(h[nt][2]);
        dstT[(c + 1) * 16 + g + 8] = __float2bfloat16_rn(h[nt][3]);
    }
}
// grad[off + c*K + k] += sum_r dZT[c][r] * HT[k][r] over the warp's 16 samples, c < 64, k < kdim
// (kdim multiple of 8; HT rows beyond kdim are not read).
__device__ __forceinline__ void weight_grad(const __nv_bfloat16* dzT, const __nv_bfloat16* HT, int kdim, float* grad, int g, int t) {
    #pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        const __nv_bfloat16* ar = dzT + (mt * 16 + g) * 16 + 2 * t;
        const uint32_t a0 = lds32(ar), a1 = lds32(ar + 8 * 16), a2 = lds32(ar + 8), a3 = lds32(ar + 8 * 16 + 8);
        for (int nt = 0; nt < kdim / 8; ++nt) {
            const __nv_bfloat16* br = HT + (nt * 8 + g) * 16 + 2 * t;
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16(c, a0, a1, a2, a3, lds32(br), lds32(br + 8));
            const int row = mt * 16 + g, col = nt * 8 + 2 * t;
            atomicAdd(grad + row * kdim + col, c[0]);
            atomicAdd(grad + row * kdim + col + 1, c[1]);
            atomicAdd(grad + (row + 8) * kdim + col, c[2]);
            atomicAdd(grad + (row + 8) * kdim + col + 1, c[3]);
        }
    }
}
// Bias gradient: sum over the 16 rows of the dz fragment (rows g, g+8 in each lane).
__device__ __forceinline__ void bias_grad(const float (&dz)[8][4], float* gb, int g, int t) {
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float s0 = dz[nt][0] + dz[nt][2], s1 = dz[nt][1] + dz[nt][3];
        #pragma unroll
        for (int o = 4; o < 32; o <<= 1) { s0 += __shfl_xor_sync(0xffffffffu, s0, o); s1 += __shfl_xor_sync(0xffffffffu, s1, o); }
        if (g == 0) { atomicAdd(gb + nt * 8 + 2 * t, s0); atomicAdd(gb + nt * 8 + 2 * t + 1, s1); }
    }
}
// dH = dZ x W (W row-major [out][in], WT = its transpose [in][out]): M = 16 samples, N = 64 in, K = 64 out.
__device__ __forceinline__ void data_grad(const uint32_t (&A)[4][4], const __nv_bfloat16* WT, int g, int t, float (&dh)[8][4]) {
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16* br = WT + (nt * 8 + g) * MLP_H + 2 * t;
        #pragma unroll
        for (int ks = 0; ks < 4; ++ks) mma_bf16(c, A[ks][0], A[ks][1], A[ks][2], A[ks][3], lds32(br + ks * 16), lds32(br + ks * 16 + 8));
        dh[nt][0] = c[0]; dh[nt][1] = c[1]; dh[nt][2] = c[2]; dh[nt][3] = c[3];
    }
}
// dz = dh * relu'(z), with z > 0 read back from the BF16 activation hT[c][r].
__device__ __forceinline__ void relu_mask(float (&dh)[8][4], const __nv_bfloat16* hT, int g, int t) {
    #pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * t;
        if (!(__bfloat162float(hT[c * 16 + g]) > 0.f)) dh[nt][0] = 0.f;
        if (!(__bfloat162float(hT[(c + 1) * 16 + g]) > 0.f)) dh[nt][1] = 0.f;
        if (!(__bfloat162float(hT[c * 16 + g + 8]) > 0.f)) dh[nt][2] = 0.f;
        if (!(__bfloat162float(hT[(c + 1) * 16 + g + 8]) > 0.f)) dh[nt][3] = 0.f;
    }
}

// Mean-squared-error gradient over n samples: grad (FP32, MLP_NPARAM) += d/dtheta of
// (1/n) sum_r (y_r - target_r)^2, and *loss += sum_r (y_r - target_r)^2 (FP64).
__global__ void __launch_bounds__(MLP_THREADS)
k_mlp_grad(const float* __restrict__ prm, int64_t n, const float* __restrict__ feats, const float* __restrict__ target,
           float* __restrict__ grad, double* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmemTrain& S = *reinterpret_cast<MlpSmemTrain*>(smem_raw);
    stage_weights(prm, S.w, S.W2T, S.W3T);
    for (int q = threadIdx.x; q < MLP_NPARAM; q += blockDim.x) S.grad[q] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    MlpWarpScratch& W = S.ws[warp];
    const float inv_n = 1.f / (float)n;
    double lsum = 0.0;
    for (int64_t r0 = ((int64_t)blockIdx.x * MLP_WARPS + warp) * 16; r0 < n; r0 += (int64_t)gridDim.x * MLP_WARPS * 16) {
        const int64_t ra = r0 + g, rb = r0 + g + 8;
        // ---- forward (keeps h3 in FP32, h1/h2/x transposed in BF16)
        uint32_t A0[4], A[4][4];
        float h1[8][4], h2[8][4], h3[8][4];
        layer1(feats, n, r0, g, t, S.w, A0, h1);
        {   // x^T for dW1 (cols 0..7 real, 8..15 zero)
            float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
            if (ra < n) { x0 = feats[ra * MLP_IN + 2 * t]; x1 = feats[ra * MLP_IN + 2 * t + 1]; }
            if (rb < n) { x2 = feats[rb * MLP_IN + 2 * t]; x3 = feats[rb * MLP_IN + 2 * t + 1]; }
            W.xT[(2 * t) * 16 + g] = __float2bfloat16_rn(x0);
            W.xT[(2 * t + 1) * 16 + g] = __float2bfloat16_rn(x1);
            W.xT[(2 * t) * 16 + g + 8] = __float2bfloat16_rn(x2);
            W.xT[(2 * t + 1) * 16 + g + 8] = __float2bfloat16_rn(x3);
        }
        store_T(h1, W.h1T, g, t);
        c_to_a(h1, A);
        hidden_layer(A, S.w.W2, S.w.b2, g, t, h2);
        store_T(h2, W.h2T, g, t);
        c_to_a(h2, A);
        hidden_layer(A, S.w.W3, S.w.b3, g, t, h3);
        float ya, yb;
        output_layer(h3, S.w, t, ya, yb);
        // ---- loss and dy (same value in the four lanes of a row group)
        const float ta = ra < n ? target[ra] : ya, tb = rb < n ? target[rb] : yb;
        const float ea = ra < n ? ya - ta : 0.f, eb = rb < n ? yb - tb : 0.f;
        if (t == 0) lsum += (double)ea * ea + (double)eb * eb;
        const float dya = 2.f * ea * inv_n, dyb = 2.f * eb * inv_n;
        // ---- layer 4: dW4 = sum dy h3, db4 = sum dy; dz3 = dy w4 * relu'(z3)
        float dz[8][4];
        #pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int c = nt * 8 + 2 * t;
            float s0 = dya * h3[nt][0] + dyb * h3[nt][2], s1 = dya * h3[nt][1] + dyb * h3[nt][3];
            #pragma unroll
            for (int o = 4; o < 32; o <<= 1) { s0 += __shfl_xor_sync(0xffffffffu, s0, o); s1 += __shfl_xor_sync(0xffffffffu, s1, o); }
            if (g == 0) { atomicAdd(S.grad + OFF_W4 + c, s0); atomicAdd(S.grad + OFF_W4 + c + 1, s1); }
            const float w0 = S.w.w4[c], w1 = S.w.w4[c + 1];
            dz[nt][0] = h3[nt][0] > 0.f ? dya * w0 : 0.f;
            dz[nt][1] = h3[nt][1] > 0.f ? dya * w1 : 0.f;
            dz[nt][2] = h3[nt][2] > 0.f ? dyb * w0 : 0.f;
            dz[nt][3] = h3[nt][3] > 0.f ? dyb * w1 : 0.f;
        }
        {
            float sd = dya + dyb;
            #pragma unroll
            for (int o = 4; o < 32; o <<= 1) sd += __shfl_xor_sync(0xffffffffu, sd, o);
            if (lane == 0) atomicAdd(S.grad + OFF_B4, sd);
        }
        // ---- layer 3
        bias_grad(dz, S.grad + OFF_B3, g, t);
        store_T(dz, W.dzT, g, t);
        __syncwarp();
        weight_grad(W.dzT, W.h2T, MLP_H, S.grad + OFF_W3, g, t);
        c_to_a(dz, A);
        data_grad(A, S.W3T, g, t, dz);       // dz <- dh2
        relu_mask(dz, W.h2T, g, t);          // dz2
        __syncwarp();
        // ---- layer 2
        bias_grad(dz, S.grad + OFF_B2, g, t);
        store_T(dz, W.dzT, g, t);
        __syncwarp();
        weight_grad(W.dzT, W.h1T, MLP_H, S.grad + OFF_W2, g, t);
        c_to_a(dz, A);
        data_grad(A, S.W2T, g, t, dz);       // dh1
        relu_mask(dz, W.h1T, g, t);          // dz1
        __syncwarp();
        // ---- layer 1 (K = 8 real inputs)
        bias_grad(dz, S.grad + OFF_B1, g, t);
        store_T(dz, W.dzT, g, t);
        __syncwarp();
        weight_grad(W.dzT, W.xT, MLP_IN, S.grad + OFF_W1, g, t);
        __syncwarp();
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) S.loss[warp] = lsum;
    __syncthreads();
    for (int q = threadIdx.x; q < MLP_NPARAM; q += blockDim.x) {
        const float v = S.grad[q];
        if (v != 0.f) atomicAdd(grad + q, v);
    }
    if (threadIdx.x == 0) {
        double l = 0.0;
        for (int w = 0; w < MLP_WARPS; ++w) l += S.loss[w];
        atomicAdd(loss, l);
    }
}

// Adam (Kingma & Ba 2015) with bias correction, elementwise over the parameter vector.
__global__ void k_mlp_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m1, float* __restrict__ m2,
                           int64_t count, float lr, float beta1, float beta2, float eps, float c1, float c2) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x) {
        const float gq = grad[q];
        const float a = beta1 * m1[q] + (1.f - beta1) * gq;
        const float b = beta2 * m2[q] + (1.f - beta2) * gq * gq;
        m1[q] = a;
        m2[q] = b;
        prm[q] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

// ---------------------------------------------------------------- inference on tcgen05
// One CTA of 4 warps takes 128 samples per tile.  Each layer is one chain of
//   D[128 x 64] (TMEM, FP32) = A[128 x K] (TMEM, BF16) x W[64 x K]^T (shared, BF16)
// of K/16 tcgen05.mma kind::f16 instructions with A read from tensor memory, issued by one
// thread and completed through tcgen05.commit on an mbarrier.  Warp w then reads TMEM
// lanes 32w..32w+31 of D (one sample per thread, tcgen05.ld 32x32b), applies ReLU while
// rounding to BF16 (cvt.rn.relu) and stores the packed pairs straight back into the A
// columns of the next layer (tcgen05.st 32x32b).  Activations never pass through shared
// memory, which holds only the weights: with A in shared memory every MMA re-read its
// activations from there (about 98 KB of shared-memory traffic per tile, the limit).
// The 64 -> 1 output layer is an FP32 dot product in registers.
//
// The biases ride in the contraction: A carries two constant-one columns after its real K
// columns (X columns 8, 9; H columns 64, 65) and W the bias split into BF16 hi + lo parts
// in the matching columns, so the FP32 accumulator receives b_hi + b_lo, which equals the
// FP32 bias to about 2^-17 relative.  The hidden layers thus run K = 80 (five k-steps).
// Rounding points otherwise match k_mlp_forward: BF16 features, weights and hidden
// activations, FP32 accumulation, FP32 output layer.
//
// TMEM columns of a CTA (128 allocated, 32-bit each):
//   0..63    D, the FP32 accumulator
//   64..103  H, the hidden-layer A operand: 64 BF16 activations (64..95), then 1, 1, 0... (96..103)
//   104..111 X, the layer-1 A operand: 8 BF16 features (104..107), then 1, 1, 0... (108..111)
constexpr int TC_M = 128, TC_THREADS = 128, TC_TMEM_COLS = 128, TC_CTAS_PER_SM = 4;
constexpr int TC_K2 = MLP_H + 16;   // hidden-layer K with the bias columns
constexpr uint32_t TC_COL_D = 0, TC_COL_H = 64, TC_COL_X = 104;
constexpr uint32_t TC_IDESC = umma_idesc_bf16_f32<TC_M, MLP_H>();
static_assert(TC_IDESC == 0x08100490u, "kind::f16 descriptor: BF16 x BF16 -> FP32, M = 128, N = 64, K-major");
static_assert(TC_COL_H >= TC_COL_D + MLP_H && TC_COL_X >= TC_COL_H + TC_K2 / 2 && TC_COL_X + K1 / 2 <= TC_TMEM_COLS,
              "TMEM column plan");
constexpr long long TC_WAIT_CYCLES = 1ll << 31;   // about a second at B200 clocks

struct MlpTcSmem {
    __nv_bfloat16 W1[MLP_H * K1];      // [64 x 16]: W1 | b1 hi | b1 lo | 0
    __nv_bfloat16 W2[MLP_H * TC_K2];   // [64 x 80]: W2 | b2 hi | b2 lo | 0
    __nv_bfloat16 W3[MLP_H * TC_K2];
    float w4[MLP_H];
    unsigned long long bar;
    float b4;
    uint32_t tmem_base;
    int abort;
    // keeps the CTA above a fifth of the SM's shared memory, so that no more than the 4
    // CTAs whose 128 TMEM columns fit in 512 are resident on one SM
    unsigned char occupancy_pad[24 * 1024];
};
static_assert((sizeof(__nv_bfloat16) * MLP_H * K1) % 128 == 0 && (sizeof(__nv_bfloat16) * MLP_H * TC_K2) % 128 == 0,
              "128 B aligned operands");
static_assert(4 * (sizeof(MlpTcSmem) + 1024) <= 228 * 1024 && 5 * (sizeof(MlpTcSmem) + 1024) > 228 * 1024 &&
              4 * TC_TMEM_COLS <= 512, "4 resident CTAs per SM, within the SM's TMEM columns");

// relu of (lo, hi) rounded to BF16 and packed, lo in the low half
__device__ __forceinline__ uint32_t relu_bf16x2(uint32_t lo, uint32_t hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(__uint_as_float(hi)), "f"(__uint_as_float(lo)));
    return d;
}
// Column `part` of the bias block: 0 -> BF16 hi part of b, 1 -> BF16 lo part
// (hi + lo reproduces b to about 2^-17 relative), 2.. -> 0.
__device__ __forceinline__ __nv_bfloat16 bias_part(float b, int part) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(b);
    return part == 0 ? hi : part == 1 ? __float2bfloat16_rn(b - __bfloat162float(hi)) : __float2bfloat16_rn(0.f);
}

__global__ void __launch_bounds__(TC_THREADS, TC_CTAS_PER_SM)
k_mlp_forward_tc(const float* __restrict__ prm, int64_t n, const float* __restrict__ feats, const float* __restrict__ scale,
                 float* __restrict__ out, int32_t* __restrict__ status) {
    __shared__ __align__(128) MlpTcSmem s;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        tmem_alloc(smem_u32(&s.tmem_base), TC_TMEM_COLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(smem_u32(&s.bar), 1);
        s.abort = 0;
        fence_mbar_init();
    }
    // weights in the K-major core-matrix layout (B operands: rows = output units)
    for (int t = tid; t < MLP_H * K1; t += TC_THREADS) {
        const int r = t / K1, k = t % K1;
        s.W1[umma_k_index(r, k, MLP_H)] = k < MLP_IN ? __float2bfloat16_rn(prm[OFF_W1 + r * MLP_IN + k])
                                                     : bias_part(prm[OFF_B1 + r], k - MLP_IN);
    }
    for (int t = tid; t < MLP_H * TC_K2; t += TC_THREADS) {
        const int r = t / TC_K2, k = t % TC_K2;
        const bool w = k < MLP_H;
        s.W2[umma_k_index(r, k, MLP_H)] = w ? __float2bfloat16_rn(prm[OFF_W2 + r * MLP_H + k]) : bias_part(prm[OFF_B2 + r], k - MLP_H);
        s.W3[umma_k_index(r, k, MLP_H)] = w ? __float2bfloat16_rn(prm[OFF_W3 + r * MLP_H + k]) : bias_part(prm[OFF_B3 + r], k - MLP_H);
    }
    if (tid < MLP_H) s.w4[tid] = prm[OFF_W4 + tid];
    if (tid == 0) s.b4 = prm[OFF_B4];
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();

    const uint32_t tbase = s.tmem_base;
    const uint32_t tlane = tbase + (static_cast<uint32_t>(warp * 32) << 16);   // this warp's 32 lanes
    {   // the constant columns of this thread's row of H and X, the same for every tile
        const uint32_t one2 = pack_bf16(1.f, 1.f);
        const uint32_t hb[8] = {one2, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        tmem_st_32x32b_x8(tlane + TC_COL_H + MLP_H / 2, hb);
        tmem_st_32x32b_x4(tlane + TC_COL_X + MLP_IN / 2, one2, 0u, 0u, 0u);
        tmem_st_wait();
    }
    const uint32_t bar = smem_u32(&s.bar);
    const uint32_t aW1 = smem_u32(s.W1), aW2 = smem_u32(s.W2), aW3 = smem_u32(s.W3);
    const uint32_t LBO_B = MLP_H * 16, SBO = 128;
    const float sc = scale ? *scale : 1.f;
    const int64_t ntiles = (n + TC_M - 1) / TC_M;
    uint32_t phase = 0;
    int64_t tile = blockIdx.x;
    for (; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * TC_M + tid;
        {   // layer-1 operand: this thread's sample, 8 features -> 4 packed BF16 pairs
            float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f), f1 = f0;
            if (row < n) {
                f0 = __ldg(reinterpret_cast<const float4*>(feats + row * MLP_IN));
                f1 = __ldg(reinterpret_cast<const float4*>(feats + row * MLP_IN) + 1);
            }
            tmem_st_32x32b_x4(tlane + TC_COL_X, pack_bf16(f0.x, f0.y), pack_bf16(f0.z, f0.w), pack_bf16(f1.x, f1.y),
                              pack_bf16(f1.z, f1.w));
            tmem_st_wait();
        }
        tc_fence_before_sync();
        __syncthreads();
        float y = 0.f;
        #pragma unroll 1
        for (int layer = 0; layer < 3; ++layer) {
            if (tid == 0) {
                tc_fence_after_sync();
                if (layer == 0) {
                    umma_bf16_ts(tbase + TC_COL_D, tbase + TC_COL_X, umma_desc_kmajor(aW1, LBO_B, SBO), TC_IDESC, 0u);
                } else {
                    const uint32_t aW = layer == 1 ? aW2 : aW3;
                    #pragma unroll
                    for (int ks = 0; ks < TC_K2 / 16; ++ks)
                        umma_bf16_ts(tbase + TC_COL_D, tbase + TC_COL_H + ks * 8, umma_desc_kmajor(aW + ks * 2 * LBO_B, LBO_B, SBO),
                                     TC_IDESC, ks > 0 ? 1u : 0u);
                }
                umma_commit(bar);
            }
            const bool done = mbar_wait_bounded(bar, phase, TC_WAIT_CYCLES);
            phase ^= 1u;
            if (!done) s.abort = 1;
            __syncthreads();
            if (s.abort) break;
            tc_fence_after_sync();
            #pragma unroll
            for (int cb = 0; cb < MLP_H; cb += 32) {
                uint32_t v[32];
                tmem_ld_32x32b_x32(tlane + TC_COL_D + cb, v);
                tmem_ld_wait(v);
                if (layer < 2) {
                    uint32_t h[16];
                    #pragma unroll
                    for (int j = 0; j < 16; ++j) h[j] = relu_bf16x2(v[2 * j], v[2 * j + 1]);
                    const uint32_t (&h0)[8] = *reinterpret_cast<const uint32_t(*)[8]>(h);
                    const uint32_t (&h1)[8] = *reinterpret_cast<const uint32_t(*)[8]>(h + 8);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2, h0);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2 + 8, h1);
                } else {
                    #pragma unroll
                    for (int j = 0; j < 32; ++j) y = fmaf(fmaxf(__uint_as_float(v[j]), 0.f), s.w4[cb + j], y);
                }
            }
            if (layer < 2) {
                tmem_st_wait();
                tc_fence_before_sync();
                __syncthreads();
            }
        }
        if (s.abort) break;
        if (row < n) out[row] = (y + s.b4) * sc;
    }
    if (s.abort) {
        // a chain did not complete in time: the samples of this and later tiles get NaN.
        // The MMA chain and its commit may still be in flight, so the issuing thread waits
        // once more (bounded) for that commit before the TMEM columns are released; the
        // timeout status tells the host that the context is suspect, and the host stops
        // issuing work to this device's MLP after it.
        for (; tile < ntiles; tile += gridDim.x) {
            const int64_t row = tile * TC_M + tid;
            if (row < n) out[row] = __int_as_float(0x7fc00000);
        }
        if (tid == 0) {
            (void)mbar_wait_bounded(bar, phase ^ 1u, TC_WAIT_CYCLES);
            if (status) atomicOr(status, SPH_STATUS_TIMEOUT);
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after_sync();
        tmem_dealloc(tbase, TC_TMEM_COLS);
    }
}

// ---------------------------------------------------------------- training on tcgen05
// The gradient of the mean squared error with every GEMM on the tensor cores.  One CTA per
// SM (4 warps, one sample per thread and TMEM lane) loops over 128-sample tiles:
//   forward   the three hidden layers as in k_mlp_forward_tc (TS form, biases in the
//             contraction), keeping each layer's BF16 input transposed in shared memory
//             (XT, H1T, H2T: rows = input unit, K = sample) and the ReLU masks in registers;
//   output    y = h3 . w4 + b4 in FP32, dy = 2 (y - t) / n; the w4 and b4 gradients are
//             warp-reduced FP32 sums;
//   backward  dZ3 = dy w4 * [z3 > 0]; then per layer l = 3, 2, 1 two MMA chains:
//               G_l (+)= H_{l-1}^T dZ_l^T   (SS form, M = 128 input rows, N = 64 outputs,
//                                           K = 128 samples; accumulated in TMEM over the
//                                           CTA's tiles; the ones row of H^T gives db_l)
//               dH_{l-1} = dZ_l W_l          (TS form, A = dZ_l in TMEM, B = W_l^T)
//             and dZ_{l-1} = dH_{l-1} * [z_{l-1} > 0] in the epilogue.
// At the end each thread adds its TMEM lane of G_1..G_3 (one input unit, all outputs) to the
// global gradient with FP32 atomics.  Rounding points: BF16 inputs, weights, activations and
// dZ, FP32 accumulation, as the oracle's BF16 gradient (oracle/mlp.py); the bias gradients
// come from the BF16 dZ, which the oracle sums unrounded.
//
// TMEM columns (512, one CTA per SM):
//   0..63     D: layer outputs in the forward pass, dH in the backward pass (FP32)
//   64..103   H: the hidden A operand; in the backward pass columns 64..95 hold dZ (BF16)
//   104..111  X: the layer-1 A operand
//   128..191, 192..255, 256..319   G_1, G_2, G_3 (lane = input unit, column = output unit)
constexpr int GT_TMEM_COLS = 512;
constexpr uint32_t GT_COL_G1 = 128, GT_COL_G2 = 192, GT_COL_G3 = 256;

struct MlpGradTcSmem {
    __nv_bfloat16 W1[MLP_H * K1];      // B of layer 1 [64 x 16]: W1 | b1 hi | b1 lo | 0
    __nv_bfloat16 W2[MLP_H * TC_K2];   // B of layer 2 [64 x 80]
    __nv_bfloat16 W3[MLP_H * TC_K2];
    __nv_bfloat16 W2T[MLP_H * MLP_H];  // B of dH1 = dZ2 W2: rows = input unit, K = output unit
    __nv_bfloat16 W3T[MLP_H * MLP_H];
    __nv_bfloat16 XT[TC_M * TC_M];     // A of the weight GEMMs: rows = input unit (+ a ones row), K = sample
    __nv_bfloat16 H1T[TC_M * TC_M];
    __nv_bfloat16 H2T[TC_M * TC_M];
    __nv_bfloat16 DZT[MLP_H * TC_M];   // B of the weight GEMMs: rows = output unit, K = sample
    float w4[MLP_H];
    float gw4[MLP_H];
    float gb4;
    float b4;
    double loss;
    unsigned long long bar;
    uint32_t tmem_base;
    int abort;
};
static_assert(sizeof(MlpGradTcSmem) + 128 <= 227 * 1024, "one CTA per SM");

__device__ __forceinline__ float bf16_lo(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t p) { return __uint_as_float(p & 0xffff0000u); }
__device__ __forceinline__ __nv_bfloat16 bf16_bits(uint32_t b) { return __ushort_as_bfloat16(static_cast<unsigned short>(b)); }

__global__ void __launch_bounds__(TC_THREADS, 1)
k_mlp_grad_tc(const float* __restrict__ prm, int64_t n, const float* __restrict__ feats, const float* __restrict__ target,
              float* __restrict__ grad, double* __restrict__ loss_out, int32_t* __restrict__ status) {
    extern __shared__ unsigned char gt_dyn[];
    MlpGradTcSmem& s = *reinterpret_cast<MlpGradTcSmem*>((reinterpret_cast<uintptr_t>(gt_dyn) + 127) & ~static_cast<uintptr_t>(127));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        tmem_alloc(smem_u32(&s.tmem_base), GT_TMEM_COLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(smem_u32(&s.bar), 1);
        s.abort = 0;
        s.gb4 = 0.f;
        s.loss = 0.0;
        fence_mbar_init();
    }
    for (int t = tid; t < MLP_H * K1; t += TC_THREADS) {
        const int r = t / K1, k = t % K1;
        s.W1[umma_k_index(r, k, MLP_H)] = k < MLP_IN ? __float2bfloat16_rn(prm[OFF_W1 + r * MLP_IN + k])
                                                     : bias_part(prm[OFF_B1 + r], k - MLP_IN);
    }
    for (int t = tid; t < MLP_H * TC_K2; t += TC_THREADS) {
        const int r = t / TC_K2, k = t % TC_K2;
        const bool w = k < MLP_H;
        s.W2[umma_k_index(r, k, MLP_H)] = w ? __float2bfloat16_rn(prm[OFF_W2 + r * MLP_H + k]) : bias_part(prm[OFF_B2 + r], k - MLP_H);
        s.W3[umma_k_index(r, k, MLP_H)] = w ? __float2bfloat16_rn(prm[OFF_W3 + r * MLP_H + k]) : bias_part(prm[OFF_B3 + r], k - MLP_H);
    }
    for (int t = tid; t < MLP_H * MLP_H; t += TC_THREADS) {
        const int o = t / MLP_H, i = t % MLP_H;      // W[o][i]
        s.W2T[umma_k_index(i, o, MLP_H)] = __float2bfloat16_rn(prm[OFF_W2 + t]);
        s.W3T[umma_k_index(i, o, MLP_H)] = __float2bfloat16_rn(prm[OFF_W3 + t]);
    }
    {   // the ones rows of the transposed inputs (row MLP_IN of XT, row MLP_H of H1T and H2T)
        const __nv_bfloat16 one = __float2bfloat16_rn(1.f);
        s.XT[umma_k_index(MLP_IN, tid, TC_M)] = one;
        s.H1T[umma_k_index(MLP_H, tid, TC_M)] = one;
        s.H2T[umma_k_index(MLP_H, tid, TC_M)] = one;
    }
    if (tid < MLP_H) { s.w4[tid] = prm[OFF_W4 + tid]; s.gw4[tid] = 0.f; }
    if (tid == 0) s.b4 = prm[OFF_B4];
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();

    const uint32_t tbase = s.tmem_base;
    const uint32_t tlane = tbase + (static_cast<uint32_t>(warp * 32) << 16);
    {
        const uint32_t one2 = pack_bf16(1.f, 1.f);
        const uint32_t hb[8] = {one2, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        tmem_st_32x32b_x8(tlane + TC_COL_H + MLP_H / 2, hb);
        tmem_st_32x32b_x4(tlane + TC_COL_X + MLP_IN / 2, one2, 0u, 0u, 0u);
        tmem_st_wait();
    }
    const uint32_t bar = smem_u32(&s.bar);
    const uint32_t aW1 = smem_u32(s.W1), aW2 = smem_u32(s.W2), aW3 = smem_u32(s.W3), aW2T = smem_u32(s.W2T),
                   aW3T = smem_u32(s.W3T), aXT = smem_u32(s.XT), aH1T = smem_u32(s.H1T), aH2T = smem_u32(s.H2T),
                   aDZT = smem_u32(s.DZT);
    constexpr uint32_t LBO_64 = MLP_H * 16, LBO_128 = TC_M * 16, SBO = 128;
    const float inv_n = 2.f / static_cast<float>(n);
    const int64_t ntiles = (n + TC_M - 1) / TC_M;
    uint32_t phase = 0;
    bool first = true;
    int64_t tile = blockIdx.x;

    // one MMA phase: issue (thread 0), commit, bounded wait, then every thread may read TMEM
    auto sync_mma = [&](auto issue) -> bool {
        if (tid == 0) {
            tc_fence_after_sync();
            issue();
            umma_commit(bar);
        }
        const bool done = mbar_wait_bounded(bar, phase, TC_WAIT_CYCLES);
        phase ^= 1u;
        if (!done) s.abort = 1;
        __syncthreads();
        tc_fence_after_sync();
        return s.abort == 0;
    };
    // this thread's BF16 value of input unit c for sample tid into a transposed operand
    auto put_t = [&](__nv_bfloat16* dstT, int rows, int c, __nv_bfloat16 v) { dstT[umma_k_index(c, tid, rows)] = v; };
    auto finish_epilogue = [&]() {
        tmem_st_wait();
        fence_proxy_async_smem();
        tc_fence_before_sync();
        __syncthreads();
    };

    for (; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * TC_M + tid;
        const bool valid = row < n;
        {
            float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f), f1 = f0;
            if (valid) {
                f0 = __ldg(reinterpret_cast<const float4*>(feats + row * MLP_IN));
                f1 = __ldg(reinterpret_cast<const float4*>(feats + row * MLP_IN) + 1);
            }
            const uint32_t x01 = pack_bf16(f0.x, f0.y), x23 = pack_bf16(f0.z, f0.w), x45 = pack_bf16(f1.x, f1.y),
                           x67 = pack_bf16(f1.z, f1.w);
            tmem_st_32x32b_x4(tlane + TC_COL_X, x01, x23, x45, x67);
            const uint32_t xp[4] = {x01, x23, x45, x67};
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                put_t(s.XT, TC_M, 2 * j, bf16_bits(xp[j]));
                put_t(s.XT, TC_M, 2 * j + 1, bf16_bits(xp[j] >> 16));
            }
            finish_epilogue();
        }
        // ---- forward
        uint32_t mask[2][2] = {{0u, 0u}, {0u, 0u}};     // [layer][32-column half]: z > 0
        float dy = 0.f;
        #pragma unroll 1
        for (int layer = 0; layer < 3; ++layer) {
            const bool ok = sync_mma([&] {
                if (layer == 0) {
                    umma_bf16_ts(tbase + TC_COL_D, tbase + TC_COL_X, umma_desc_kmajor(aW1, LBO_64, SBO), TC_IDESC, 0u);
                } else {
                    const uint32_t aW = layer == 1 ? aW2 : aW3;
                    #pragma unroll
                    for (int ks = 0; ks < TC_K2 / 16; ++ks)
                        umma_bf16_ts(tbase + TC_COL_D, tbase + TC_COL_H + ks * 8, umma_desc_kmajor(aW + ks * 2 * LBO_64, LBO_64, SBO),
                                     TC_IDESC, ks > 0 ? 1u : 0u);
                }
            });
            if (!ok) break;
            float y = 0.f;
            #pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int cb = 32 * half;
                uint32_t v[32];
                tmem_ld_32x32b_x32(tlane + TC_COL_D + cb, v);
                tmem_ld_wait(v);
                if (layer < 2) {
                    uint32_t h[16], m = 0u;
                    #pragma unroll
                    for (int j = 0; j < 16; ++j) h[j] = relu_bf16x2(v[2 * j], v[2 * j + 1]);
                    #pragma unroll
                    for (int j = 0; j < 32; ++j) m |= (__uint_as_float(v[j]) > 0.f ? 1u : 0u) << j;
                    mask[layer][half] = m;
                    const uint32_t (&h0)[8] = *reinterpret_cast<const uint32_t(*)[8]>(h);
                    const uint32_t (&h1)[8] = *reinterpret_cast<const uint32_t(*)[8]>(h + 8);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2, h0);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2 + 8, h1);
                    __nv_bfloat16* dstT = layer == 0 ? s.H1T : s.H2T;
                    #pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        put_t(dstT, TC_M, cb + 2 * j, bf16_bits(h[j]));
                        put_t(dstT, TC_M, cb + 2 * j + 1, bf16_bits(h[j] >> 16));
                    }
                } else {
                    #pragma unroll
                    for (int j = 0; j < 32; ++j) y = fmaf(fmaxf(__uint_as_float(v[j]), 0.f), s.w4[cb + j], y);
                }
            }
            if (layer < 2) {
                finish_epilogue();
            } else {
                // ---- output layer and dZ3
                y += s.b4;
                const float e = valid ? y - __ldg(target + row) : 0.f;
                dy = e * inv_n;
                double le = static_cast<double>(e) * static_cast<double>(e);
                float gb = dy;
                #pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    le += __shfl_xor_sync(0xffffffffu, le, o);
                    gb += __shfl_xor_sync(0xffffffffu, gb, o);
                }
                if (lane == 0) { atomicAdd(&s.loss, le); atomicAdd(&s.gb4, gb); }
                #pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const int cb = 32 * half;
                    uint32_t v[32];      // z3 of this half, read again now that dy is known
                    tmem_ld_32x32b_x32(tlane + TC_COL_D + cb, v);
                    tmem_ld_wait(v);
                    uint32_t p[16];
                    {   // d loss / d w4_j summed over the warp's samples: a butterfly that
                        // halves the values per lane each round leaves lane l with column l
                        float g[32];
                        #pragma unroll
                        for (int j = 0; j < 32; ++j) g[j] = dy * fmaxf(__uint_as_float(v[j]), 0.f);
                        #pragma unroll
                        for (int off = 16; off >= 1; off >>= 1) {
                            const bool upper = (lane & off) != 0;
                            #pragma unroll
                            for (int t = 0; t < off; ++t) {
                                const float send = upper ? g[t] : g[t + off];
                                const float keep = upper ? g[t + off] : g[t];
                                g[t] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                            }
                        }
                        atomicAdd(&s.gw4[cb + lane], g[0]);
                    }
                    #pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float d0 = __uint_as_float(v[2 * j]) > 0.f ? dy * s.w4[cb + 2 * j] : 0.f;
                        const float d1 = __uint_as_float(v[2 * j + 1]) > 0.f ? dy * s.w4[cb + 2 * j + 1] : 0.f;
                        p[j] = pack_bf16(d0, d1);
                        put_t(s.DZT, MLP_H, cb + 2 * j, bf16_bits(p[j]));
                        put_t(s.DZT, MLP_H, cb + 2 * j + 1, bf16_bits(p[j] >> 16));
                    }
                    const uint32_t (&p0)[8] = *reinterpret_cast<const uint32_t(*)[8]>(p);
                    const uint32_t (&p1)[8] = *reinterpret_cast<const uint32_t(*)[8]>(p + 8);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2, p0);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2 + 8, p1);
                }
                finish_epilogue();
            }
        }
        if (s.abort) break;
        // ---- backward: l = 3, 2, 1
        #pragma unroll 1
        for (int l = 3; l >= 1; --l) {
            const uint32_t aA = l == 3 ? aH2T : (l == 2 ? aH1T : aXT);
            const uint32_t colG = l == 3 ? GT_COL_G3 : (l == 2 ? GT_COL_G2 : GT_COL_G1);
            const uint32_t aWT = l == 3 ? aW3T : aW2T;
            const bool acc0 = !first;
            const bool ok = sync_mma([&] {
                #pragma unroll
                for (int ks = 0; ks < TC_M / 16; ++ks)
                    umma_bf16_ss(tbase + colG, umma_desc_kmajor(aA + ks * 2 * LBO_128, LBO_128, SBO),
                                 umma_desc_kmajor(aDZT + ks * 2 * LBO_64, LBO_64, SBO), TC_IDESC, (acc0 || ks > 0) ? 1u : 0u);
                if (l > 1) {
                    #pragma unroll
                    for (int ks = 0; ks < MLP_H / 16; ++ks)
                        umma_bf16_ts(tbase + TC_COL_D, tbase + TC_COL_H + ks * 8, umma_desc_kmajor(aWT + ks * 2 * LBO_64, LBO_64, SBO),
                                     TC_IDESC, ks > 0 ? 1u : 0u);
                }
            });
            if (!ok) break;
            if (l == 1) break;
            // dZ_{l-1} = dH_{l-1} * [z_{l-1} > 0]
            #pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int cb = 32 * half;
                const uint32_t m = mask[l - 2][half];
                uint32_t v[32];
                tmem_ld_32x32b_x32(tlane + TC_COL_D + cb, v);
                tmem_ld_wait(v);
                uint32_t p[16];
                #pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float d0 = ((m >> (2 * j)) & 1u) ? __uint_as_float(v[2 * j]) : 0.f;
                    const float d1 = ((m >> (2 * j + 1)) & 1u) ? __uint_as_float(v[2 * j + 1]) : 0.f;
                    p[j] = pack_bf16(d0, d1);
                    put_t(s.DZT, MLP_H, cb + 2 * j, bf16_bits(p[j]));
                    put_t(s.DZT, MLP_H, cb + 2 * j + 1, bf16_bits(p[j] >> 16));
                }
                if (l == 3) {     // dZ2 is the A operand of dH1 = dZ2 W2
                    const uint32_t (&p0)[8] = *reinterpret_cast<const uint32_t(*)[8]>(p);
                    const uint32_t (&p1)[8] = *reinterpret_cast<const uint32_t(*)[8]>(p + 8);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2, p0);
                    tmem_st_32x32b_x8(tlane + TC_COL_H + cb / 2 + 8, p1);
                }
            }
            finish_epilogue();
        }
        if (s.abort) break;
        first = false;
    }
    if (s.abort) {
        if (tid == 0) {
            (void)mbar_wait_bounded(bar, phase ^ 1u, TC_WAIT_CYCLES);
            if (status) atomicOr(status, SPH_STATUS_TIMEOUT);
        }
    } else if (!first) {
        // this thread's TMEM lane of G_1..G_3: input unit r = tid, every output unit
        const int r = tid;
        #pragma unroll 1
        for (int l = 1; l <= 3; ++l) {
            const uint32_t colG = l == 3 ? GT_COL_G3 : (l == 2 ? GT_COL_G2 : GT_COL_G1);
            const int nin = l == 1 ? MLP_IN : MLP_H;
            const int offW = l == 1 ? OFF_W1 : (l == 2 ? OFF_W2 : OFF_W3), offB = l == 1 ? OFF_B1 : (l == 2 ? OFF_B2 : OFF_B3);
            #pragma unroll
            for (int half = 0; half < 2; ++half) {
                uint32_t v[32];
                tmem_ld_32x32b_x32(tlane + colG + 32 * half, v);
                tmem_ld_wait(v);
                if (r < nin) {
                    #pragma unroll 4
                    for (int j = 0; j < 32; ++j) atomicAdd(&grad[offW + (32 * half + j) * nin + r], __uint_as_float(v[j]));
                } else if (r == nin) {
                    #pragma unroll 4
                    for (int j = 0; j < 32; ++j) atomicAdd(&grad[offB + 32 * half + j], __uint_as_float(v[j]));
                }
            }
        }
        __syncthreads();
        if (tid < MLP_H) atomicAdd(&grad[OFF_W4 + tid], s.gw4[tid]);
        if (tid == 0) {
            atomicAdd(&grad[OFF_B4], s.gb4);
            atomicAdd(loss_out, s.loss);
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after_sync();
        tmem_dealloc(tbase, GT_TMEM_COLS);
    }
}

static int grad_tc_smem_bytes() { return (int)sizeof(MlpGradTcSmem) + 128; }

static int train_smem_bytes() { return (int)sizeof(MlpSmemTrain); }

}  // namespace wsph

using namespace wsph;

extern "C" {

int64_t sph_mlp_param_count(void) { return MLP_NPARAM; }

int sph_mlp_forward(const float* params, int64_t n, const float* feats, const float* scale, float* out, void* stream) {
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_forward: n < 0");
    if (n == 0) return SPH_OK;
    WSPH_CHECK_PTR(params); WSPH_CHECK_PTR(feats); WSPH_CHECK_PTR(out);
    if (reinterpret_cast<uintptr_t>(feats) & 7) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_forward: feats must be 8-byte aligned");
    const int64_t tiles = (n + 16 * MLP_WARPS - 1) / (16 * MLP_WARPS);
    const int grid = (int)(tiles < 148 * 16 ? tiles : 148 * 16);
    count_launch();
    k_mlp_forward<<<grid, MLP_THREADS, 0, WSPH_STREAM(stream)>>>(params, n, feats, scale, out);
    return check_launch("sph_mlp_forward");
}

int sph_mlp_forward_tc(const float* params, int64_t n, const float* feats, const float* scale, float* out, int32_t* status,
                       void* stream) {
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_forward_tc: n < 0");
    if (n == 0) return SPH_OK;
    WSPH_CHECK_PTR(params); WSPH_CHECK_PTR(feats); WSPH_CHECK_PTR(out);
    if (reinterpret_cast<uintptr_t>(feats) & 15) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_forward_tc: feats must be 16-byte aligned");
    const int64_t tiles = (n + TC_M - 1) / TC_M;
    const int64_t cap = 148 * TC_CTAS_PER_SM;
    const int grid = (int)(tiles < cap ? tiles : cap);
    count_launch();
    k_mlp_forward_tc<<<grid, TC_THREADS, 0, WSPH_STREAM(stream)>>>(params, n, feats, scale, out, status);
    return check_launch("sph_mlp_forward_tc");
}

int sph_mlp_grad(const float* params, int64_t n, const float* feats, const float* target, float* grad, double* loss, void* stream) {
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_grad: n < 0");
    WSPH_CHECK_PTR(params); WSPH_CHECK_PTR(grad); WSPH_CHECK_PTR(loss);
    cudaStream_t s = WSPH_STREAM(stream);
    cudaMemsetAsync(grad, 0, sizeof(float) * MLP_NPARAM, s);
    cudaMemsetAsync(loss, 0, sizeof(double), s);
    if (n == 0) return check_launch("sph_mlp_grad");
    WSPH_CHECK_PTR(feats); WSPH_CHECK_PTR(target);
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, train_smem_bytes());
    });
    if (attr_err != cudaSuccess) return set_error(SPH_ERR_CUDA, "sph_mlp_grad: shared memory opt-in: %s", cudaGetErrorString(attr_err));
    const int64_t tiles = (n + 16 * MLP_WARPS - 1) / (16 * MLP_WARPS);
    const int grid = (int)(tiles < 148 * 2 ? tiles : 148 * 2);
    count_launch();
    k_mlp_grad<<<grid, MLP_THREADS, train_smem_bytes(), s>>>(params, n, feats, target, grad, loss);
    return check_launch("sph_mlp_grad");
}

int sph_mlp_grad_tc(const float* params, int64_t n, const float* feats, const float* target, float* grad, double* loss,
                    int32_t* status, void* stream) {
    if (n < 0) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_grad_tc: n < 0");
    WSPH_CHECK_PTR(params); WSPH_CHECK_PTR(grad); WSPH_CHECK_PTR(loss);
    cudaStream_t s = WSPH_STREAM(stream);
    cudaMemsetAsync(grad, 0, sizeof(float) * MLP_NPARAM, s);
    cudaMemsetAsync(loss, 0, sizeof(double), s);
    if (n == 0) return check_launch("sph_mlp_grad_tc");
    WSPH_CHECK_PTR(feats); WSPH_CHECK_PTR(target);
    if (reinterpret_cast<uintptr_t>(feats) & 15) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_grad_tc: feats must be 16-byte aligned");
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, grad_tc_smem_bytes());
    });
    if (attr_err != cudaSuccess)
        return set_error(SPH_ERR_CUDA, "sph_mlp_grad_tc: shared memory opt-in: %s", cudaGetErrorString(attr_err));
    const int64_t tiles = (n + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < 148 ? tiles : 148);
    count_launch();
    k_mlp_grad_tc<<<grid, TC_THREADS, grad_tc_smem_bytes(), s>>>(params, n, feats, target, grad, loss, status);
    return check_launch("sph_mlp_grad_tc");
}

int sph_mlp_adam(float* params, const float* grad, float* m1, float* m2, int64_t count, float lr, float beta1, float beta2, float eps,
                 int64_t step, void* stream) {
    if (count < 0 || step < 1) return set_error(SPH_ERR_BAD_ARG, "sph_mlp_adam: count < 0 or step < 1");
    if (count == 0) return SPH_OK;
    WSPH_CHECK_PTR(params); WSPH_CHECK_PTR(grad); WSPH_CHECK_PTR(m1); WSPH_CHECK_PTR(m2);
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    count_launch();
    k_mlp_adam<<<grid_for(count, 256), 256, 0, WSPH_STREAM(stream)>>>(params, grad, m1, m2, count, lr, beta1, beta2, eps, c1, c2);
    return check_launch("sph_mlp_adam");
}

}  // extern "C"
