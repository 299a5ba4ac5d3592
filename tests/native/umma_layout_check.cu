// Host-side check of the tcgen05 operand conventions in sph_tcgen05.cuh against CuTe's
// own construction (cute/atom/mma_traits_sm100.hpp): the K-major no-swizzle core-matrix
// layout, the shared-memory descriptor strides and the kind::f16 instruction descriptor.
// Prints "ok" and exits 0 when everything agrees.
#include <cstdio>
#include <cute/tensor.hpp>
#include <cute/atom/mma_traits_sm100.hpp>
#include "sph_tcgen05.cuh"

template <int R, int K>
static int check_operand() {
    using namespace cute;
    auto L = tile_to_shape(UMMA::Layout_K_INTER_Atom<bfloat16_t>{}, make_shape(Int<R>{}, Int<K>{}));
    int bad = 0;
    for (int r = 0; r < R; ++r)
        for (int k = 0; k < K; ++k)
            if (wsph::umma_k_index(r, k, R) != static_cast<int>(L(r, k))) ++bad;
    // one k-step (K = 16) of the operand, as the kernels describe it
    auto Lk = tile_to_shape(UMMA::Layout_K_INTER_Atom<bfloat16_t>{}, make_shape(Int<R>{}, Int<16>{}));
    UMMA::SmemDescriptor d = UMMA::make_umma_desc<UMMA::Major::K>(make_tensor(make_smem_ptr((bfloat16_t*)nullptr), Lk));
    const uint64_t mine = wsph::umma_desc_kmajor(0u, R * 16, 128);
    const uint64_t theirs = static_cast<uint64_t>(d) & ~0x3FFFull;   // start address is not known on the host
    if (mine != theirs) {
        std::printf("R=%d: descriptor %016llx, CuTe %016llx\n", R, (unsigned long long)mine, (unsigned long long)theirs);
        ++bad;
    }
    if (bad) std::printf("R=%d K=%d: %d mismatches\n", R, K, bad);
    return bad;
}

int main() {
    using namespace cute;
    int bad = check_operand<128, 16>() + check_operand<128, 80>() + check_operand<64, 16>() + check_operand<64, 80>();
    const uint32_t idesc = static_cast<uint32_t>(UMMA::make_instr_desc<bfloat16_t, bfloat16_t, float, 128, 64, UMMA::Major::K, UMMA::Major::K>());
    if (idesc != wsph::umma_idesc_bf16_f32<128, 64>()) {
        std::printf("instruction descriptor %08x, CuTe %08x\n", wsph::umma_idesc_bf16_f32<128, 64>(), idesc);
        ++bad;
    }
    std::printf(bad ? "mismatch\n" : "ok\n");
    return bad ? 1 : 0;
}
