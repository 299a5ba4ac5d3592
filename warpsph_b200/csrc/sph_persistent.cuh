// Bounded grid-wide barrier for cooperative persistent kernels (the DFSPH Jacobi solves
// and the batched delta-SPH step).  The launch must be cooperative (every block
// co-resident).  A wait gives up after limit_ns nanoseconds of the global timer (2 s by
// default; the Jacobi solves take the limit from their launch arguments) or 2^26 polls,
// sets SPH_STATUS_TIMEOUT in the control block and makes every block return, so a
// failure ends the kernel instead of hanging the GPU.
#pragma once
#include <cuda_runtime.h>
#include "sph_common.cuh"

namespace wsph {

struct BarrierCtl {
    unsigned int count;        // arrivals in the current generation
    unsigned int gen;          // barrier generation
    int status;                // SPH_STATUS_* bits
    int pad;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned long long kBarrierLimitNs = 2000000000ull;

// Returns false when any block gave up (SPH_STATUS_TIMEOUT); the caller then returns.
static __device__ __noinline__ bool grid_barrier(BarrierCtl* c, unsigned long long limit_ns = kBarrierLimitNs) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = &c->gen;
        volatile int* vstat = &c->status;
        const unsigned int g = *vgen;
        int good = 1;
        __threadfence();
        const unsigned int arrived = atomicAdd(&c->count, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&c->count, 0u);
            __threadfence();
            atomicAdd(&c->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (*vgen == g) {
                if (*vstat & SPH_STATUS_TIMEOUT) { good = 0; break; }
                if (++spins > (1u << 26) || global_ns() - t0 > limit_ns) {
                    atomicOr(&c->status, SPH_STATUS_TIMEOUT);
                    good = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace wsph
