// Grid-wide barrier of the persistent kernels (cooperative launches: every CTA
// resident). Bounded: a wait that runs past kWaitLimitNs reports failure.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "swe_common.cuh"

namespace swe {

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Generic-proxy writes of this phase before bulk-copy (async-proxy) reads of the next.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

struct GridSync {
    uint32_t *count;  // arrivals of the current barrier
    uint32_t *gen;    // barriers completed
    uint32_t epoch;   // this CTA's view of gen (thread 0)
};

// Grid-wide barrier. The last CTA to arrive runs `last` (all its threads)
// before it releases the others. False when this CTA's wait timed out.
template <typename F>
__device__ __forceinline__ bool grid_sync(GridSync &g, int *flag, F last) {
    fence_proxy_async_global();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        flag[0] = (atomicAdd(g.count, 1u) == gridDim.x - 1) ? 1 : 0;
        flag[1] = 1;
    }
    __syncthreads();
    if (flag[0]) {
        __threadfence();
        last();
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicExch(g.count, 0u);
            __threadfence();
            atomicAdd(g.gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        const uint64_t t0 = global_ns();
        while (ld_acquire_u32(g.gen) == g.epoch) {
            if (global_ns() - t0 > kWaitLimitNs) {
                flag[1] = 0;
                break;
            }
        }
        __threadfence();
    }
    g.epoch += 1u;
    __syncthreads();
    const bool ok = flag[1] != 0;
    fence_proxy_async_global();
    return ok;
}

}  // namespace swe
