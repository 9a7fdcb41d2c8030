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
    uint32_t *count;  // arrivals: count[0] counts the even barriers of a launch, count[16] the odd ones
    uint32_t *gen;    // barriers completed
    uint32_t epoch;   // this CTA's view of gen (thread 0)
    uint32_t parity;  // barriers this CTA has passed in this launch, mod 2
};

// Add with acquire-release semantics at GPU scope: publishes this CTA's writes
// (ordered before it by the preceding __syncthreads) and, for the last
// arriver, acquires every earlier arriver's.
__device__ __forceinline__ uint32_t atom_add_acq_rel_gpu(uint32_t *p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void red_add_release_gpu(uint32_t *p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier. The last CTA to arrive runs `last` (all its threads)
// before it releases the others. False when this CTA's wait timed out.
// Arrivals alternate between two counters: the last arriver zeroes its
// barrier's counter with a plain store before the releasing add, and that
// counter is next used two barriers on, by CTAs that have acquired a later
// release. So no reset has to complete before the release, and the release
// and acquire orderings replace full fences.
template <typename F>
__device__ __forceinline__ bool grid_sync(GridSync &g, int *flag, F last) {
    fence_proxy_async_global();
    __syncthreads();
    uint32_t *const cnt = g.count + 16u * g.parity;
    if (threadIdx.x == 0) {
        flag[0] = (atom_add_acq_rel_gpu(cnt, 1u) == gridDim.x - 1) ? 1 : 0;
        flag[1] = 1;
    }
    __syncthreads();
    if (flag[0]) {
        last();
        __syncthreads();
        if (threadIdx.x == 0) {
            *reinterpret_cast<volatile uint32_t *>(cnt) = 0u;
            red_add_release_gpu(g.gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        const uint64_t t0 = global_ns();
        while (ld_acquire_u32(g.gen) == g.epoch) {
            if (global_ns() - t0 > kWaitLimitNs) {
                flag[1] = 0;
                break;
            }
        }
    }
    g.epoch += 1u;
    g.parity ^= 1u;
    __syncthreads();
    const bool ok = flag[1] != 0;
    fence_proxy_async_global();
    return ok;
}

// Grid-wide barrier on one arrival counter, zeroed before the launch: barrier k
// of the launch completes when the counter reaches (k + 1) x CTAs, and every
// CTA waits on the counter itself, so the others go on as soon as the last
// arrival lands (no separate release word to write and see). The last arriver,
// which learns it from its add, then runs `after` (all its threads): work that
// nobody reads before the next barrier, or that the readers wait for by other
// means. Acquire-release adds on one location form one release sequence, so a
// CTA that reads the full count has acquired every arrival's writes.
struct CountSync {
    uint32_t *count;  // arrivals in this launch
    uint32_t target;  // arrivals that complete the next barrier
};

template <typename F>
__device__ __forceinline__ bool count_sync(CountSync &g, int *flag, F after) {
    fence_proxy_async_global();
    __syncthreads();
    g.target += gridDim.x;
    if (threadIdx.x == 0) {
        flag[1] = 1;
        const uint32_t old = atom_add_acq_rel_gpu(g.count, 1u);
        flag[0] = old + 1u == g.target ? 1 : 0;
        if (old + 1u != g.target) {
            const uint64_t t0 = global_ns();
            while (ld_acquire_u32(g.count) < g.target) {
                if (global_ns() - t0 > kWaitLimitNs) {
                    flag[1] = 0;
                    break;
                }
            }
        }
    }
    __syncthreads();
    const bool last = flag[0] != 0, ok = flag[1] != 0;
    if (last) {
        after();
        __syncthreads();
    }
    fence_proxy_async_global();
    return ok;
}

}  // namespace swe
