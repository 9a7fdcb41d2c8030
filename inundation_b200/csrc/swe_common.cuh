// Shared device and host helpers of the shallow-water kernels.
//
// Meshes: cells in Hilbert order, grouped in 256-cell blocks (the active-set
// unit of the reference, inundation/tuning.py:53-55) and 64-cell compute
// tiles (four per block). A batch concatenates several meshes (instances),
// each starting on a block boundary; block_inst names a block's instance,
// block_cells its real cells. Every instance has its own clock (control
// block) and its own dt words: dt_buf[4 i] is the dt of its current step
// (0 = no-op), dt_buf[4 i + 1] the CFL bound reduced for its next step,
// dt_buf[4 i + 2..3] the (dt, step epoch) pair the persistent kernel publishes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/inundation_b200.h"
#include "swe_math.cuh"

namespace swe {

constexpr int kBlockCells = 256;
constexpr int kThreads = 256;
constexpr int kTileCells = 64;
constexpr int kTileThreads = 128;     // threads of a tile CTA of the tiled stage kernel
constexpr int kPersistThreads = 256;  // threads of a tile CTA of the persistent kernel: one edge record each
constexpr uint32_t kBlkWords = 3, kBlkWet = 0, kBlkActive = 1, kBlkForced = 2;
constexpr uint32_t kNoBound = 0xFFFFFFFFu;
constexpr uint32_t kDtWords = 4;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // bound of every device wait: 2 s

// sched words
constexpr int kSchedActive = 0;     // blocks in active_list for the current step
constexpr int kSchedNext = 1;       // blocks appended by the dilation
constexpr int kSchedDone = 2;       // CTAs of the dilation that finished
constexpr int kSchedItems = 3;      // tile work items of the current step
constexpr int kSchedNextItems = 4;  // tile work items appended by the dilation
constexpr int kSchedComputed = 6;   // [6,7]: uint64 cells computed over real steps
constexpr int kSchedEpoch = 10;     // steps of the persistent kernel since the run's prologue
constexpr int kSchedStartTaken = 11;  // tiles of the start list taken (persistent kernel)
constexpr int kSchedQProd = 12;       // [12, 13]: tiles queued for steps of each parity (persistent kernel)
constexpr int kSchedQCons = 14;       // [14, 15]: tiles taken from those queues (persistent kernel)

// A tile work item: x = tile | (real cells << 25), y = first edge record,
// z = first local-CSR entry, w = edge count | (padded slot count << 11) | (instance << 22).
__device__ __forceinline__ uint4 make_item(uint32_t tile, uint32_t cells, uint32_t e0, uint32_t l0, uint32_t ne,
                                           uint32_t lp, uint32_t inst) {
    return make_uint4(tile | (cells << 25), e0, l0, ne | (lp << 11) | (inst << 22));
}

__device__ __forceinline__ bool block_active(const uint32_t *blk, uint32_t b) {
    return blk[kBlkWords * b + kBlkActive] != 0u;
}

// The stage's input state of cell c: the predictor in the corrector, except
// in an inactive block, whose predictor is stale (resident.py:209-226). In
// the corrector both candidates are loaded with the flag, in one round trip.
template <int STAGE>
__device__ __forceinline__ void load_state(const swe_state_t &s, int c, float &h, float &hu, float &hv) {
    if (STAGE == 0) {
        h = s.h[c];
        hu = s.hu[c];
        hv = s.hv[c];
    } else {
        const bool pred = block_active(s.blk, static_cast<uint32_t>(c) >> 8);
        const float a0 = s.h1[c], a1 = s.hu1[c], a2 = s.hv1[c];
        const float b0 = s.h[c], b1 = s.hu[c], b2 = s.hv[c];
        h = pred ? a0 : b0;
        hu = pred ? a1 : b1;
        hv = pred ? a2 : b2;
    }
}

// A corrector tile's two results after one CTA barrier: whether any thread's cell is wet and the
// minimum of the threads' CFL bounds, both valid in warp 0 (scratch: 2 words per warp). Every thread
// has finished its update when the barrier passes; the scratch is next written after a later barrier.
__device__ __forceinline__ void tile_outcome(bool wet, uint32_t bound, uint32_t *scratch, bool &any_wet,
                                             uint32_t &bmin) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
    const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, bound);
    const bool w = __any_sync(0xFFFFFFFFu, wet);
    if (lane == 0) {
        scratch[warp] = m;
        scratch[nw + warp] = w ? 1u : 0u;
    }
    __syncthreads();
    any_wet = false;
    bmin = kNoBound;
    if (warp == 0) {
        bmin = __reduce_min_sync(0xFFFFFFFFu, lane < nw ? scratch[lane] : kNoBound);
        any_wet = __any_sync(0xFFFFFFFFu, lane < nw && scratch[nw + lane] != 0u);
    }
}

__device__ __forceinline__ uint32_t block_min_any(uint32_t v, uint32_t *scratch) {
    v = __reduce_min_sync(0xFFFFFFFFu, v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < nw) ? scratch[lane] : kNoBound;
        w = __reduce_min_sync(0xFFFFFFFFu, w);
        if (lane == 0) scratch[0] = w;
    }
    __syncthreads();
    const uint32_t r = scratch[0];
    __syncthreads();
    return r;
}

// -- bulk copies (TMA, 1-D, into this CTA's own shared memory) on an mbarrier --------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0u;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// True once the barrier's phase of this parity completed; false after the deadline.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity)) {
        if (global_ns() - t0 > kWaitLimitNs) return false;
    }
    return true;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// -- integer-tick step control (resident.py:813-885) ---------------------------------------------
__device__ __forceinline__ uint32_t step_control(swe_ctrl_t *c, uint32_t *dt_buf, int mode) {
    // Every input is read before anything is written, so all the loads are in flight at
    // once (one round trip: this runs on the critical path of the persistent kernel).
    const uint64_t now0 = c->now_ticks, stop = c->stop_ticks, steps0 = c->steps;
    const uint32_t done = c->dt_ticks, dt_max = c->dt_max_ticks, dry_dt = c->dry_dt_ticks;
    const float last0 = c->last_raw, safety = c->cfl_safety;
    const uint32_t bound0 = dt_buf[0], bound1 = dt_buf[1];
    uint64_t now = now0, steps = steps0;
    float raw = last0;  // a no-op step computed no bound; RETARGET replans from the last one
    if (mode == 0) {
        raw = __uint_as_float(bound0);
    } else if (mode == 1) {
        now += static_cast<uint64_t>(done);
        if (done > 0u) {
            steps += 1u;
            raw = __uint_as_float(bound1);
        }
    }
    const uint64_t remaining = (stop > now) ? stop - now : 0ull;
    uint32_t ticks;
    if (remaining == 0ull || raw < 1e-10f || raw != raw) {
        ticks = 0u;  // window done, or a degenerate bound: the host sees no progress
    } else if (raw >= 1e10f) {
        ticks = dry_dt;  // no wet edge anywhere
    } else {
        const float cap = static_cast<float>(dt_max) / kTicksPerSecond;
        ticks = static_cast<uint32_t>(gmin(raw * safety, cap) * kTicksPerSecond);
    }
    if (dt_max < ticks) ticks = dt_max;
    if (static_cast<uint64_t>(ticks) > remaining) ticks = static_cast<uint32_t>(remaining);
    c->now_ticks = now;
    c->steps = steps;
    c->last_raw = raw;
    c->dt_ticks = ticks;
    const uint32_t dt = __float_as_uint(static_cast<float>(ticks) / kTicksPerSecond);
    dt_buf[0] = dt;
    dt_buf[1] = __float_as_uint(kDtSentinel);
    return dt;
}

// The persistent kernel's step control publishes an instance's next dt as the
// pair (dt, epoch of that step) in dt words 2..3 after it has released the grid.
// The dt of the step of `epoch` from the pair's value v, read again until the
// pair carries that epoch (bounded: 0 and error bit 4 when it does not come).
__device__ __forceinline__ uint32_t published_dt(const swe_state_t &s, const uint64_t *pair, uint32_t epoch,
                                                 uint64_t v) {
    if (static_cast<uint32_t>(v >> 32) == epoch) return static_cast<uint32_t>(v);
    const uint64_t t0 = global_ns();
    for (;;) {
        v = ld_relaxed_u64(pair);
        if (static_cast<uint32_t>(v >> 32) == epoch) return static_cast<uint32_t>(v);
        if (global_ns() - t0 > kWaitLimitNs) {
            atomicOr(&s.ctrl->error, 4u);
            return 0u;
        }
    }
}
__device__ __forceinline__ const uint64_t *dt_pair(const swe_state_t &s, uint32_t inst) {
    return reinterpret_cast<const uint64_t *>(s.dt_buf + kDtWords * inst + 2u);
}

// The state beyond boundary edge cR < 0 from the cell inside it: a wall's
// mirror (cR == -1), or open edge -2 - cR's ghost under its condition, which
// comes back in kind/value (resident.py:127-145). kind/value stay wall/0 for a
// wall, so open_forced(kind, value) is the edge's forced liveness either way.
__device__ __forceinline__ void boundary_state(const swe_mesh_t &m, const Phys &p, int cR, float hL, float huL,
                                               float hvL, float nx, float ny, float &hR, float &huR, float &hvR,
                                               uint32_t &kind, float &value) {
    if (cR == -1) {
        hR = hL;
        wall_mirror(huL, hvL, nx, ny, huR, hvR);
        return;
    }
    const uint32_t k = static_cast<uint32_t>(-2 - cR);
    kind = m.open_cond[2u * k];
    value = __uint_as_float(m.open_cond[2u * k + 1u]);
    ghost_state(p, kind, value, hL, huL, hvL, nx, ny, hR, huR, hvR);
}

// Adds one stage's volume through open edge k to its out (v >= 0) or in
// (v < 0) pair: two-sum of |v| into the high word, the old low word folded
// into the error (resident.py:617-660, per edge). Only the thread computing
// the edge touches its words within a stage.
__device__ __forceinline__ void tally_open(float *vol, uint32_t k, float v) {
    float *t = vol + 4u * k + (v < 0.0f ? 2u : 0u);
    float sm, err, hi, lo;
    two_sum(t[0], fabsf(v), sm, err);
    err += t[1];
    two_sum(sm, err, hi, lo);
    t[0] = hi;
    t[1] = lo;
}

// -- host helpers --------------------------------------------------------------------------------
inline int check_launch() { return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ERR_CUDA; }
constexpr size_t kMaxSmem = 227 * 1024;  // dynamic shared memory a CTA may opt in to

template <typename K>
inline int set_smem(K kernel, size_t bytes) {
    if (bytes > kMaxSmem) return SWE_ERR_TOO_LARGE;
    if (bytes > 48 * 1024 &&
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)) != cudaSuccess)
        return SWE_ERR_CUDA;
    return SWE_OK;
}

inline bool mesh_ok(const swe_mesh_t *m) {
    return m && m->n_cells && m->n_blocks && m->n_inst && m->tile_cl && m->tile_cr && m->tile_nx && m->tile_ny &&
           m->tile_len && m->tile_dzl && m->tile_dzr && m->tile_ptr && m->tile_count && m->cptr && m->lcsr &&
           m->area && m->n_mann && m->ring_ptr && m->ring_idx && m->sub_cl && m->sub_cr && m->sub_nx && m->sub_ny &&
           m->sub_len && m->sub_dzl && m->sub_dzr && m->sub_ptr && m->sub_count && m->sub_lcsr && m->sub_lcsr_ptr &&
           m->block_inst && m->block_cells && (m->n_open == 0u || m->open_cond);
}

// The open-edge tally words must exist when the mesh has open edges.
inline bool open_ok(const swe_mesh_t *m, const swe_state_t *s) { return m->n_open == 0u || s->open_vol; }

inline bool state_ok(const swe_state_t *s) {
    return s && s->h && s->hu && s->hv && s->h_lo && s->h1 && s->hu1 && s->hv1 && s->h1_lo && s->clamp_mass &&
           s->blk && s->active_list && s->items && s->sched && s->dt_buf && s->ctrl;
}

}  // namespace swe
