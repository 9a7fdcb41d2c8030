// Whole steps in one persistent, cooperative launch.
//
// The same phases as the per-kernel step (swe_step: predictor, corrector,
// sources, dilation + step control) run back to back inside one kernel,
// separated by grid-wide barriers instead of kernel boundaries, for
// `n_steps` steps. A step with a few active tiles is a chain of short
// dependent phases; between kernels each link pays a launch gap and a grid
// ramp, between barriers about a microsecond.
//
// Every CTA is resident (cooperative launch), every barrier wait is bounded
// (2 s, then the CTA records error 2 in the control block and stops), and the
// staged-data waits of the tile passes are bounded as in the stage kernels.
// The arithmetic is the stage kernels' own, so results are bit-identical.
#include <cuda_runtime.h>

#include <cstdint>

#include "swe_grid.cuh"
#include "swe_sources.cuh"
#include "swe_tiled.cuh"

namespace swe {

// Dilation of the wet marks over each block's two-ring and compaction into the
// next step's block list and tile work items (the dilate_compact kernel's
// work), for active_set = 0: every block of a running instance is listed.
// One warp per block.
__device__ __forceinline__ void dilate_all_pass(const swe_mesh_t &m, const swe_state_t &s, const Spread &sp) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); b < m.n_blocks; b += warps) {
        if (s.dt_buf[kDtWords * m.block_inst[b]] == 0u) continue;  // a no-op step keeps its flags
        if (lane == 0) {
            s.blk[kBlkWords * b + kBlkActive] = 1u;
            list_block(m, s, sp, b);
        }
    }
}

// Active flags of the step whose lists were just built by spreading: every block
// of the current list is active; a block of the previous list that was not listed
// again is not, unless its instance did not run the previous step (a no-op step
// keeps its flags, as the dilation does). dt_buf[4 i + 2] holds each instance's
// dt of the previous step. Spread over the CTAs from the last one down, which
// are the ones without tiles when the lists are short.
__device__ __forceinline__ void flag_pass(const swe_mesh_t &m, const swe_state_t &s, const uint32_t *cur, uint32_t n_cur,
                                          const uint32_t *prev, uint32_t n_prev, uint32_t listed_epoch) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = (gridDim.x - 1u - blockIdx.x) * blockDim.x + threadIdx.x; t < n_cur + n_prev; t += stride) {
        if (t < n_cur) {
            s.blk[kBlkWords * cur[t] + kBlkActive] = 1u;
        } else {
            const uint32_t b = prev[t - n_cur];
            if (s.marks[2u * b] != listed_epoch && s.dt_buf[kDtWords * m.block_inst[b] + 2u] != 0u)
                s.blk[kBlkWords * b + kBlkActive] = 0u;
        }
    }
}

template <bool COMP, bool CLAMP, bool OPEN>
__global__ void __launch_bounds__(kPersistThreads, 1024 / kPersistThreads)
    persistent_steps_kernel(swe_mesh_t m, swe_state_t s, swe_sources_t src, Phys p, float cfl, int all_active,
                            uint32_t n_steps) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ TiledShared<kPersistThreads> sh;
    __shared__ int flag[2];
    __shared__ uint32_t epoch0;
    GridSync g{s.sync, s.sync + 32, 0u, 0u};
    if (threadIdx.x == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(smem), 1u);
        mbar_init(reinterpret_cast<uint64_t *>(smem) + 1, 1u);
        fence_barrier_init();
        g.epoch = ld_acquire_u32(g.gen);
        epoch0 = *reinterpret_cast<volatile uint32_t *>(s.sched + kSchedEpoch);  // before any CTA's first barrier
    }
    __syncthreads();
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    // the two halves of the lists: the step's current list in half (step & 1)
    uint32_t *const list0 = s.active_list, *const list1 = s.active_list + m.n_blocks;
    uint4 *const items0 = reinterpret_cast<uint4 *>(s.items), *const items1 = items0 + 4u * m.n_blocks;
    auto lists = [&](uint32_t h) { return h ? list1 : list0; };
    auto item_sets = [&](uint32_t h) { return h ? items1 : items0; };
    auto nothing = [] {};
    uint32_t k = 0;
    uint64_t computed = 0;
    bool ok = true;
    uint32_t step = 0;
    for (; step < n_steps; ++step) {
        const uint32_t cur = step & 1u, nxt = cur ^ 1u;
        const uint32_t epoch = epoch0 + step + 1u;
        swe_state_t sj = s;
        sj.active_list = lists(cur);
        sj.items = reinterpret_cast<uint32_t *>(item_sets(cur));
        const Spread sp{lists(nxt), item_sets(nxt), epoch};
        const Spread none{};
        if (!(ok = tiled_pass<0, COMP, CLAMP, kPersistThreads, true, OPEN>(m, sj, p, cfl, smem, sh, k, computed))) break;
        if (step > 0u && !all_active) {
            const volatile uint32_t *sched = s.sched;
            flag_pass(m, s, lists(cur), sched[kSchedActive], lists(nxt), sched[kSchedPrevActive], epoch - 1u);
        }
        if (!(ok = grid_sync(g, flag, nothing))) break;
        if (!(ok = tiled_pass<1, COMP, CLAMP, kPersistThreads, true, OPEN>(m, sj, p, cfl, smem, sh, k, computed,
                                                                      all_active ? none : sp)))
            break;
        if (src.count) {
            if (!(ok = grid_sync(g, flag, nothing))) break;
            source_apply(m, sj, src, p.dry_tol, COMP ? 1 : 0, first, stride);
            if (!(ok = grid_sync(g, flag, nothing))) break;
            source_bound(m, sj, src, p, cfl, first, stride);
            if (!all_active) {
                for (uint32_t q = first; q < src.count; q += stride) {
                    const uint32_t b = src.cells[q] >> 8;
                    if (s.blk[kBlkWords * b + kBlkWet] != 0u && s.dt_buf[kDtWords * m.block_inst[b]] != 0u)
                        spread_thread(m, s, sp, b);
                }
            }
        }
        if (all_active) {
            if (!(ok = grid_sync(g, flag, nothing))) break;
            dilate_all_pass(m, s, sp);
        }
        auto control = [&] {
            // every instance's step control (keeping the dt of the step it ends), then the new lists become current
            for (uint32_t i = threadIdx.x; i < m.n_inst; i += blockDim.x) {
                s.dt_buf[kDtWords * i + 2u] = s.dt_buf[kDtWords * i];
                step_control(s.ctrl + i, s.dt_buf + kDtWords * i, 1);
            }
            if (threadIdx.x == blockDim.x - 1u) {  // beside instance 0's control, not after it
                volatile uint32_t *sched = s.sched;
                sched[kSchedPrevActive] = sched[kSchedActive];
                sched[kSchedActive] = sched[kSchedNext];
                sched[kSchedItems] = sched[kSchedNextItems];
                sched[kSchedNext] = 0u;
                sched[kSchedNextItems] = 0u;
                sched[kSchedEpoch] = epoch;
            }
        };
        if (!(ok = grid_sync(g, flag, control))) break;
    }
    if (ok && step > 0u) {
        // Hand the lists over in the first halves with their flags, as the other kernels expect them.
        const uint32_t cur = step & 1u;
        const volatile uint32_t *sched = s.sched;
        const uint32_t n_cur = sched[kSchedActive], n_items = sched[kSchedItems];
        if (!all_active) flag_pass(m, s, lists(cur), n_cur, lists(cur ^ 1u), sched[kSchedPrevActive], epoch0 + step);
        if (cur == 1u) {
            ok = grid_sync(g, flag, nothing);
            if (ok) {
                for (uint32_t i = first; i < n_cur; i += stride) list0[i] = list1[i];
                for (uint32_t i = first; i < n_items; i += stride) items0[i] = items1[i];
            }
        }
    }
    if (threadIdx.x == 0) {
        if (!ok) atomicOr(&s.ctrl->error, 2u);
        if (computed) atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed), computed);
    }
}

template <bool COMP, bool CLAMP, bool OPEN>
int launch_persistent(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, const swe_sources_t *src,
                      uint32_t n_steps, cudaStream_t st) {
    auto kern = persistent_steps_kernel<COMP, CLAMP, OPEN>;
    const size_t bytes = tiled_smem_bytes(m->max_sub_edges, m->max_sub_slots, true);
    int rc = set_smem(kern, bytes);
    if (rc) return rc;
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPersistThreads, bytes) != cudaSuccess)
        return SWE_ERR_CUDA;
    if (per_sm < 1) return SWE_ERR_TOO_LARGE;
    const uint32_t fit = static_cast<uint32_t>(per_sm) * static_cast<uint32_t>(sms);
    const uint32_t grid = (p->grid == 0u || p->grid > fit) ? fit : p->grid;
    Phys ph{p->g, p->dry_tol};
    float cfl = p->cfl;
    int all_active = p->active_set ? 0 : 1;
    swe_mesh_t mm = *m;
    swe_state_t ss = *s;
    swe_sources_t sc = *src;
    void *args[] = {&mm, &ss, &sc, &ph, &cfl, &all_active, &n_steps};
    if (cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(grid), dim3(kPersistThreads), args, bytes,
                                    st) != cudaSuccess)
        return SWE_ERR_CUDA;
    return SWE_OK;
}

template <bool OPEN>
int dispatch_persistent(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, const swe_sources_t *src,
                        uint32_t n_steps, cudaStream_t st) {
    if (p->compensated)
        return p->track_clamp ? launch_persistent<true, true, OPEN>(m, s, p, src, n_steps, st)
                              : launch_persistent<true, false, OPEN>(m, s, p, src, n_steps, st);
    return p->track_clamp ? launch_persistent<false, true, OPEN>(m, s, p, src, n_steps, st)
                          : launch_persistent<false, false, OPEN>(m, s, p, src, n_steps, st);
}

int configure_persistent(const swe_mesh_t *mesh, int *blocks_per_sm) {
    const size_t bytes = tiled_smem_bytes(mesh->max_sub_edges, mesh->max_sub_slots, true);
    int rc = set_smem(persistent_steps_kernel<true, false, false>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<true, true, false>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<false, false, false>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<false, true, false>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<true, false, true>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<true, true, true>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<false, false, true>, bytes);
    if (!rc) rc = set_smem(persistent_steps_kernel<false, true, true>, bytes);
    if (rc) return rc;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, persistent_steps_kernel<true, false, false>,
                                                         kPersistThreads, bytes) == cudaSuccess
               ? SWE_OK
               : SWE_ERR_CUDA;
}

}  // namespace swe

using namespace swe;

extern "C" int swe_steps(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                         const swe_sources_t *sources, uint32_t n_steps, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !open_ok(mesh, state) || !params || !sources || params->kernel > 2u)
        return SWE_ERR_ARGUMENT;
    if (n_steps == 0u) return SWE_OK;
    if (params->kernel < 2u) {
        for (uint32_t k = 0; k < n_steps; ++k) {
            const int rc = swe_step(mesh, state, params, sources, stream);
            if (rc) return rc;
        }
        return SWE_OK;
    }
    if (!state->sync || !state->marks) return SWE_ERR_ARGUMENT;
    if (mesh->max_sub_edges > 2047u || mesh->max_sub_slots > 2047u || mesh->n_inst > 1023u) return SWE_ERR_TOO_LARGE;
    if (sources->count && (!sources->cells || !sources->rate)) return SWE_ERR_ARGUMENT;
    return mesh->n_open ? dispatch_persistent<true>(mesh, state, params, sources, n_steps, stream)
                        : dispatch_persistent<false>(mesh, state, params, sources, n_steps, stream);
}
