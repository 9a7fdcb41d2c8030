// Step control around the stage kernels: active-set dilation and compaction
// into work lists, the integer-tick clock of every instance, the start-of-run
// marks and CFL bound, and the sparse sources (with device-evaluated inflow
// hydrographs).
//
// Reference: inundation/vulkan/shaders/resident.py (block_mark, block_dilate,
// step_control, source_resident, cfl_edge_gather + cfl_gather) as dispatched
// by inundation/vulkan/gpu_resident_batch.py.
#include <cuda_runtime.h>

#include <cstdint>

#include "swe_sources.cuh"

namespace swe {

// ---------------------------------------------------------------------------
// Dilation of the wet marks over each block's two-ring, compaction of the
// active blocks and their 64-cell tiles, then (last CTA) step control of
// every instance (resident.py:778-805, 813-885).
// One warp per block reads the block's two-ring in parallel; each CTA of
// kDilateWarps warps appends its active blocks and tiles with one atomic each.
// An instance on a no-op step (dt 0) keeps its flags and is left out of the
// lists, unless force is set: its clock only moves again after a RETARGET,
// which the host issues through a forced dilation.
// ---------------------------------------------------------------------------
constexpr int kDilateWarps = 32;

__global__ void __launch_bounds__(kDilateWarps * 32)
    dilate_compact_kernel(swe_mesh_t m, swe_state_t s, int all_active, int force, int control_mode) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * kDilateWarps + warp;
    __shared__ uint32_t flag[kDilateWarps];
    __shared__ bool last;
    uint32_t v = 0u;
    if (b < m.n_blocks) {
        const uint32_t inst = m.block_inst[b];
        const bool run = force || s.dt_buf[kDtWords * inst] != 0u;
        if (run) {
            if (all_active) {
                v = 1u;
            } else {
                const uint32_t k0 = m.ring_ptr[b], k1 = m.ring_ptr[b + 1];
                if (lane == 0) v = s.blk[kBlkWords * b + kBlkWet] | s.blk[kBlkWords * b + kBlkForced];
                for (uint32_t k = k0 + lane; k < k1; k += 32) {
                    const uint32_t nb = m.ring_idx[k];
                    v |= s.blk[kBlkWords * nb + kBlkWet] | s.blk[kBlkWords * nb + kBlkForced];
                }
                v = __any_sync(0xFFFFFFFFu, v != 0u) ? 1u : 0u;
            }
            if (lane == 0) s.blk[kBlkWords * b + kBlkActive] = v;
        }
    }
    if (lane == 0) flag[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const uint32_t blk = blockIdx.x * kDilateWarps + lane;
        const bool on = flag[lane] != 0u;
        const uint32_t cells = on ? m.block_cells[blk] : 0u;
        const uint32_t n_items = (cells + kTileCells - 1) / kTileCells;
        const unsigned ballot = __ballot_sync(0xFFFFFFFFu, on);
        uint32_t items_before = n_items;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, items_before, d);
            if (lane >= d) items_before += up;
        }
        const uint32_t items_total = __shfl_sync(0xFFFFFFFFu, items_before, 31);
        items_before -= n_items;
        uint32_t pos = 0, ipos = 0;
        if (lane == 0 && ballot) {
            pos = atomicAdd(&s.sched[kSchedNext], static_cast<uint32_t>(__popc(ballot)));
            ipos = atomicAdd(&s.sched[kSchedNextItems], items_total);
        }
        pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
        ipos = __shfl_sync(0xFFFFFFFFu, ipos, 0) + items_before;
        if (on) {
            const uint32_t slot = pos + __popc(ballot & ((1u << lane) - 1u));
            if (slot < m.n_blocks) s.active_list[slot] = blk;
            const uint32_t inst = m.block_inst[blk];
            uint4 *out = reinterpret_cast<uint4 *>(s.items);
            for (uint32_t q = 0; q < n_items && ipos + q < 4u * m.n_blocks; ++q) {
                const uint32_t t = 4u * blk + q;
                const uint32_t l0 = m.sub_lcsr_ptr[t];
                out[ipos + q] = make_item(t, min(static_cast<uint32_t>(kTileCells), cells - q * kTileCells),
                                          m.sub_ptr[t], l0, m.sub_count[t], m.sub_lcsr_ptr[t + 1] - l0, inst);
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&s.sched[kSchedDone], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (control_mode >= 0) {
        for (uint32_t i = threadIdx.x; i < m.n_inst; i += blockDim.x)
            step_control(s.ctrl + i, s.dt_buf + kDtWords * i, control_mode);
    }
    if (threadIdx.x == 0) {
        volatile uint32_t *sched = s.sched;
        sched[kSchedActive] = sched[kSchedNext];
        sched[kSchedItems] = sched[kSchedNextItems];
        sched[kSchedNext] = 0u;
        sched[kSchedNextItems] = 0u;
        sched[kSchedDone] = 0u;
    }
}

__global__ void step_control_kernel(swe_ctrl_t *c, uint32_t *dt_buf, uint32_t n_inst, int mode) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_inst; i += gridDim.x * blockDim.x)
        step_control(c + i, dt_buf + kDtWords * i, mode);
}

// ---------------------------------------------------------------------------
// Start of a run: wet flag per block (resident.py:738-773).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) block_mark_kernel(swe_mesh_t m, swe_state_t s, float dry_tol, int all_active) {
    for (uint32_t b = blockIdx.x; b < m.n_blocks; b += gridDim.x) {
        const uint32_t i = b * kBlockCells + threadIdx.x;
        bool live = false;
        if (threadIdx.x < m.block_cells[b]) live = s.h[i] >= dry_tol || s.hu[i] != 0.0f || s.hv[i] != 0.0f;
        const int any = __syncthreads_or(live);
        if (threadIdx.x == 0) {
            if (all_active) {
                s.blk[kBlkWords * b + kBlkWet] = 0u;
                s.blk[kBlkWords * b + kBlkActive] = 1u;
            } else {
                s.blk[kBlkWords * b + kBlkWet] = any ? 1u : 0u;
            }
        }
    }
}

__global__ void dt_reset_kernel(uint32_t *dt_buf, uint32_t n_inst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_inst; i += gridDim.x * blockDim.x)
        dt_buf[kDtWords * i] = __float_as_uint(kDtSentinel);
}

// ---------------------------------------------------------------------------
// Prologue CFL bound over every block (cfl_edge_gather + cfl_gather,
// resident.py:528-610): every edge's wave term (0 if dry) into shared memory,
// every cell sums all its slots, each instance's minimum bound into its dt
// word 0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) cfl_prologue_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl) {
    extern __shared__ float4 smem4[];
    float *C = reinterpret_cast<float *>(smem4);
    __shared__ uint32_t red[kThreads / 32];
    for (uint32_t b = blockIdx.x; b < m.n_blocks; b += gridDim.x) {
        const uint32_t base = m.tile_ptr[b], ne = m.tile_count[b];
        for (uint32_t j = threadIdx.x; j < ne; j += kThreads) {
            const uint32_t e = base + j;
            const int cL = m.tile_cl[e], cR = m.tile_cr[e];
            const float nx = m.tile_nx[e], ny = m.tile_ny[e];
            const float hL = s.h[cL], huL = s.hu[cL], hvL = s.hv[cL];
            float hR, huR, hvR;
            if (cR < 0) {
                uint32_t kind = kOpenWall;
                float value = 0.0f;
                boundary_state(m, p, cR, hL, huL, hvL, nx, ny, hR, huR, hvR, kind, value);
            } else {
                hR = s.h[cR];
                huR = s.hu[cR];
                hvR = s.hv[cR];
            }
            float contrib = 0.0f;
            if (hL >= p.dry_tol || hR >= p.dry_tol)
                contrib = wave_bound(p, hL, huL, hvL, m.tile_dzl[e], hR, huR, hvR, m.tile_dzr[e], nx, ny) * m.tile_len[e];
            C[j] = contrib;
        }
        __syncthreads();
        const uint32_t i = b * kBlockCells + threadIdx.x;
        uint32_t bound = kNoBound;
        if (threadIdx.x < m.block_cells[b]) {
            float lam = 0.0f;
            for (uint32_t k = m.cptr[i]; k < m.cptr[i + 1]; ++k) lam += C[m.lcsr[k] >> 1];
            const float A = m.area[i];
            if (lam > 1e-30f && A > 1e-10f) bound = __float_as_uint(cfl * A / lam);
        }
        const uint32_t bmin = block_min_any(bound, red);
        if (threadIdx.x == 0 && bmin != kNoBound) atomicMin(&s.dt_buf[kDtWords * m.block_inst[b]], bmin);
    }
}

__global__ void source_apply_kernel(swe_mesh_t m, swe_state_t s, swe_sources_t src, float dry_tol, int comp) {
    source_apply(m, s, src, dry_tol, comp, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__global__ void source_bound_kernel(swe_mesh_t m, swe_state_t s, swe_sources_t src, Phys p, float cfl) {
    source_bound(m, s, src, p, cfl, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

inline size_t cfl_smem_bytes(uint32_t max_tile_edges) { return ((max_tile_edges + 3u) & ~3u) * sizeof(float); }

inline bool items_fit(const swe_mesh_t *m) {
    return m->max_sub_edges <= 2047u && m->max_sub_slots <= 2047u && m->n_inst <= 1023u && m->n_blocks <= (1u << 23);
}

}  // namespace swe

using namespace swe;

extern "C" {

size_t swe_workspace_bytes(uint32_t n_blocks, uint32_t n_inst) {
    return static_cast<size_t>(n_blocks) * 2u * sizeof(uint32_t)          // active_list, two halves
           + static_cast<size_t>(n_blocks) * 2u * 4u * 4u * sizeof(uint32_t)  // items, two halves
           + static_cast<size_t>(n_blocks) * 2u * sizeof(uint32_t)          // marks
           + 64u * sizeof(uint32_t)                                        // sync
           + 16u * sizeof(uint32_t)                                   // sched
           + static_cast<size_t>(n_inst) * kDtWords * sizeof(uint32_t)  // dt_buf
           + static_cast<size_t>(n_inst) * sizeof(swe_ctrl_t);       // ctrl
}

int swe_apply_sources(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                      const swe_sources_t *sources, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || !sources) return SWE_ERR_ARGUMENT;
    if (sources->count == 0u) return SWE_OK;
    if (!sources->cells || !sources->rate) return SWE_ERR_ARGUMENT;
    if (sources->hydro &&
        (!sources->hscale || !sources->knot_ptr || !sources->knot_t || !sources->knot_q || sources->n_hydro == 0u))
        return SWE_ERR_ARGUMENT;
    const uint32_t grid = min((sources->count + kThreads - 1) / kThreads, 148u * 16u);
    source_apply_kernel<<<grid, kThreads, 0, stream>>>(*mesh, *state, *sources, params->dry_tol,
                                                      static_cast<int>(params->compensated));
    int rc = check_launch();
    if (rc) return rc;
    source_bound_kernel<<<grid, kThreads, 0, stream>>>(*mesh, *state, *sources, Phys{params->g, params->dry_tol}, params->cfl);
    return check_launch();
}

int swe_block_dilate_compact(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int force,
                             int control_mode, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || control_mode < -1 || control_mode > 2) return SWE_ERR_ARGUMENT;
    if (!items_fit(mesh)) return SWE_ERR_TOO_LARGE;
    const uint32_t grid = (mesh->n_blocks + kDilateWarps - 1) / kDilateWarps;
    dilate_compact_kernel<<<grid, kDilateWarps * 32, 0, stream>>>(*mesh, *state, params->active_set ? 0 : 1, force, control_mode);
    return check_launch();
}

int swe_block_mark(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params) return SWE_ERR_ARGUMENT;
    block_mark_kernel<<<min(mesh->n_blocks, 148u * 8u), kThreads, 0, stream>>>(*mesh, *state, params->dry_tol,
                                                                             params->active_set ? 0 : 1);
    return check_launch();
}

int swe_cfl_prologue(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params) return SWE_ERR_ARGUMENT;
    dt_reset_kernel<<<(mesh->n_inst + 255u) / 256u, 256, 0, stream>>>(state->dt_buf, mesh->n_inst);
    int rc = check_launch();
    if (rc) return rc;
    const size_t bytes = cfl_smem_bytes(mesh->max_tile_edges);
    rc = set_smem(cfl_prologue_kernel, bytes);
    if (rc) return rc;
    const uint32_t grid = (params->grid == 0u || params->grid > mesh->n_blocks) ? mesh->n_blocks : params->grid;
    cfl_prologue_kernel<<<grid, kThreads, bytes, stream>>>(*mesh, *state, Phys{params->g, params->dry_tol}, params->cfl);
    return check_launch();
}

int swe_step_control(swe_ctrl_t *ctrl, uint32_t *dt_buf, uint32_t n_inst, int mode, swe_stream_t stream) {
    if (!ctrl || !dt_buf || n_inst == 0u || mode < 0 || mode > 2) return SWE_ERR_ARGUMENT;
    step_control_kernel<<<(n_inst + 255u) / 256u, 256, 0, stream>>>(ctrl, dt_buf, n_inst, mode);
    return check_launch();
}

int swe_prologue(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, swe_stream_t stream) {
    int rc = swe_block_mark(mesh, state, params, stream);
    if (rc) return rc;
    rc = swe_block_dilate_compact(mesh, state, params, 1, -1, stream);
    if (rc) return rc;
    rc = swe_cfl_prologue(mesh, state, params, stream);
    if (rc) return rc;
    return swe_step_control(state->ctrl, state->dt_buf, mesh->n_inst, 0, stream);
}

int swe_step(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, const swe_sources_t *sources,
             swe_stream_t stream) {
    int rc = swe_stage(mesh, state, params, 0, stream);
    if (rc) return rc;
    rc = swe_stage(mesh, state, params, 1, stream);
    if (rc) return rc;
    if (sources && sources->count) {
        rc = swe_apply_sources(mesh, state, params, sources, stream);
        if (rc) return rc;
    }
    return swe_block_dilate_compact(mesh, state, params, 0, 1, stream);
}

}  // extern "C"
