// One Heun stage of the shallow-water step (flux_resident_gather +
// update_resident_gather[_comp], inundation/vulkan/shaders/resident.py:187-291,
// 312-344, 354-513), fused per tile: every edge flux a tile's cells need is
// computed into shared memory, gathered in the reference's fixed per-cell CSR
// order and applied by the compensated Heun update. An edge shared by two
// tiles is computed by both, from the same inputs by the same instructions,
// so both see the same bits. No per-edge buffer goes through HBM and no float
// atomics are used.
//
// Three kernels with the same arithmetic:
//  * stage_tiled_kernel: 64-cell tiles from the dilation's work items,
//    staged into shared memory by bulk copies (double-buffered) -- the default;
//  * stage_block_kernel: 256-cell blocks with plain loads;
//  * stage_staged_kernel: 256-cell blocks staged into shared memory by bulk copies.
#include <cuda_runtime.h>

#include <cstdint>

#include "swe_tiled.cuh"

namespace swe {

// A block's edge words in shared memory: the six side words, then the CFL word.
__device__ __forceinline__ SideWords block_side_words(uint32_t cap) {
    extern __shared__ float4 smem4[];
    float *f = reinterpret_cast<float *>(smem4);
    return SideWords{f, f + 6 * cap, cap};
}

inline size_t block_smem_bytes(uint32_t max_tile_edges) {
    const size_t cap = (max_tile_edges + 3u) & ~3u;
    return cap * 7 * sizeof(float);
}

// ---------------------------------------------------------------------------
// 256-cell blocks, plain loads: persistent CTAs stride over the active list.
// sums != nullptr: also store every computed cell's gathered sums (sdh, sdhu,
// sdhv at sums[i], sums[n + i], sums[2n + i], n = padded cells), the record
// the adjoint reverses. OPEN: the mesh has open edges.
// ---------------------------------------------------------------------------
// CTAs of the block kernel that must fit on one SM: 8 x 256 threads caps a thread at 32
// registers, so the SM holds its full 64 warps; the measured all-wet step is fastest there
// (fewer registers and CTAs cost more than the few spilled words).
#ifndef SWE_BLOCK_MIN_CTAS
#define SWE_BLOCK_MIN_CTAS 8
#endif

template <int STAGE, bool COMP, bool CLAMP, bool OPEN>
__global__ void __launch_bounds__(kThreads, SWE_BLOCK_MIN_CTAS)
    stage_block_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl, float *sums) {
    const uint32_t cap = (m.max_tile_edges + 3u) & ~3u;
    const SideWords S = block_side_words(cap);
    __shared__ uint32_t red[2 * kThreads / 32];
    const uint32_t count = s.sched[kSchedActive];
    uint64_t computed = 0;

    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        const uint32_t b = s.active_list[w];
        const uint32_t inst = m.block_inst[b];
        const uint32_t dt_bits = s.dt_buf[kDtWords * inst];
        if (dt_bits == 0u) continue;  // this instance's window is done: a no-op step
        const float dt = __uint_as_float(dt_bits);
        const uint32_t base = m.tile_ptr[b], ne = m.tile_count[b], cells = m.block_cells[b];

        for (uint32_t j = threadIdx.x; j < ne; j += kThreads) {
            const uint32_t e = base + j;
            const int cL = m.tile_cl[e], cR = m.tile_cr[e];
            const float nx = m.tile_nx[e], ny = m.tile_ny[e];
            float hL, huL, hvL, hR, huR, hvR;
            load_state<STAGE>(s, cL, hL, huL, hvL);
            uint32_t kind = kOpenWall;
            float value = 0.0f;
            if (cR < 0) {
                if (OPEN) {
                    boundary_state(m, p, cR, hL, huL, hvL, nx, ny, hR, huR, hvR, kind, value);
                } else {
                    hR = hL;
                    wall_mirror(huL, hvL, nx, ny, huR, hvR);
                }
            } else {
                load_state<STAGE>(s, cR, hR, huR, hvR);
            }
            const bool live = !(hL < p.dry_tol && hR < p.dry_tol) || (OPEN && open_forced(kind, value));
            float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f, w4 = 0.0f, w5 = 0.0f;
            if (live) {
                edge_words<OPEN>(p, cR, nx, ny, m.tile_len[e], m.tile_dzl[e], m.tile_dzr[e], hL, huL, hvL, hR, huR,
                                 hvR, w0, w1, w2, w3, w4, w5, kind, value);
                if (OPEN && cR < -1) tally_open(s.open_vol, static_cast<uint32_t>(-2 - cR), (0.5f * dt) * w0);
            }
            put_side_words<STAGE>(S, j, live, w0, w1, w2, w3, w4, w5);
        }
        __syncthreads();

        const uint32_t i = b * kBlockCells + threadIdx.x;
        bool wet = false;
        uint32_t bound = kNoBound;
        if (threadIdx.x < cells) {
            float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
            for (uint32_t k = m.cptr[i], k1 = m.cptr[i + 1]; k < k1; ++k)
                add_side_words<STAGE>(S, m.lcsr[k], sdh, sdhu, sdhv, lam);
            const float hi = STAGE ? s.h1[i] : s.h[i], hui = STAGE ? s.hu1[i] : s.hu[i];
            const float hvi = STAGE ? s.hv1[i] : s.hv[i];
            const float loi = COMP ? (STAGE ? s.h1_lo[i] : s.h_lo[i]) : 0.0f;
            const float h0 = STAGE ? s.h[i] : 0.0f, hu0 = STAGE ? s.hu[i] : 0.0f, hv0 = STAGE ? s.hv[i] : 0.0f;
            const float lo0 = (STAGE && COMP) ? s.h_lo[i] : 0.0f;
            if (sums) {
                const uint32_t n = m.n_blocks * kBlockCells;
                sums[i] = sdh;
                sums[n + i] = sdhu;
                sums[2 * n + i] = sdhv;
            }
            update_cell<STAGE, COMP, CLAMP>(s, p, cfl, dt, i, m.area[i], m.n_mann[i], hi, hui, hvi, loi, h0, hu0, hv0,
                                            lo0, sdh, sdhu, sdhv, lam, wet, bound);
        }
        if (STAGE == 1) {
            bool any_wet;
            uint32_t bmin;
            tile_outcome(wet, bound, red, any_wet, bmin);
            if (threadIdx.x == 0) {
                s.blk[kBlkWords * b + kBlkWet] = any_wet ? 1u : 0u;
                if (bmin != kNoBound) atomicMin(&s.dt_buf[kDtWords * inst + 1], bmin);
                computed += cells;
            }
        } else {
            __syncthreads();
        }
    }
    if (STAGE == 1 && threadIdx.x == 0 && computed)
        atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed), computed);
}

// ---------------------------------------------------------------------------
// 256-cell blocks staged by bulk copies: a CTA's shared memory holds one block
// at a time -- its edge records (7 arrays), its cells' columns (the stage's
// input state, area, n, and the committed state in the corrector), its CSR
// pointers and local CSR -- copied in by one mbarrier's bulk copies, so a
// block's bytes are in flight at once instead of a few loads per thread.
// The flux words overwrite the records they came from. CTAs stride over the
// active list; each CTA reads its next block's indices while that block's
// predecessor is staged. Same arithmetic as the other stage kernels.
// ---------------------------------------------------------------------------
#ifndef SWE_STAGED_MIN_CTAS
#define SWE_STAGED_MIN_CTAS 5
#endif
// Cell columns a stage stages: the input state, area and n, and in the corrector the committed state.
__host__ __device__ constexpr uint32_t staged_cols(int stage) { return stage ? 10u : 6u; }

struct StagedPlan {
    uint32_t capE, capS, nc, total;
};

// Layout: mbarrier (128 B), records 7 x capE words, nc cell columns of 256 words, 260
// CSR pointers, capS local-CSR slots.
__host__ __device__ inline StagedPlan staged_plan(uint32_t max_edges, uint32_t max_slots, uint32_t nc) {
    StagedPlan L;
    L.capE = (max_edges + 31u) & ~31u;
    L.capS = (max_slots + 7u) & ~7u;
    L.nc = nc;
    L.total = 128u + 28u * L.capE + nc * 1024u + 1040u + ((2u * L.capS + 15u) & ~15u);
    return L;
}

// The fields of the block at active-list position w (thread 0): block, dt bits, first
// record, records, first local-CSR slot, slots, real cells.
__device__ __forceinline__ void staged_fields(const swe_mesh_t &m, const swe_state_t &s, uint32_t w, uint32_t *f) {
    const uint32_t b = s.active_list[w];
    const uint32_t inst = m.block_inst[b];
    const uint32_t l0 = m.blk_lcsr_ptr[b];
    f[0] = b;
    f[1] = s.dt_buf[kDtWords * inst];
    f[2] = m.tile_ptr[b];
    f[3] = m.tile_count[b];
    f[4] = l0;
    f[5] = m.blk_lcsr_ptr[b + 1] - l0;
    f[6] = m.block_cells[b];
}

template <int STAGE, bool COMP, bool CLAMP, bool OPEN>
__global__ void __launch_bounds__(kThreads, SWE_STAGED_MIN_CTAS)
    stage_staged_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl, float *sums) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t red[2 * kThreads / 32];
    __shared__ uint32_t fields[2][8];
    constexpr uint32_t nc = staged_cols(STAGE);
    const StagedPlan L = staged_plan(m.max_tile_edges, m.max_blk_slots, nc);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    int32_t *Rcl = reinterpret_cast<int32_t *>(smem + 128);
    int32_t *Rcr = Rcl + L.capE;
    float *Rnx = reinterpret_cast<float *>(Rcr + L.capE), *Rny = Rnx + L.capE, *Rlen = Rny + L.capE;
    float *Rdzl = Rlen + L.capE, *Rdzr = Rdzl + L.capE;
    float *C = Rdzr + L.capE;  // columns: 0..3 the stage's input state, 4 area, 5 n, 6..9 committed
    uint32_t *Cp = reinterpret_cast<uint32_t *>(C + nc * kBlockCells);
    uint16_t *Lc = reinterpret_cast<uint16_t *>(Cp + 260);
    // The flux words overwrite the records: the six side words over cR..dzr, the CFL word over cL.
    const SideWords S{reinterpret_cast<float *>(Rcr), reinterpret_cast<float *>(Rcl), L.capE};
    const uint32_t tid = threadIdx.x;
    const uint32_t count = s.sched[kSchedActive];
    if (tid == 0) {
        mbar_init(bar, 1u);
        fence_barrier_init();
        if (blockIdx.x < count) staged_fields(m, s, blockIdx.x, fields[0]);
    }
    __syncthreads();
    uint64_t computed = 0;
    uint32_t k = 0, phase = 0;
    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x, ++k) {
        const uint32_t *f = fields[k & 1u];
        const uint32_t b = f[0], dt_bits = f[1], e0 = f[2], ne = f[3], l0 = f[4], lp = f[5], cells = f[6];
        if (dt_bits != 0u && tid < 32u) {
            const uint32_t lane = tid, ep = (ne + 31u) & ~31u;  // segments are padded to 32 records
            if (lane == 0) mbar_expect_tx(bar, 28u * ep + nc * 1024u + 1040u + 2u * lp);
            __syncwarp();
            if (lane < 7u) {
                if (ep != 0u) {
                    const void *src;
                    void *dst;
                    switch (lane) {
                        case 0: src = m.tile_cl; dst = Rcl; break;
                        case 1: src = m.tile_cr; dst = Rcr; break;
                        case 2: src = m.tile_nx; dst = Rnx; break;
                        case 3: src = m.tile_ny; dst = Rny; break;
                        case 4: src = m.tile_len; dst = Rlen; break;
                        case 5: src = m.tile_dzl; dst = Rdzl; break;
                        default: src = m.tile_dzr; dst = Rdzr; break;
                    }
                    bulk_load(dst, static_cast<const char *>(src) + 4ull * e0, ep * 4u, bar);
                }
            } else if (lane < 7u + nc) {
                const uint32_t c = lane - 7u;
                const float *src;
                switch (c) {
                    case 0: src = STAGE ? s.h1 : s.h; break;
                    case 1: src = STAGE ? s.hu1 : s.hu; break;
                    case 2: src = STAGE ? s.hv1 : s.hv; break;
                    case 3: src = STAGE ? s.h1_lo : s.h_lo; break;
                    case 4: src = m.area; break;
                    case 5: src = m.n_mann; break;
                    case 6: src = s.h; break;
                    case 7: src = s.hu; break;
                    case 8: src = s.hv; break;
                    default: src = s.h_lo; break;
                }
                bulk_load(C + c * kBlockCells, src + static_cast<size_t>(b) * kBlockCells, 1024u, bar);
            } else if (lane == 7u + nc) {
                bulk_load(Cp, m.cptr + static_cast<size_t>(b) * kBlockCells, 1040u, bar);
            } else if (lane == 8u + nc && lp != 0u) {
                bulk_load(Lc, m.blk_lcsr + l0, 2u * lp, bar);
            }
        }
        // the next block's indices arrive while this one is staged
        if (tid == 0 && w + gridDim.x < count) staged_fields(m, s, w + gridDim.x, fields[(k + 1u) & 1u]);
        if (dt_bits == 0u) {  // this instance's window is done: a no-op step
            __syncthreads();
            continue;
        }
        const bool ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!__syncthreads_and(ok)) {
            // The staged data never arrived: report it, give the copies one more bounded wait, stop.
            if (tid == 0) atomicOr(&s.ctrl->error, 1u);
            mbar_wait(bar, phase ^ 1u);
            return;
        }
        const float dt = __uint_as_float(dt_bits);
        const int base = static_cast<int>(b * kBlockCells);
        const float *C0 = C, *C1 = C + kBlockCells, *C2 = C + 2 * kBlockCells;

        for (uint32_t j = tid; j < ne; j += kThreads) {
            const int cL = Rcl[j], cR = Rcr[j];
            const float nx = Rnx[j], ny = Rny[j];
            float hL, huL, hvL, hR, huR, hvR;
            const uint32_t lL = static_cast<uint32_t>(cL - base);
            if (lL < static_cast<uint32_t>(kBlockCells)) {
                hL = C0[lL];
                huL = C1[lL];
                hvL = C2[lL];
            } else {
                load_state<STAGE>(s, cL, hL, huL, hvL);
            }
            uint32_t kind = kOpenWall;
            float value = 0.0f;
            if (cR < 0) {
                if (OPEN) {
                    boundary_state(m, p, cR, hL, huL, hvL, nx, ny, hR, huR, hvR, kind, value);
                } else {
                    hR = hL;
                    wall_mirror(huL, hvL, nx, ny, huR, hvR);
                }
            } else {
                const uint32_t lR = static_cast<uint32_t>(cR - base);
                if (lR < static_cast<uint32_t>(kBlockCells)) {
                    hR = C0[lR];
                    huR = C1[lR];
                    hvR = C2[lR];
                } else {
                    load_state<STAGE>(s, cR, hR, huR, hvR);
                }
            }
            const bool live = !(hL < p.dry_tol && hR < p.dry_tol) || (OPEN && open_forced(kind, value));
            const float len = Rlen[j], dzl = Rdzl[j], dzr = Rdzr[j];
            float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f, w4 = 0.0f, w5 = 0.0f;
            if (live) {
                edge_words<OPEN>(p, cR, nx, ny, len, dzl, dzr, hL, huL, hvL, hR, huR, hvR, w0, w1, w2, w3, w4, w5,
                                 kind, value);
                if (OPEN && cR < -1) tally_open(s.open_vol, static_cast<uint32_t>(-2 - cR), (0.5f * dt) * w0);
            }
            put_side_words<STAGE>(S, j, live, w0, w1, w2, w3, w4, w5);
        }
        __syncthreads();

        bool wet = false;
        uint32_t bound = kNoBound;
        if (tid < cells) {
            const uint32_t i = b * kBlockCells + tid;
            float h0 = 0.0f, hu0 = 0.0f, hv0 = 0.0f, lo0 = 0.0f;  // the corrector's committed state
            if (STAGE) {
                h0 = C[6 * kBlockCells + tid];
                hu0 = C[7 * kBlockCells + tid];
                hv0 = C[8 * kBlockCells + tid];
                lo0 = C[9 * kBlockCells + tid];
            }
            float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
            const uint32_t q0 = Cp[tid] - Cp[0], q1 = Cp[tid + 1] - Cp[0];
            for (uint32_t q = q0; q < q1; ++q) add_side_words<STAGE>(S, Lc[q], sdh, sdhu, sdhv, lam);
            if (sums) {
                const uint32_t n = m.n_blocks * kBlockCells;
                sums[i] = sdh;
                sums[n + i] = sdhu;
                sums[2 * n + i] = sdhv;
            }
            update_cell<STAGE, COMP, CLAMP>(s, p, cfl, dt, i, C[4 * kBlockCells + tid], C[5 * kBlockCells + tid],
                                            C[tid], C[kBlockCells + tid], C[2 * kBlockCells + tid],
                                            C[3 * kBlockCells + tid], h0, hu0, hv0, lo0, sdh, sdhu, sdhv, lam, wet,
                                            bound);
        }
        if (STAGE == 1) {
            bool any_wet;
            uint32_t bmin;
            tile_outcome(wet, bound, red, any_wet, bmin);
            if (tid == 0) {
                s.blk[kBlkWords * b + kBlkWet] = any_wet ? 1u : 0u;
                if (bmin != kNoBound) atomicMin(&s.dt_buf[kDtWords * m.block_inst[b] + 1], bmin);
                computed += cells;
            }
        }
        // the shared memory is refilled by the next block's bulk copies
        fence_proxy_async();
        __syncthreads();
    }
    if (STAGE == 1 && tid == 0 && computed)
        atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed), computed);
}

template <int STAGE, bool COMP, bool CLAMP, bool OPEN>
__global__ void __launch_bounds__(kTileThreads, 8)
    stage_tiled_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl, float *sums) {
    if (blockIdx.x >= s.sched[kSchedItems]) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ TiledShared<kTileThreads> sh;
    if (threadIdx.x == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(smem), 1u);
        mbar_init(reinterpret_cast<uint64_t *>(smem) + 1, 1u);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t k = 0;
    uint64_t computed = 0;
    if (!tiled_pass<STAGE, COMP, CLAMP, kTileThreads, OPEN>(m, s, p, cfl, smem, sh, k, computed, sums))
        return;
    if (STAGE == 1 && threadIdx.x == 0 && computed)
        atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed), computed);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
template <int STAGE, bool COMP, bool CLAMP, bool OPEN>
int launch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st,
                 float *sums = nullptr) {
    const Phys ph{p->g, p->dry_tol};
    if (p->kernel == 3u) {
        if (!m->blk_lcsr || !m->blk_lcsr_ptr) return SWE_ERR_ARGUMENT;
        auto kern = stage_staged_kernel<STAGE, COMP, CLAMP, OPEN>;
        const size_t bytes = staged_plan(m->max_tile_edges, m->max_blk_slots, staged_cols(STAGE)).total;
        int rc = set_smem(kern, bytes);
        if (rc) return rc;
        const uint32_t grid = (p->grid == 0u || p->grid > m->n_blocks) ? m->n_blocks : p->grid;
        kern<<<grid, kThreads, bytes, st>>>(*m, *s, ph, p->cfl, sums);
        return check_launch();
    }
    if (p->kernel == 1u) {
        auto kern = stage_block_kernel<STAGE, COMP, CLAMP, OPEN>;
        const size_t bytes = block_smem_bytes(m->max_tile_edges);
        int rc = set_smem(kern, bytes);
        if (rc) return rc;
        const uint32_t grid = (p->grid == 0u || p->grid > m->n_blocks) ? m->n_blocks : p->grid;
        kern<<<grid, kThreads, bytes, st>>>(*m, *s, ph, p->cfl, sums);
        return check_launch();
    }
    auto kern = stage_tiled_kernel<STAGE, COMP, CLAMP, OPEN>;
    const size_t bytes = tile_plan(m->max_sub_edges, m->max_sub_slots, STAGE ? 10u : 6u).total;
    int rc = set_smem(kern, bytes);
    if (rc) return rc;
    kern<<<p->grid ? p->grid : 148u * 8u, kTileThreads, bytes, st>>>(*m, *s, ph, p->cfl, sums);
    return check_launch();
}

template <int STAGE, bool OPEN>
int dispatch_open(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st, float *sums) {
    if (p->compensated) {
        return p->track_clamp ? launch_stage<STAGE, true, true, OPEN>(m, s, p, st, sums)
                              : launch_stage<STAGE, true, false, OPEN>(m, s, p, st, sums);
    }
    return p->track_clamp ? launch_stage<STAGE, false, true, OPEN>(m, s, p, st, sums)
                          : launch_stage<STAGE, false, false, OPEN>(m, s, p, st, sums);
}

template <int STAGE>
int dispatch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st,
                   float *sums = nullptr) {
    return m->n_open ? dispatch_open<STAGE, true>(m, s, p, st, sums) : dispatch_open<STAGE, false>(m, s, p, st, sums);
}

template <int STAGE, bool COMP, bool CLAMP>
int configure_stage(const swe_mesh_t *m) {
    const size_t block = block_smem_bytes(m->max_tile_edges);
    const size_t tiled = tile_plan(m->max_sub_edges, m->max_sub_slots, STAGE ? 10u : 6u).total;
    const size_t staged = staged_plan(m->max_tile_edges, m->max_blk_slots, staged_cols(STAGE)).total;
    int rc = set_smem(stage_block_kernel<STAGE, COMP, CLAMP, false>, block);
    if (!rc) rc = set_smem(stage_block_kernel<STAGE, COMP, CLAMP, true>, block);
    // a mesh whose largest block does not fit the staged kernel's shared memory runs the others
    if (!rc && staged <= kMaxSmem) rc = set_smem(stage_staged_kernel<STAGE, COMP, CLAMP, false>, staged);
    if (!rc && staged <= kMaxSmem) rc = set_smem(stage_staged_kernel<STAGE, COMP, CLAMP, true>, staged);
    if (!rc) rc = set_smem(stage_tiled_kernel<STAGE, COMP, CLAMP, false>, tiled);
    if (!rc) rc = set_smem(stage_tiled_kernel<STAGE, COMP, CLAMP, true>, tiled);
    return rc;
}

int configure_persistent(const swe_mesh_t *mesh, int *blocks_per_sm);  // swe_persist.cu

}  // namespace swe

using namespace swe;

extern "C" {

int swe_configure(const swe_mesh_t *mesh, int kernel, int *blocks_per_sm) {
    if (!mesh_ok(mesh) || !blocks_per_sm || kernel < 0 || kernel > 3) return SWE_ERR_ARGUMENT;
    if (mesh->max_sub_edges > 2047u || mesh->max_sub_slots > 2047u || mesh->n_inst > 1023u) return SWE_ERR_TOO_LARGE;
    int rc = configure_stage<0, false, false>(mesh);
    if (!rc) rc = configure_stage<0, false, true>(mesh);
    if (!rc) rc = configure_stage<0, true, false>(mesh);
    if (!rc) rc = configure_stage<0, true, true>(mesh);
    if (!rc) rc = configure_stage<1, false, false>(mesh);
    if (!rc) rc = configure_stage<1, false, true>(mesh);
    if (!rc) rc = configure_stage<1, true, false>(mesh);
    if (!rc) rc = configure_stage<1, true, true>(mesh);
    if (rc) return rc;
    if (kernel == 2) return configure_persistent(mesh, blocks_per_sm);
    cudaError_t err;
    if (kernel == 0) {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            blocks_per_sm, stage_tiled_kernel<1, true, false, false>, kTileThreads,
            tile_plan(mesh->max_sub_edges, mesh->max_sub_slots, 10u).total);
    } else if (kernel == 3) {
        const size_t bytes = staged_plan(mesh->max_tile_edges, mesh->max_blk_slots, staged_cols(1)).total;
        *blocks_per_sm = 0;  // 0: this mesh's blocks do not fit
        err = bytes > kMaxSmem ? cudaSuccess
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                     blocks_per_sm, stage_staged_kernel<1, true, false, false>, kThreads, bytes);
    } else {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, stage_block_kernel<1, true, false, false>, kThreads,
                                                            block_smem_bytes(mesh->max_tile_edges));
    }
    return err == cudaSuccess ? SWE_OK : SWE_ERR_CUDA;
}

int swe_stage(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !open_ok(mesh, state) || !params || params->kernel == 2u ||
        params->kernel > 3u)
        return SWE_ERR_ARGUMENT;
    if (stage == 0) return dispatch_stage<0>(mesh, state, params, stream);
    if (stage == 1) return dispatch_stage<1>(mesh, state, params, stream);
    return SWE_ERR_ARGUMENT;
}

int swe_stage_taped(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage,
                    float *sums, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || !sums || mesh->n_open) return SWE_ERR_ARGUMENT;
    if (stage == 0) return dispatch_stage<0>(mesh, state, params, stream, sums);
    if (stage == 1) return dispatch_stage<1>(mesh, state, params, stream, sums);
    return SWE_ERR_ARGUMENT;
}

}  // extern "C"
