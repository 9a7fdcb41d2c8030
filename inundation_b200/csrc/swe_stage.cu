// One Heun stage of the shallow-water step (flux_resident_gather +
// update_resident_gather[_comp], inundation/vulkan/shaders/resident.py:187-291,
// 312-344, 354-513), fused per tile: every edge flux a tile's cells need is
// computed into shared memory, gathered in the reference's fixed per-cell CSR
// order and applied by the compensated Heun update. An edge shared by two
// tiles is computed by both, from the same inputs by the same instructions,
// so both see the same bits. No per-edge buffer goes through HBM and no float
// atomics are used.
//
// Two kernels with the same arithmetic:
//  * stage_tiled_kernel: 64-cell tiles from the dilation's work items,
//    staged into shared memory by bulk copies (double-buffered) -- the default;
//  * stage_block_kernel: 256-cell blocks with plain loads.
#include <cuda_runtime.h>

#include <cstdint>

#include "swe_common.cuh"

namespace swe {

// Per-edge words of a tile in shared memory (also used by the prologue).
struct TileSmem {
    float *F0, *L1, *L2, *R1, *R2, *C;
    uint8_t *live;
};

__device__ __forceinline__ TileSmem tile_smem(uint32_t cap) {
    extern __shared__ float4 smem4[];
    float *f = reinterpret_cast<float *>(smem4);
    TileSmem t;
    t.F0 = f;
    t.L1 = f + cap;
    t.L2 = f + 2 * cap;
    t.R1 = f + 3 * cap;
    t.R2 = f + 4 * cap;
    t.C = f + 5 * cap;
    t.live = reinterpret_cast<uint8_t *>(f + 6 * cap);
    return t;
}

inline size_t block_smem_bytes(uint32_t max_tile_edges) {
    const size_t cap = (max_tile_edges + 3u) & ~3u;
    return cap * 6 * sizeof(float) + ((cap + 15) & ~size_t(15));
}

// The compensated Heun update of one cell from its gathered sums (resident.py:354-513).
template <int STAGE, bool COMP, bool CLAMP>
__device__ __forceinline__ void update_cell(const swe_state_t &s, const Phys &p, float cfl, float dt, uint32_t i,
                                            float A, float n, float hi, float hui, float hvi, float loi, float h0,
                                            float hu0, float hv0, float lo0, float sdh, float sdhu, float sdhv,
                                            float lam, bool &wet, uint32_t &bound) {
    const float dti = dt / A;
    float h_new, lo_new, h_raw;
    if (COMP) {
        add_compensated(hi, loi, -dti * sdh, h_new, lo_new);
        float s_raw, e_raw;
        two_sum(hi, -dti * sdh, s_raw, e_raw);
        h_raw = s_raw + (e_raw + loi);
    } else {
        h_raw = hi - dti * sdh;
        h_new = gmax(h_raw, 0.0f);
        lo_new = 0.0f;
    }
    float hu_new = hui - dti * sdhu;
    float hv_new = hvi - dti * sdhv;
    if (CLAMP) s.clamp_mass[i] += 0.5f * A * (h_new - h_raw);
    if (h_new < p.dry_tol) {
        hu_new = 0.0f;
        hv_new = 0.0f;
    }
    if (h_new >= p.dry_tol) {
        const float drag = film_drag(p, h_new, dt);
        hu_new *= drag;
        hv_new *= drag;
        const float u_ = hu_new / h_new, v_ = hv_new / h_new;
        const float spd = sqrtf(u_ * u_ + v_ * v_);
        const float Sf = p.g * n * n * spd / pow43(h_new);
        const float den = 1.0f + dt * Sf;
        hu_new = hu_new / den;
        hv_new = hv_new / den;
    }
    if (STAGE == 0) {
        s.h1[i] = h_new;
        if (COMP) s.h1_lo[i] = lo_new;
        s.hu1[i] = hu_new;
        s.hv1[i] = hv_new;
        return;
    }
    float hf;
    if (COMP) {
        float sm, em, lof;
        two_sum(h0, h_new, sm, em);
        em += lo0 + lo_new;
        two_sum(0.5f * sm, 0.5f * em, hf, lof);
        s.h_lo[i] = lof;
    } else {
        hf = 0.5f * (h0 + h_new);
    }
    s.h[i] = hf;
    float huf = 0.5f * (hu0 + hu_new);
    float hvf = 0.5f * (hv0 + hv_new);
    if (hf < p.dry_tol) {
        huf = 0.0f;
        hvf = 0.0f;
    }
    s.hu[i] = huf;
    s.hv[i] = hvf;
    wet = hf >= p.dry_tol;
    if (lam > 1e-30f && A > 1e-10f) bound = __float_as_uint(cfl * A / lam);
}

// Flux of one edge from its two cell states: the five gather words and the
// corrector's CFL word (resident.py:254-284).
__device__ __forceinline__ void edge_words(const Phys &p, int cR, float nx, float ny, float len, float dzL,
                                           float dzR, float hL, float huL, float hvL, float hR, float huR,
                                           float hvR, float &w0, float &w1, float &w2, float &w3, float &w4,
                                           float &w5) {
    float hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, smax;
    face_states(p, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx, ny, hLs, hqnL, hqtL, hRs, hqnR, hqtR);
    hllc(p, hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, smax);
    if (cR < 0) Fh = 0.0f;  // a wall passes no mass
    const float Fhu = Fhn * nx - Fht * ny;
    const float Fhv = Fhn * ny + Fht * nx;
    const float SL_g = 0.5f * p.g * (hL * hL - hLs * hLs);
    const float SR_g = 0.5f * p.g * (hR * hR - hRs * hRs);
    w0 = Fh * len;
    w1 = Fhu * len + SL_g * nx * len;
    w2 = Fhv * len + SL_g * ny * len;
    w3 = Fhu * len + SR_g * nx * len;
    w4 = Fhv * len + SR_g * ny * len;
    w5 = smax * len;
}

// ---------------------------------------------------------------------------
// 256-cell blocks, plain loads: persistent CTAs stride over the active list.
// sums != nullptr: also store every computed cell's gathered sums (sdh, sdhu,
// sdhv at sums[i], sums[n + i], sums[2n + i], n = padded cells), the record
// the adjoint reverses.
// ---------------------------------------------------------------------------
template <int STAGE, bool COMP, bool CLAMP>
__global__ void __launch_bounds__(kThreads)
    stage_block_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl, float *sums) {
    const uint32_t cap = (m.max_tile_edges + 3u) & ~3u;
    const TileSmem t = tile_smem(cap);
    __shared__ uint32_t red[kThreads / 32];
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
            if (cR < 0) {
                hR = hL;
                wall_mirror(huL, hvL, nx, ny, huR, hvR);
            } else {
                load_state<STAGE>(s, cR, hR, huR, hvR);
            }
            const bool live = !(hL < p.dry_tol && hR < p.dry_tol);
            t.live[j] = live;
            if (!live) continue;
            float c;
            edge_words(p, cR, nx, ny, m.tile_len[e], m.tile_dzl[e], m.tile_dzr[e], hL, huL, hvL, hR, huR, hvR,
                       t.F0[j], t.L1[j], t.L2[j], t.R1[j], t.R2[j], c);
            if (STAGE == 1) t.C[j] = c;
        }
        __syncthreads();

        const uint32_t i = b * kBlockCells + threadIdx.x;
        bool wet = false;
        uint32_t bound = kNoBound;
        if (threadIdx.x < cells) {
            float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
            for (uint32_t k = m.cptr[i], k1 = m.cptr[i + 1]; k < k1; ++k) {
                const uint32_t v = m.lcsr[k];
                const uint32_t j = v >> 1;
                if (!t.live[j]) continue;  // a dry-dry edge was not computed and adds nothing
                if (v & 1u) {
                    sdh -= t.F0[j];
                    sdhu -= t.R1[j];
                    sdhv -= t.R2[j];
                } else {
                    sdh += t.F0[j];
                    sdhu += t.L1[j];
                    sdhv += t.L2[j];
                }
                if (STAGE == 1) lam += t.C[j];
            }
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
            const int any_wet = __syncthreads_or(wet);
            const uint32_t bmin = block_min_any(bound, red);
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
// 64-cell tiles from work items, staged by bulk copies.
// ---------------------------------------------------------------------------
struct TilePlan {
    uint32_t capE, capS, nc, buf_bytes, total;
};

__host__ __device__ inline TilePlan tile_plan(uint32_t max_edges, uint32_t max_slots, uint32_t nc) {
    TilePlan L;
    L.capE = (max_edges + 31u) & ~31u;
    L.capS = (max_slots + 63u) & ~63u;
    L.nc = nc;
    L.buf_bytes = 7u * L.capE * 4u + nc * 256u + 384u + L.capS * 2u;
    L.total = 128u + 2u * L.buf_bytes;
    return L;
}

struct TileBuf {
    int32_t *cl, *cr;
    float *nx, *ny, *len, *dzl, *dzr;
    float *c;        // nc x 64: [0..3] the stage's input state, [4] area, [5] n, [6..9] committed state (stage 1)
    uint32_t *cptr;  // 68
    uint16_t *lcsr;
    uint64_t *bar;
};

__device__ __forceinline__ TileBuf tile_buf(unsigned char *smem, const TilePlan &L, uint32_t k) {
    unsigned char *base = smem + 128u + k * L.buf_bytes;
    const uint32_t e = L.capE * 4u;
    TileBuf B;
    B.cl = reinterpret_cast<int32_t *>(base);
    B.cr = reinterpret_cast<int32_t *>(base + e);
    B.nx = reinterpret_cast<float *>(base + 2u * e);
    B.ny = reinterpret_cast<float *>(base + 3u * e);
    B.len = reinterpret_cast<float *>(base + 4u * e);
    B.dzl = reinterpret_cast<float *>(base + 5u * e);
    B.dzr = reinterpret_cast<float *>(base + 6u * e);
    B.c = reinterpret_cast<float *>(base + 7u * e);
    B.cptr = reinterpret_cast<uint32_t *>(base + 7u * e + L.nc * 256u);
    B.lcsr = reinterpret_cast<uint16_t *>(base + 7u * e + L.nc * 256u + 384u);
    B.bar = reinterpret_cast<uint64_t *>(smem) + k;
    return B;
}

struct Item {
    uint32_t tile, cells, e0, l0, ne, lp, inst;
};

__device__ __forceinline__ Item unpack(uint4 v) {
    return Item{v.x & 0x1FFFFFFu, v.x >> 25, v.y, v.z, v.w & 2047u, (v.w >> 11) & 2047u, v.w >> 22};
}

// Warp 0 stages a work item into buffer B: one bulk copy per lane.
template <int STAGE>
__device__ __forceinline__ void tile_issue(const swe_mesh_t &m, const swe_state_t &s, const Item &it, const TileBuf &B) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ep = (it.ne + 31u) & ~31u;  // the record segment is padded to 32
    const uint32_t c0 = it.tile * kTileCells;
    constexpr uint32_t nc = STAGE ? 10u : 6u;
    if (lane == 0) mbar_expect_tx(B.bar, 7u * ep * 4u + nc * 256u + 272u + it.lp * 2u);
    __syncwarp();
    if (lane < 7u) {
        if (ep != 0u) {
            const void *src;
            void *dst;
            switch (lane) {
                case 0: src = m.sub_cl; dst = B.cl; break;
                case 1: src = m.sub_cr; dst = B.cr; break;
                case 2: src = m.sub_nx; dst = B.nx; break;
                case 3: src = m.sub_ny; dst = B.ny; break;
                case 4: src = m.sub_len; dst = B.len; break;
                case 5: src = m.sub_dzl; dst = B.dzl; break;
                default: src = m.sub_dzr; dst = B.dzr; break;
            }
            bulk_load(dst, static_cast<const char *>(src) + 4ull * it.e0, ep * 4u, B.bar);
        }
    } else if (lane < 7u + nc) {
        const uint32_t k = lane - 7u;
        const float *src;
        switch (k) {
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
        bulk_load(B.c + k * kTileCells, src + c0, 256u, B.bar);
    } else if (lane == 7u + nc) {
        bulk_load(B.cptr, m.cptr + c0, 272u, B.bar);
    } else if (lane == 8u + nc && it.lp != 0u) {
        bulk_load(B.lcsr, m.sub_lcsr + it.l0, it.lp * 2u, B.bar);
    }
}

template <int STAGE, bool COMP, bool CLAMP>
__global__ void __launch_bounds__(kTileThreads, 8) stage_tiled_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl) {
    const uint32_t count = s.sched[kSchedItems];
    if (blockIdx.x >= count) return;
    constexpr uint32_t nc = STAGE ? 10u : 6u;
    const TilePlan L = tile_plan(m.max_sub_edges, m.max_sub_slots, nc);
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t red[kTileThreads / 32];
    __shared__ uint4 items[2];
    __shared__ uint32_t dts[2];
    const uint4 *work = reinterpret_cast<const uint4 *>(s.items);
    const uint32_t tid = threadIdx.x;
    uint64_t computed = 0;
    if (tid == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(smem), 1u);
        mbar_init(reinterpret_cast<uint64_t *>(smem) + 1, 1u);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid < 32u) {
        const uint4 v = work[blockIdx.x];
        const Item it = unpack(v);
        if (tid == 0) {
            items[0] = v;
            dts[0] = s.dt_buf[kDtWords * it.inst];
        }
        tile_issue<STAGE>(m, s, it, tile_buf(smem, L, 0));
    }

    uint32_t k = 0;
    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x, ++k) {
        const TileBuf B = tile_buf(smem, L, k & 1u);
        const uint32_t wn = w + gridDim.x;
        if (tid < 32u && wn < count) {
            const uint4 v = work[wn];
            const Item itn = unpack(v);
            if (tid == 0) {
                items[(k + 1u) & 1u] = v;
                dts[(k + 1u) & 1u] = s.dt_buf[kDtWords * itn.inst];
            }
            tile_issue<STAGE>(m, s, itn, tile_buf(smem, L, (k + 1u) & 1u));
        }
        const bool ok = mbar_wait(B.bar, (k >> 1) & 1u);
        if (!__syncthreads_and(ok)) {
            // The staged data never arrived: report it, give the copies in flight
            // one more bounded wait, stop.
            if (tid == 0) atomicOr(&s.ctrl->error, 1u);
            mbar_wait(B.bar, (k >> 1) & 1u);
            if (wn < count) mbar_wait(tile_buf(smem, L, (k + 1u) & 1u).bar, ((k + 1u) >> 1) & 1u);
            return;
        }
        const Item it = unpack(items[k & 1u]);
        const uint32_t dt_bits = dts[k & 1u];
        if (dt_bits != 0u) {
            const float dt = __uint_as_float(dt_bits);
            const uint32_t b = it.tile >> 2;
            if (STAGE == 0 && (it.tile & 3u) == 0u && tid == 0) s.blk[kBlkWords * b + kBlkWet] = 0u;
            const float *C0 = B.c, *C1 = B.c + kTileCells, *C2 = B.c + 2 * kTileCells;
            const int base = static_cast<int>(it.tile * kTileCells);

            // Edge fluxes, written in place over the consumed records.
            for (uint32_t j = tid; j < it.ne; j += kTileThreads) {
                const int cL = B.cl[j], cR = B.cr[j];
                const float nx = B.nx[j], ny = B.ny[j];
                float hL, huL, hvL, hR, huR, hvR;
                const uint32_t lL = static_cast<uint32_t>(cL - base);
                if (lL < static_cast<uint32_t>(kTileCells)) {
                    hL = C0[lL];
                    huL = C1[lL];
                    hvL = C2[lL];
                } else {
                    load_state<STAGE>(s, cL, hL, huL, hvL);
                }
                if (cR < 0) {
                    hR = hL;
                    wall_mirror(huL, hvL, nx, ny, huR, hvR);
                } else {
                    const uint32_t lR = static_cast<uint32_t>(cR - base);
                    if (lR < static_cast<uint32_t>(kTileCells)) {
                        hR = C0[lR];
                        huR = C1[lR];
                        hvR = C2[lR];
                    } else {
                        load_state<STAGE>(s, cR, hR, huR, hvR);
                    }
                }
                const bool live = !(hL < p.dry_tol && hR < p.dry_tol);
                B.cr[j] = live ? 1 : 0;
                if (!live) continue;
                float w0, w1, w2, w3, w4, w5;
                edge_words(p, cR, nx, ny, B.len[j], B.dzl[j], B.dzr[j], hL, huL, hvL, hR, huR, hvR, w0, w1, w2, w3,
                           w4, w5);
                B.nx[j] = w0;
                B.ny[j] = w1;
                B.len[j] = w2;
                B.dzl[j] = w3;
                B.dzr[j] = w4;
                if (STAGE == 1) B.cl[j] = __float_as_int(w5);
            }
            __syncthreads();

            bool wet = false;
            uint32_t bound = kNoBound;
            if (tid < it.cells) {
                float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
                const uint32_t k0 = B.cptr[tid] - B.cptr[0], k1 = B.cptr[tid + 1] - B.cptr[0];
                for (uint32_t q = k0; q < k1; ++q) {
                    const uint32_t v = B.lcsr[q];
                    const uint32_t j = v >> 1;
                    if (!B.cr[j]) continue;
                    if (v & 1u) {
                        sdh -= B.nx[j];
                        sdhu -= B.dzl[j];
                        sdhv -= B.dzr[j];
                    } else {
                        sdh += B.nx[j];
                        sdhu += B.ny[j];
                        sdhv += B.len[j];
                    }
                    if (STAGE == 1) lam += __int_as_float(B.cl[j]);
                }
                const float *c = B.c;
                update_cell<STAGE, COMP, CLAMP>(s, p, cfl, dt, base + tid, c[4 * kTileCells + tid],
                                                c[5 * kTileCells + tid], c[tid], c[kTileCells + tid],
                                                c[2 * kTileCells + tid], c[3 * kTileCells + tid],
                                                STAGE ? c[6 * kTileCells + tid] : 0.0f,
                                                STAGE ? c[7 * kTileCells + tid] : 0.0f,
                                                STAGE ? c[8 * kTileCells + tid] : 0.0f,
                                                STAGE ? c[9 * kTileCells + tid] : 0.0f, sdh, sdhu, sdhv, lam, wet,
                                                bound);
            }
            if (STAGE == 1) {
                const int any_wet = __syncthreads_or(wet);
                const uint32_t bmin = block_min_any(bound, red);
                if (tid == 0) {
                    if (any_wet) s.blk[kBlkWords * b + kBlkWet] = 1u;
                    if (bmin != kNoBound) atomicMin(&s.dt_buf[kDtWords * it.inst + 1], bmin);
                    computed += it.cells;
                }
            }
        }
        // This buffer is refilled by bulk copies two items on.
        fence_proxy_async();
        __syncthreads();
    }
    if (STAGE == 1 && tid == 0 && computed)
        atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed), computed);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
template <int STAGE, bool COMP, bool CLAMP>
int launch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st,
                 float *sums = nullptr) {
    const Phys ph{p->g, p->dry_tol};
    if (p->kernel == 1u || sums) {
        auto kern = stage_block_kernel<STAGE, COMP, CLAMP>;
        const size_t bytes = block_smem_bytes(m->max_tile_edges);
        int rc = set_smem(kern, bytes);
        if (rc) return rc;
        const uint32_t grid = (p->grid == 0u || p->grid > m->n_blocks) ? m->n_blocks : p->grid;
        kern<<<grid, kThreads, bytes, st>>>(*m, *s, ph, p->cfl, sums);
        return check_launch();
    }
    auto kern = stage_tiled_kernel<STAGE, COMP, CLAMP>;
    const size_t bytes = tile_plan(m->max_sub_edges, m->max_sub_slots, STAGE ? 10u : 6u).total;
    int rc = set_smem(kern, bytes);
    if (rc) return rc;
    kern<<<p->grid ? p->grid : 148u * 8u, kTileThreads, bytes, st>>>(*m, *s, ph, p->cfl);
    return check_launch();
}

template <int STAGE>
int dispatch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st,
                   float *sums = nullptr) {
    if (p->compensated) {
        return p->track_clamp ? launch_stage<STAGE, true, true>(m, s, p, st, sums)
                              : launch_stage<STAGE, true, false>(m, s, p, st, sums);
    }
    return p->track_clamp ? launch_stage<STAGE, false, true>(m, s, p, st, sums)
                          : launch_stage<STAGE, false, false>(m, s, p, st, sums);
}

template <int STAGE, bool COMP, bool CLAMP>
int configure_stage(const swe_mesh_t *m) {
    int rc = set_smem(stage_block_kernel<STAGE, COMP, CLAMP>, block_smem_bytes(m->max_tile_edges));
    if (rc) return rc;
    return set_smem(stage_tiled_kernel<STAGE, COMP, CLAMP>, tile_plan(m->max_sub_edges, m->max_sub_slots, STAGE ? 10u : 6u).total);
}

}  // namespace swe

using namespace swe;

extern "C" {

int swe_configure(const swe_mesh_t *mesh, int kernel, int *blocks_per_sm) {
    if (!mesh_ok(mesh) || !blocks_per_sm || kernel < 0 || kernel > 1) return SWE_ERR_ARGUMENT;
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
    cudaError_t err;
    if (kernel == 0) {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            blocks_per_sm, stage_tiled_kernel<1, true, false>, kTileThreads,
            tile_plan(mesh->max_sub_edges, mesh->max_sub_slots, 10u).total);
    } else {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, stage_block_kernel<1, true, false>, kThreads,
                                                            block_smem_bytes(mesh->max_tile_edges));
    }
    return err == cudaSuccess ? SWE_OK : SWE_ERR_CUDA;
}

int swe_stage(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || params->kernel > 1u) return SWE_ERR_ARGUMENT;
    if (stage == 0) return dispatch_stage<0>(mesh, state, params, stream);
    if (stage == 1) return dispatch_stage<1>(mesh, state, params, stream);
    return SWE_ERR_ARGUMENT;
}

int swe_stage_taped(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage,
                    float *sums, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || !sums) return SWE_ERR_ARGUMENT;
    if (stage == 0) return dispatch_stage<0>(mesh, state, params, stream, sums);
    if (stage == 1) return dispatch_stage<1>(mesh, state, params, stream, sums);
    return SWE_ERR_ARGUMENT;
}

}  // extern "C"
