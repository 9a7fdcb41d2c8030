// B200 kernels of the inundation shallow-water step and their C ABI.
//
// Layout: cells in Hilbert order, 256-cell blocks; each block's edges are a
// contiguous tile (its own edges, then the edges it shares with a left cell
// in another block) so one CTA computes every flux its cells need into shared
// memory, gathers them in the reference's fixed per-cell CSR order and
// updates the cells, with no per-edge buffer in HBM and no float atomics.
// An edge shared by two blocks is computed by both, from the same inputs by
// the same instructions, so both see the same bits.
//
// Reference: inundation/vulkan/shaders/resident.py (GLSL) driven by
// inundation/vulkan/gpu_resident_batch.py; the per-function comments give
// the lines each kernel replaces.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "../../include/inundation_b200.h"
#include "swe_math.cuh"

namespace swe {

constexpr int kBlockCells = 256;
constexpr int kThreads = 256;
constexpr uint32_t kBlkWords = 3, kBlkWet = 0, kBlkActive = 1, kBlkForced = 2;
constexpr uint32_t kNoBound = 0xFFFFFFFFu;

// sched words
constexpr int kSchedActive = 0;    // blocks in active_list for the current step
constexpr int kSchedNext = 1;      // append counter of the dilation
constexpr int kSchedDone = 2;      // CTAs of the dilation that finished
constexpr int kSchedCells = 3;     // cells in the current active blocks
constexpr int kSchedNextCells = 4; // cells appended by the dilation
constexpr int kSchedComputed = 6;  // [6,7]: uint64 cells computed over real steps

__device__ __forceinline__ bool block_active(const uint32_t *blk, uint32_t b) {
    return blk[kBlkWords * b + kBlkActive] != 0u;
}

// The stage's input state of cell c: the predictor in the corrector, except
// in an inactive block, whose predictor is stale (resident.py:209-226).
template <int STAGE>
__device__ __forceinline__ void load_state(const swe_state_t &s, int c, float &h, float &hu, float &hv) {
    if (STAGE == 1 && block_active(s.blk, static_cast<uint32_t>(c) >> 8)) {
        h = s.h1[c];
        hu = s.hu1[c];
        hv = s.hv1[c];
    } else {
        h = s.h[c];
        hu = s.hu[c];
        hv = s.hv[c];
    }
}

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

__device__ __forceinline__ uint32_t block_min_u32(uint32_t v, uint32_t *scratch) {
    v = __reduce_min_sync(0xFFFFFFFFu, v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < (kThreads >> 5)) ? scratch[lane] : kNoBound;
        w = __reduce_min_sync(0xFFFFFFFFu, w);
        if (lane == 0) scratch[0] = w;
    }
    __syncthreads();
    const uint32_t r = scratch[0];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// One Heun stage over the active blocks (flux_resident_gather +
// update_resident_gather[_comp], resident.py:187-291, 312-344, 354-513).
// ---------------------------------------------------------------------------
template <int STAGE, bool COMP, bool CLAMP>
__global__ void __launch_bounds__(kThreads) stage_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl) {
    const uint32_t dt_bits = s.dt_buf[0];
    if (dt_bits == 0u) return;  // the window is done: a no-op step
    const float dt = __uint_as_float(dt_bits);
    const uint32_t cap = (m.max_tile_edges + 3u) & ~3u;
    const TileSmem t = tile_smem(cap);
    __shared__ uint32_t red[kThreads / 32];
    const uint32_t count = s.sched[kSchedActive];

    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        const uint32_t b = s.active_list[w];
        const uint32_t base = m.tile_ptr[b], ne = m.tile_count[b];

        // Edge fluxes of the tile (resident.py:241-284).
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
            const float len = m.tile_len[e], dzL = m.tile_dzl[e], dzR = m.tile_dzr[e];
            float hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, smax;
            face_states(p, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx, ny, hLs, hqnL, hqtL, hRs, hqnR, hqtR);
            hllc(p, hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, smax);
            if (cR < 0) Fh = 0.0f;  // a wall passes no mass
            const float Fhu = Fhn * nx - Fht * ny;
            const float Fhv = Fhn * ny + Fht * nx;
            const float SL_g = 0.5f * p.g * (hL * hL - hLs * hLs);
            const float SR_g = 0.5f * p.g * (hR * hR - hRs * hRs);
            t.F0[j] = Fh * len;
            t.L1[j] = Fhu * len + SL_g * nx * len;
            t.L2[j] = Fhv * len + SL_g * ny * len;
            t.R1[j] = Fhu * len + SR_g * nx * len;
            t.R2[j] = Fhv * len + SR_g * ny * len;
            if (STAGE == 1) t.C[j] = smax * len;
        }
        __syncthreads();

        const uint32_t i = b * kBlockCells + threadIdx.x;
        bool wet = false;
        uint32_t bound = kNoBound;
        if (i < m.n_cells) {
            const float A = m.area[i];
            const float dti = dt / A;
            float hi, hui, hvi;
            if (STAGE == 0) {
                hi = s.h[i];
                hui = s.hu[i];
                hvi = s.hv[i];
            } else {
                hi = s.h1[i];
                hui = s.hu1[i];
                hvi = s.hv1[i];
            }
            // Fixed-order gather; a dry-dry edge was not computed and adds nothing.
            float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
            const uint32_t k0 = m.cptr[i], k1 = m.cptr[i + 1];
            for (uint32_t k = k0; k < k1; ++k) {
                const uint32_t v = m.lcsr[k];
                const uint32_t j = v >> 1;
                if (!t.live[j]) continue;
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
            float h_new, lo_new, h_raw;
            if (COMP) {
                const float loi = (STAGE == 0) ? s.h_lo[i] : s.h1_lo[i];
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
                const float n = m.n_mann[i];
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
            } else {
                float hf;
                if (COMP) {
                    float sm, em, lof;
                    two_sum(s.h[i], h_new, sm, em);
                    em += s.h_lo[i] + lo_new;
                    two_sum(0.5f * sm, 0.5f * em, hf, lof);
                    s.h_lo[i] = lof;
                } else {
                    hf = 0.5f * (s.h[i] + h_new);
                }
                s.h[i] = hf;
                float huf = 0.5f * (s.hu[i] + hu_new);
                float hvf = 0.5f * (s.hv[i] + hv_new);
                if (hf < p.dry_tol) {
                    huf = 0.0f;
                    hvf = 0.0f;
                }
                s.hu[i] = huf;
                s.hv[i] = hvf;
                wet = hf >= p.dry_tol;
                if (lam > 1e-30f && A > 1e-10f) bound = __float_as_uint(cfl * A / lam);
            }
        }
        if (STAGE == 1) {
            // The block's wet mark and its share of the next step's CFL bound.
            const int any_wet = __syncthreads_or(wet);
            const uint32_t bmin = block_min_u32(bound, red);
            if (threadIdx.x == 0) {
                s.blk[kBlkWords * b + kBlkWet] = any_wet ? 1u : 0u;
                if (bmin != kNoBound) atomicMin(&s.dt_buf[1], bmin);
            }
        } else {
            __syncthreads();
        }
    }
}


// ---------------------------------------------------------------------------
// Bulk copies (TMA, 1-D, no multicast) into shared memory, completed on an
// mbarrier; every wait is bounded by a deadline on the global timer.
// ---------------------------------------------------------------------------
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s
constexpr int kStageThreads = 512;

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
__device__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity)) {
        if (global_ns() - t0 > kWaitLimitNs) return false;
    }
    return true;
}

// Shared-memory plan of the staged stage kernel: two buffers, each holding a
// block's tile (7 arrays of capE), its cell data (nc arrays of 256), its
// cptr window (260 words) and its local CSR (capS halfwords), then the
// per-cell velocities of the block being computed.
struct StagePlan {
    uint32_t capE, capS, nc, buf_bytes, off_vel, total;
};

__host__ __device__ inline StagePlan stage_plan(uint32_t max_tile_edges, uint32_t max_block_slots, uint32_t nc) {
    StagePlan L;
    L.capE = (max_tile_edges + 31u) & ~31u;
    L.capS = (max_block_slots + 63u) & ~63u;
    L.nc = nc;
    L.buf_bytes = 7u * L.capE * 4u + nc * 1024u + 1152u + L.capS * 2u;
    L.off_vel = 128u + 2u * L.buf_bytes;
    L.total = L.off_vel + 2u * 256u * 4u;
    return L;
}

struct StageBuf {
    int32_t *cl, *cr;
    float *nx, *ny, *len, *dzl, *dzr;
    float *c;          // nc x 256: [0..3] the stage's input state, [4] area, [5] n, [6..9] committed state (stage 1)
    uint32_t *cptr;    // 260
    uint16_t *lcsr;    // capS
    uint64_t *bar;
};

__device__ __forceinline__ StageBuf stage_buf(unsigned char *smem, const StagePlan &L, uint32_t k) {
    unsigned char *base = smem + 128u + k * L.buf_bytes;
    StageBuf B;
    const uint32_t e = L.capE * 4u;
    B.cl = reinterpret_cast<int32_t *>(base);
    B.cr = reinterpret_cast<int32_t *>(base + e);
    B.nx = reinterpret_cast<float *>(base + 2u * e);
    B.ny = reinterpret_cast<float *>(base + 3u * e);
    B.len = reinterpret_cast<float *>(base + 4u * e);
    B.dzl = reinterpret_cast<float *>(base + 5u * e);
    B.dzr = reinterpret_cast<float *>(base + 6u * e);
    B.c = reinterpret_cast<float *>(base + 7u * e);
    B.cptr = reinterpret_cast<uint32_t *>(base + 7u * e + L.nc * 1024u);
    B.lcsr = reinterpret_cast<uint16_t *>(base + 7u * e + L.nc * 1024u + 1152u);
    B.bar = reinterpret_cast<uint64_t *>(smem) + k;
    return B;
}

// Warp 0 stages block b into buffer B: one bulk copy per lane.
template <int STAGE>
__device__ void stage_issue(const swe_mesh_t &m, const swe_state_t &s, uint32_t b, const StageBuf &B) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t e0 = m.tile_ptr[b], ep = m.tile_ptr[b + 1] - e0;
    const uint32_t l0 = m.lcsr_ptr[b], lp = m.lcsr_ptr[b + 1] - l0;
    const uint32_t c0 = b * kBlockCells;
    constexpr uint32_t nc = STAGE ? 10u : 6u;
    if (lane == 0) mbar_expect_tx(B.bar, 7u * ep * 4u + nc * 1024u + 1040u + lp * 2u);
    __syncwarp();
    if (lane < 7u) {
        const void *src;
        void *dst;
        switch (lane) {
            case 0: src = m.tile_cl; dst = B.cl; break;
            case 1: src = m.tile_cr; dst = B.cr; break;
            case 2: src = m.tile_nx; dst = B.nx; break;
            case 3: src = m.tile_ny; dst = B.ny; break;
            case 4: src = m.tile_len; dst = B.len; break;
            case 5: src = m.tile_dzl; dst = B.dzl; break;
            default: src = m.tile_dzr; dst = B.dzr; break;
        }
        bulk_load(dst, static_cast<const char *>(src) + 4ull * e0, ep * 4u, B.bar);
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
        bulk_load(B.c + k * 256u, src + c0, 1024u, B.bar);
    } else if (lane == 7u + nc) {
        bulk_load(B.cptr, m.cptr + c0, 1040u, B.bar);
    } else if (lane == 8u + nc && lp != 0u) {
        bulk_load(B.lcsr, m.lcsr_blk + l0, lp * 2u, B.bar);
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

// HLLC with the face-frame velocities of the reconstructed states, written
// without divergent branches: the star state of the side the contact wave
// leaves behind is formed once. Same expressions as hllc(), bit for bit.
__device__ __forceinline__ void hllc_select(const Phys &p, float hL, float hqnL, float hqtL, float hR, float hqnR,
                                            float hqtR, float &Fh, float &Fhn, float &Fht, float &smax) {
    const float unL = safe_vel(p, hL, hqnL), utL = safe_vel(p, hL, hqtL);
    const float unR = safe_vel(p, hR, hqnR), utR = safe_vel(p, hR, hqtR);
    float SL, SR;
    hllc_speeds_fast(p, hL, unL, hR, unR, SL, SR);
    smax = gmax(fabsf(SL), fabsf(SR));
    const float num_sm = SL * hR * (unR - SR) - SR * hL * (unL - SL);
    const float den_sm = hR * (unR - SR) - hL * (unL - SL);
    const float SM = (fabsf(den_sm) > 1e-12f) ? num_sm / den_sm : 0.0f;
    const float FLh = hL * unL, FLn = hL * unL * unL + 0.5f * p.g * hL * hL, FLt = hL * unL * utL;
    const float FRh = hR * unR, FRn = hR * unR * unR + 0.5f * p.g * hR * hR, FRt = hR * unR * utR;
    const bool left = SM >= 0.0f;
    const float hK = left ? hL : hR, unK = left ? unL : unR, utK = left ? utL : utR, SK = left ? SL : SR;
    const float FKh = left ? FLh : FRh, FKn = left ? FLn : FRn, FKt = left ? FLt : FRt;
    const float dSK = SK - SM;
    const float kK = hK * (SK - unK) / ((fabsf(dSK) > 1e-14f) ? dSK : 1e-14f);
    const float Fsh = FKh + SK * (kK - hK);
    const float Fsn = FKn + SK * (kK * SM - hK * unK);
    const float Fst = FKt + SK * (kK * utK - hK * utK);
    const bool useL = SL >= 0.0f, useR = !useL && !left && !(SR >= 0.0f);
    Fh = useL ? FLh : (useR ? FRh : Fsh);
    Fhn = useL ? FLn : (useR ? FRn : Fsn);
    Fht = useL ? FLt : (useR ? FRt : Fst);
}

// ---------------------------------------------------------------------------
// One Heun stage over the active blocks, staged: each CTA prefetches its next
// block (tile, cell data, cptr window, local CSR) with bulk copies while it
// computes the current one. Same arithmetic as stage_kernel, bit for bit.
// ---------------------------------------------------------------------------
template <int STAGE, bool COMP, bool CLAMP>
__global__ void __launch_bounds__(kStageThreads, 2) stage_staged_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl) {
    const uint32_t dt_bits = s.dt_buf[0];
    if (dt_bits == 0u) return;
    const uint32_t count = s.sched[kSchedActive];
    if (blockIdx.x >= count) return;
    const float dt = __uint_as_float(dt_bits);
    constexpr uint32_t nc = STAGE ? 10u : 6u;
    const StagePlan L = stage_plan(m.max_tile_edges, m.max_block_slots, nc);
    extern __shared__ __align__(128) unsigned char smem[];
    float *su = reinterpret_cast<float *>(smem + L.off_vel);
    float *sv = su + 256;
    __shared__ uint32_t red[kStageThreads / 32];
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(smem), 1u);
        mbar_init(reinterpret_cast<uint64_t *>(smem) + 1, 1u);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid < 32u) stage_issue<STAGE>(m, s, s.active_list[blockIdx.x], stage_buf(smem, L, 0));

    uint32_t it = 0;
    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x, ++it) {
        const uint32_t b = s.active_list[w];
        const StageBuf B = stage_buf(smem, L, it & 1u);
        const uint32_t wn = w + gridDim.x;
        if (tid < 32u && wn < count) stage_issue<STAGE>(m, s, s.active_list[wn], stage_buf(smem, L, (it + 1u) & 1u));
        const bool ok = mbar_wait(B.bar, (it >> 1) & 1u);
        if (!__syncthreads_and(ok)) {
            // The staged data never arrived: report it, let any prefetch land, stop.
            if (tid == 0) atomicOr(&s.ctrl->error, 1u);
            if (wn < count) mbar_wait(stage_buf(smem, L, (it + 1u) & 1u).bar, ((it + 1u) >> 1) & 1u);
            return;
        }
        const float *C0 = B.c, *C1 = B.c + 256, *C2 = B.c + 512;
        const int base = static_cast<int>(b * kBlockCells);
        if (tid < 256u) {
            su[tid] = safe_vel(p, C0[tid], C1[tid]);
            sv[tid] = safe_vel(p, C0[tid], C2[tid]);
        }
        __syncthreads();

        // Edge fluxes of the tile, written in place over the consumed records.
        const uint32_t ne = m.tile_count[b];
        for (uint32_t j = tid; j < ne; j += kStageThreads) {
            const int cL = B.cl[j], cR = B.cr[j];
            const float nx = B.nx[j], ny = B.ny[j];
            float hL, huL, hvL, uL, vL, hR, huR, hvR, uR, vR;
            const uint32_t lL = static_cast<uint32_t>(cL - base);
            if (lL < 256u) {
                hL = C0[lL]; huL = C1[lL]; hvL = C2[lL]; uL = su[lL]; vL = sv[lL];
            } else {
                load_state<STAGE>(s, cL, hL, huL, hvL);
                uL = safe_vel(p, hL, huL);
                vL = safe_vel(p, hL, hvL);
            }
            if (cR < 0) {
                hR = hL;
                wall_mirror(huL, hvL, nx, ny, huR, hvR);
                uR = safe_vel(p, hR, huR);
                vR = safe_vel(p, hR, hvR);
            } else {
                const uint32_t lR = static_cast<uint32_t>(cR - base);
                if (lR < 256u) {
                    hR = C0[lR]; huR = C1[lR]; hvR = C2[lR]; uR = su[lR]; vR = sv[lR];
                } else {
                    load_state<STAGE>(s, cR, hR, huR, hvR);
                    uR = safe_vel(p, hR, huR);
                    vR = safe_vel(p, hR, hvR);
                }
            }
            const bool live = !(hL < p.dry_tol && hR < p.dry_tol);
            B.cr[j] = live ? 1 : 0;
            if (!live) continue;
            const float len = B.len[j], dzL = B.dzl[j], dzR = B.dzr[j];
            const float hLs = gmax(0.0f, hL - dzL), hRs = gmax(0.0f, hR - dzR);
            const float huLs = hLs * uL, hvLs = hLs * vL, huRs = hRs * uR, hvRs = hRs * vR;
            const float hqnL = huLs * nx + hvLs * ny, hqtL = -huLs * ny + hvLs * nx;
            const float hqnR = huRs * nx + hvRs * ny, hqtR = -huRs * ny + hvRs * nx;
            float Fh, Fhn, Fht, smax;
            hllc_select(p, hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, smax);
            if (cR < 0) Fh = 0.0f;  // a wall passes no mass
            const float Fhu = Fhn * nx - Fht * ny;
            const float Fhv = Fhn * ny + Fht * nx;
            const float SL_g = 0.5f * p.g * (hL * hL - hLs * hLs);
            const float SR_g = 0.5f * p.g * (hR * hR - hRs * hRs);
            B.nx[j] = Fh * len;
            B.ny[j] = Fhu * len + SL_g * nx * len;
            B.len[j] = Fhv * len + SL_g * ny * len;
            B.dzl[j] = Fhu * len + SR_g * nx * len;
            B.dzr[j] = Fhv * len + SR_g * ny * len;
            if (STAGE == 1) B.cl[j] = __float_as_int(smax * len);
        }
        __syncthreads();

        const uint32_t i = b * kBlockCells + tid;
        bool wet = false;
        uint32_t bound = kNoBound;
        if (tid < 256u && i < m.n_cells) {
            const float A = B.c[4 * 256 + tid];
            const float dti = dt / A;
            const float hi = C0[tid], hui = C1[tid], hvi = C2[tid];
            float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
            const uint32_t k0 = B.cptr[tid] - B.cptr[0], k1 = B.cptr[tid + 1] - B.cptr[0];
            for (uint32_t k = k0; k < k1; ++k) {
                const uint32_t v = B.lcsr[k];
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
            float h_new, lo_new, h_raw;
            if (COMP) {
                const float loi = B.c[3 * 256 + tid];
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
                const float n = B.c[5 * 256 + tid];
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
            } else {
                const float h0 = B.c[6 * 256 + tid], hu0 = B.c[7 * 256 + tid], hv0 = B.c[8 * 256 + tid];
                float hf;
                if (COMP) {
                    float sm, em, lof;
                    two_sum(h0, h_new, sm, em);
                    em += B.c[9 * 256 + tid] + lo_new;
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
        }
        if (STAGE == 1) {
            const int any_wet = __syncthreads_or(wet);
            const uint32_t bmin = block_min_any(bound, red);
            if (tid == 0) {
                s.blk[kBlkWords * b + kBlkWet] = any_wet ? 1u : 0u;
                if (bmin != kNoBound) atomicMin(&s.dt_buf[1], bmin);
            }
        }
        // This buffer is refilled by bulk copies two iterations on.
        fence_proxy_async();
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Integer-tick step control (resident.py:813-885).
// ---------------------------------------------------------------------------
__device__ void step_control(swe_ctrl_t *c, uint32_t *dt_buf, int mode) {
    float raw;
    if (mode == 0) {
        raw = __uint_as_float(dt_buf[0]);
        c->last_raw = raw;
    } else if (mode == 1) {
        const uint32_t done = c->dt_ticks;
        c->now_ticks += static_cast<uint64_t>(done);
        if (done > 0u) {
            c->steps += 1u;
            raw = __uint_as_float(dt_buf[1]);
            c->last_raw = raw;
        } else {
            raw = c->last_raw;  // a no-op step computed no bound
        }
    } else {
        raw = c->last_raw;
    }
    const uint64_t remaining = (c->stop_ticks > c->now_ticks) ? c->stop_ticks - c->now_ticks : 0ull;
    uint32_t ticks;
    if (remaining == 0ull || raw < 1e-10f || raw != raw) {
        ticks = 0u;  // window done, or a degenerate bound: the host sees no progress
    } else if (raw >= 1e10f) {
        ticks = c->dry_dt_ticks;  // no wet edge anywhere
    } else {
        const float cap = static_cast<float>(c->dt_max_ticks) / kTicksPerSecond;
        ticks = static_cast<uint32_t>(gmin(raw * c->cfl_safety, cap) * kTicksPerSecond);
    }
    if (c->dt_max_ticks < ticks) ticks = c->dt_max_ticks;
    if (static_cast<uint64_t>(ticks) > remaining) ticks = static_cast<uint32_t>(remaining);
    c->dt_ticks = ticks;
    dt_buf[0] = __float_as_uint(static_cast<float>(ticks) / kTicksPerSecond);
    dt_buf[1] = __float_as_uint(kDtSentinel);
}

__global__ void step_control_kernel(swe_ctrl_t *c, uint32_t *dt_buf, int mode) { step_control(c, dt_buf, mode); }

// ---------------------------------------------------------------------------
// Dilation of the wet marks over each block's two-ring, compaction of the
// active blocks, then (last CTA) step control (resident.py:778-805, 813-885).
// One warp per block reads the block's two-ring in parallel; each CTA of
// kDilateWarps warps appends its active blocks with one atomic, in order.
// ---------------------------------------------------------------------------
constexpr int kDilateWarps = 32;

__global__ void __launch_bounds__(kDilateWarps * 32)
    dilate_compact_kernel(swe_mesh_t m, swe_state_t s, int all_active, int force, int control_mode) {
    const bool run = force || s.dt_buf[0] != 0u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * kDilateWarps + warp;
    __shared__ uint32_t flag[kDilateWarps];
    __shared__ bool last;
    if (run) {
        uint32_t v = 0u;
        if (b < m.n_blocks) {
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
        if (lane == 0) flag[warp] = v;
        __syncthreads();
        if (warp == 0) {
            const uint32_t blk = blockIdx.x * kDilateWarps + lane;
            const bool on = flag[lane] != 0u;
            const unsigned ballot = __ballot_sync(0xFFFFFFFFu, on);
            const uint32_t cells = on ? min(static_cast<uint32_t>(kBlockCells), m.n_cells - blk * kBlockCells) : 0u;
            const uint32_t total_cells = __reduce_add_sync(0xFFFFFFFFu, cells);
            uint32_t pos = 0;
            if (lane == 0 && ballot) {
                pos = atomicAdd(&s.sched[kSchedNext], static_cast<uint32_t>(__popc(ballot)));
                atomicAdd(&s.sched[kSchedNextCells], total_cells);
            }
            pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
            const uint32_t slot = pos + __popc(ballot & ((1u << lane) - 1u));
            if (on && slot < m.n_blocks) s.active_list[slot] = blk;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&s.sched[kSchedDone], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    volatile uint32_t *sched = s.sched;
    if (control_mode == 1 && s.dt_buf[0] != 0u) {
        // The step that just ran computed the blocks of the previous list.
        atomicAdd(reinterpret_cast<unsigned long long *>(s.sched + kSchedComputed),
                  static_cast<unsigned long long>(sched[kSchedCells]));
    }
    if (run) {
        sched[kSchedActive] = sched[kSchedNext];
        sched[kSchedCells] = sched[kSchedNextCells];
    }
    sched[kSchedNext] = 0u;
    sched[kSchedNextCells] = 0u;
    sched[kSchedDone] = 0u;
    if (control_mode >= 0) step_control(s.ctrl, s.dt_buf, control_mode);
}

// ---------------------------------------------------------------------------
// Start of a run: wet flag per block (resident.py:738-773).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) block_mark_kernel(swe_mesh_t m, swe_state_t s, float dry_tol, int all_active) {
    for (uint32_t b = blockIdx.x; b < m.n_blocks; b += gridDim.x) {
        const uint32_t i = b * kBlockCells + threadIdx.x;
        bool live = false;
        if (i < m.n_cells) live = s.h[i] >= dry_tol || s.hu[i] != 0.0f || s.hv[i] != 0.0f;
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

__global__ void dt_reset_kernel(uint32_t *dt_buf) { dt_buf[0] = __float_as_uint(kDtSentinel); }

// ---------------------------------------------------------------------------
// Prologue CFL bound over every block (cfl_edge_gather + cfl_gather,
// resident.py:528-610): every edge's wave term (0 if dry) into the tile,
// every cell sums all its slots, the minimum bound into dt_buf[0].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) cfl_prologue_kernel(swe_mesh_t m, swe_state_t s, Phys p, float cfl) {
    const uint32_t cap = (m.max_tile_edges + 3u) & ~3u;
    const TileSmem t = tile_smem(cap);
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
                hR = hL;
                wall_mirror(huL, hvL, nx, ny, huR, hvR);
            } else {
                hR = s.h[cR];
                huR = s.hu[cR];
                hvR = s.hv[cR];
            }
            float contrib = 0.0f;
            if (hL >= p.dry_tol || hR >= p.dry_tol)
                contrib = wave_bound(p, hL, huL, hvL, m.tile_dzl[e], hR, huR, hvR, m.tile_dzr[e], nx, ny) * m.tile_len[e];
            t.C[j] = contrib;
        }
        __syncthreads();
        const uint32_t i = b * kBlockCells + threadIdx.x;
        uint32_t bound = kNoBound;
        if (i < m.n_cells) {
            float lam = 0.0f;
            for (uint32_t k = m.cptr[i]; k < m.cptr[i + 1]; ++k) lam += t.C[m.lcsr[k] >> 1];
            const float A = m.area[i];
            if (lam > 1e-30f && A > 1e-10f) bound = __float_as_uint(cfl * A / lam);
        }
        const uint32_t bmin = block_min_u32(bound, red);
        if (threadIdx.x == 0 && bmin != kNoBound) atomicMin(&s.dt_buf[0], bmin);
    }
}

// ---------------------------------------------------------------------------
// Sparse sources (resident.py:665-733): all increments, then the bounds.
// ---------------------------------------------------------------------------
__global__ void source_apply_kernel(swe_state_t s, swe_sources_t src, float dry_tol, int comp) {
    const uint32_t dt_bits = s.dt_buf[0];
    if (dt_bits == 0u) return;
    const float dt = __uint_as_float(dt_bits);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < src.count; k += gridDim.x * blockDim.x) {
        const uint32_t i = src.cells[k];
        const float inc = dt * src.rate[k];
        float h_new;
        if (comp) {
            float lo_new;
            add_compensated(s.h[i], s.h_lo[i], inc, h_new, lo_new);
            s.h_lo[i] = lo_new;
        } else {
            h_new = gmax(s.h[i] + inc, 0.0f);
        }
        s.h[i] = h_new;
        if (h_new >= dry_tol) s.blk[kBlkWords * (i >> 8) + kBlkWet] = 1u;
    }
}

__global__ void source_bound_kernel(swe_mesh_t m, swe_state_t s, swe_sources_t src, Phys p, float cfl) {
    if (s.dt_buf[0] == 0u) return;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < src.count; k += gridDim.x * blockDim.x) {
        const uint32_t i = src.cells[k];
        const float h_new = s.h[i];
        if (!(h_new >= p.dry_tol)) continue;
        const float u = sqrtf(s.hu[i] * s.hu[i] + s.hv[i] * s.hv[i]) / h_new;
        const float c = sqrtf(p.g * h_new);
        const uint32_t base = m.tile_ptr[i >> 8];
        float lam = 0.0f;
        for (uint32_t q = m.cptr[i]; q < m.cptr[i + 1]; ++q) {
            const uint32_t v = m.lcsr[q];
            const uint32_t e = base + (v >> 1);
            const int nb = (v & 1u) ? m.tile_cl[e] : m.tile_cr[e];
            const bool dry_side = nb >= 0 && s.h[nb] < p.dry_tol;
            lam += (u + (dry_side ? 2.0f : 1.0f) * c) * m.tile_len[e];
        }
        const float A = m.area[i];
        if (lam > 1e-30f && A > 1e-10f) atomicMin(&s.dt_buf[1], __float_as_uint(cfl * A / lam));
    }
}

// ---------------------------------------------------------------------------
// Float64 volume, fixed order: per-CTA partials, then one CTA over them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
    volume_partial_kernel(const float *h, const float *h_lo, const float *area, uint32_t n, uint32_t per_cta, double *partials) {
    __shared__ double acc[kThreads];
    const uint32_t lo = blockIdx.x * per_cta;
    const uint32_t hi = min(n, lo + per_cta);
    double sum = 0.0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += kThreads)
        sum += (static_cast<double>(h[i]) + static_cast<double>(h_lo ? h_lo[i] : 0.0f)) * static_cast<double>(area[i]);
    acc[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) acc[threadIdx.x] += acc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

__global__ void __launch_bounds__(kThreads) volume_final_kernel(const double *partials, uint32_t count, double *out) {
    __shared__ double acc[kThreads];
    double sum = 0.0;
    for (uint32_t i = threadIdx.x; i < count; i += kThreads) sum += partials[i];
    acc[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) acc[threadIdx.x] += acc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = acc[0];
}

__global__ void eft_probe_kernel(float *v) {
    float se, ee;
    two_sum(v[0], v[1], se, ee);
    v[2] = ee;
}

__global__ void pow43_kernel(const float *x, float *out, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = pow43(x[i]);
}

// ---------------------------------------------------------------------------
// Host helpers.
// ---------------------------------------------------------------------------
inline size_t tile_smem_bytes(uint32_t max_tile_edges) {
    const size_t cap = (max_tile_edges + 3u) & ~3u;
    return cap * 6 * sizeof(float) + ((cap + 15) & ~size_t(15));
}

inline int check_launch() { return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ERR_CUDA; }

inline bool mesh_ok(const swe_mesh_t *m) {
    return m && m->n_cells && m->n_blocks && m->tile_cl && m->tile_cr && m->tile_nx && m->tile_ny && m->tile_len &&
           m->tile_dzl && m->tile_dzr && m->tile_ptr && m->tile_count && m->cptr && m->lcsr && m->area &&
           m->n_mann && m->ring_ptr && m->ring_idx && m->lcsr_blk && m->lcsr_ptr;
}

inline bool state_ok(const swe_state_t *s) {
    return s && s->h && s->hu && s->hv && s->h_lo && s->h1 && s->hu1 && s->hv1 && s->h1_lo && s->clamp_mass &&
           s->blk && s->active_list && s->sched && s->dt_buf && s->ctrl;
}

template <typename K>
int set_smem(K kernel, size_t bytes) {
    if (bytes > 227 * 1024) return SWE_ERR_TOO_LARGE;
    if (bytes > 48 * 1024 &&
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)) != cudaSuccess)
        return SWE_ERR_CUDA;
    return SWE_OK;
}

inline uint32_t grid_of(const swe_mesh_t *m, const swe_params_t *p) {
    return (p->grid == 0u || p->grid > m->n_blocks) ? m->n_blocks : p->grid;
}

template <int STAGE, bool COMP, bool CLAMP>
int launch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st) {
    if (p->kernel == 1u) {
        auto kern = stage_kernel<STAGE, COMP, CLAMP>;
        const size_t bytes = tile_smem_bytes(m->max_tile_edges);
        int rc = set_smem(kern, bytes);
        if (rc) return rc;
        kern<<<grid_of(m, p), kThreads, bytes, st>>>(*m, *s, Phys{p->g, p->dry_tol}, p->cfl);
        return check_launch();
    }
    auto kern = stage_staged_kernel<STAGE, COMP, CLAMP>;
    const size_t bytes = stage_plan(m->max_tile_edges, m->max_block_slots, STAGE ? 10u : 6u).total;
    int rc = set_smem(kern, bytes);
    if (rc) return rc;
    kern<<<grid_of(m, p), kStageThreads, bytes, st>>>(*m, *s, Phys{p->g, p->dry_tol}, p->cfl);
    return check_launch();
}

template <int STAGE, bool COMP, bool CLAMP>
int configure_stage(const swe_mesh_t *m) {
    int rc = set_smem(stage_kernel<STAGE, COMP, CLAMP>, tile_smem_bytes(m->max_tile_edges));
    if (rc) return rc;
    return set_smem(stage_staged_kernel<STAGE, COMP, CLAMP>,
                    stage_plan(m->max_tile_edges, m->max_block_slots, STAGE ? 10u : 6u).total);
}

template <int STAGE>
int dispatch_stage(const swe_mesh_t *m, const swe_state_t *s, const swe_params_t *p, cudaStream_t st) {
    if (p->compensated) {
        return p->track_clamp ? launch_stage<STAGE, true, true>(m, s, p, st) : launch_stage<STAGE, true, false>(m, s, p, st);
    }
    return p->track_clamp ? launch_stage<STAGE, false, true>(m, s, p, st) : launch_stage<STAGE, false, false>(m, s, p, st);
}

}  // namespace swe

using namespace swe;

extern "C" {

size_t swe_workspace_bytes(uint32_t n_cells) {
    const size_t blocks = (n_cells + kBlockCells - 1) / kBlockCells;
    return blocks * sizeof(uint32_t) + 8 * sizeof(uint32_t) + 4 * sizeof(uint32_t) + swe_volume_partials(n_cells) * sizeof(double) + 8;
}

size_t swe_tile_smem_bytes(uint32_t max_tile_edges) { return tile_smem_bytes(max_tile_edges); }

int swe_configure(const swe_mesh_t *mesh, int kernel, int *blocks_per_sm) {
    if (!mesh_ok(mesh) || !blocks_per_sm || kernel < 0 || kernel > 1) return SWE_ERR_ARGUMENT;
    int rc = configure_stage<0, false, false>(mesh);
    if (!rc) rc = configure_stage<0, false, true>(mesh);
    if (!rc) rc = configure_stage<0, true, false>(mesh);
    if (!rc) rc = configure_stage<0, true, true>(mesh);
    if (!rc) rc = configure_stage<1, false, false>(mesh);
    if (!rc) rc = configure_stage<1, false, true>(mesh);
    if (!rc) rc = configure_stage<1, true, false>(mesh);
    if (!rc) rc = configure_stage<1, true, true>(mesh);
    if (!rc) rc = set_smem(cfl_prologue_kernel, tile_smem_bytes(mesh->max_tile_edges));
    if (rc) return rc;
    cudaError_t err;
    if (kernel == 1) {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, stage_kernel<1, true, false>, kThreads,
                                                            tile_smem_bytes(mesh->max_tile_edges));
    } else {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            blocks_per_sm, stage_staged_kernel<1, true, false>, kStageThreads,
            stage_plan(mesh->max_tile_edges, mesh->max_block_slots, 10u).total);
    }
    return err == cudaSuccess ? SWE_OK : SWE_ERR_CUDA;
}

int swe_stage(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params) return SWE_ERR_ARGUMENT;
    if (stage == 0) return dispatch_stage<0>(mesh, state, params, stream);
    if (stage == 1) return dispatch_stage<1>(mesh, state, params, stream);
    return SWE_ERR_ARGUMENT;
}

int swe_apply_sources(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                      const swe_sources_t *sources, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || !sources) return SWE_ERR_ARGUMENT;
    if (sources->count == 0u) return SWE_OK;
    if (!sources->cells || !sources->rate) return SWE_ERR_ARGUMENT;
    const uint32_t grid = min((sources->count + kThreads - 1) / kThreads, 148u * 16u);
    source_apply_kernel<<<grid, kThreads, 0, stream>>>(*state, *sources, params->dry_tol, static_cast<int>(params->compensated));
    int rc = check_launch();
    if (rc) return rc;
    source_bound_kernel<<<grid, kThreads, 0, stream>>>(*mesh, *state, *sources, Phys{params->g, params->dry_tol}, params->cfl);
    return check_launch();
}

int swe_block_dilate_compact(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int force,
                             int control_mode, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !params || control_mode < -1 || control_mode > 2) return SWE_ERR_ARGUMENT;
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
    dt_reset_kernel<<<1, 1, 0, stream>>>(state->dt_buf);
    int rc = check_launch();
    if (rc) return rc;
    const size_t bytes = tile_smem_bytes(mesh->max_tile_edges);
    rc = set_smem(cfl_prologue_kernel, bytes);
    if (rc) return rc;
    cfl_prologue_kernel<<<grid_of(mesh, params), kThreads, bytes, stream>>>(*mesh, *state, Phys{params->g, params->dry_tol},
                                                                           params->cfl);
    return check_launch();
}

int swe_step_control(swe_ctrl_t *ctrl, uint32_t *dt_buf, int mode, swe_stream_t stream) {
    if (!ctrl || !dt_buf || mode < 0 || mode > 2) return SWE_ERR_ARGUMENT;
    step_control_kernel<<<1, 1, 0, stream>>>(ctrl, dt_buf, mode);
    return check_launch();
}

int swe_prologue(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, swe_stream_t stream) {
    int rc = swe_block_mark(mesh, state, params, stream);
    if (rc) return rc;
    rc = swe_block_dilate_compact(mesh, state, params, 1, -1, stream);
    if (rc) return rc;
    rc = swe_cfl_prologue(mesh, state, params, stream);
    if (rc) return rc;
    return swe_step_control(state->ctrl, state->dt_buf, 0, stream);
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

uint32_t swe_volume_partials(uint32_t n_cells) {
    const uint32_t p = (n_cells + 4095u) / 4096u;
    return p < 1u ? 1u : (p > 1024u ? 1024u : p);
}

int swe_volume_fp64(const float *h, const float *h_lo, const float *area, uint32_t n_cells, double *partials, double *out,
                    swe_stream_t stream) {
    if (!h || !area || !partials || !out || n_cells == 0u) return SWE_ERR_ARGUMENT;
    const uint32_t parts = swe_volume_partials(n_cells);
    const uint32_t per = (n_cells + parts - 1) / parts;
    volume_partial_kernel<<<parts, kThreads, 0, stream>>>(h, h_lo, area, n_cells, per, partials);
    int rc = check_launch();
    if (rc) return rc;
    volume_final_kernel<<<1, kThreads, 0, stream>>>(partials, parts, out);
    return check_launch();
}

int swe_eft_probe(float *v, swe_stream_t stream) {
    if (!v) return SWE_ERR_ARGUMENT;
    eft_probe_kernel<<<1, 1, 0, stream>>>(v);
    return check_launch();
}

int swe_pow43(const float *x, float *out, uint32_t n, swe_stream_t stream) {
    if (!x || !out || n == 0u) return SWE_ERR_ARGUMENT;
    pow43_kernel<<<min((n + 255u) / 256u, 4096u), 256, 0, stream>>>(x, out, n);
    return check_launch();
}

const char *swe_status_string(int status) {
    switch (status) {
        case SWE_OK: return "ok";
        case SWE_ERR_ARGUMENT: return "invalid argument";
        case SWE_ERR_CUDA: return "CUDA launch or runtime error";
        case SWE_ERR_TOO_LARGE:
            return "size beyond a fixed limit (an edge tile larger than shared memory, or more cells than the "
                   "allocation-free volume's static scratch holds)";
        case SWE_ERR_MATH: return "device arithmetic lost the two-sum error term";
        default: return "unknown status";
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free float64 volume.
//
// For callers that must not allocate device memory during a run: a host that
// runs under a fixed device-memory budget checked at start-up, an embedding
// application that owns the CUDA allocator, or code called from a context
// where cudaMalloc is not allowed. The per-CTA partial sums that
// swe_volume_fp64 takes from its caller live here in a static device array
// instead; every GPU that loads this library holds it (8 KiB) until exit.
// ---------------------------------------------------------------------------
namespace swe {

constexpr uint32_t kNoAllocPartials = 1024;
constexpr uint32_t kNoAllocCellsPerPartial = 4096;
constexpr uint32_t kNoAllocMaxCells = kNoAllocPartials * kNoAllocCellsPerPartial;
constexpr int kNoAllocDevices = 64;

static __device__ __align__(256) double g_volume_scratch[kNoAllocPartials];

// Device address of g_volume_scratch per device ordinal. In host code the
// array's name is only a host-side stand-in, never a device address.
static std::atomic<double *> g_volume_scratch_addr[kNoAllocDevices];

}  // namespace swe

extern "C" int swe_volume_fp64_noalloc(const float *h, const float *h_lo, const float *area, uint32_t n_cells,
                                       double *out, swe_stream_t stream) {
    if (!h || !area || !out || n_cells == 0u) return SWE_ERR_ARGUMENT;
    if (n_cells > kNoAllocMaxCells) return SWE_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return SWE_ERR_CUDA;
    if (dev < 0 || dev >= kNoAllocDevices) return SWE_ERR_ARGUMENT;
    double *scratch = g_volume_scratch_addr[dev].load(std::memory_order_acquire);
    if (scratch == nullptr) {
        // First call on this device (the device must be current): look up the
        // array's device address once and keep it.
        void *addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_volume_scratch) != cudaSuccess || addr == nullptr) return SWE_ERR_CUDA;
        scratch = static_cast<double *>(addr);
        g_volume_scratch_addr[dev].store(scratch, std::memory_order_release);
    }
    // Same partition as swe_volume_fp64 (one partial per 4096 cells below the
    // limit), so both entry points sum in the same order. Every partial the
    // final pass reads is rewritten first, so the array needs no clearing.
    const uint32_t parts = swe_volume_partials(n_cells);
    const uint32_t per = (n_cells + parts - 1) / parts;
    volume_partial_kernel<<<parts, kThreads, 0, stream>>>(h, h_lo, area, n_cells, per, scratch);
    int rc = check_launch();
    if (rc) return rc;
    volume_final_kernel<<<1, kThreads, 0, stream>>>(scratch, parts, out);
    return check_launch();
}
