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

// Sticky seats. Each CTA of the launch has a seat: a tile it computes in every
// step for as long as the tile stays active, kept staged in its first buffer
// from step to step (edge records, local CSR, areas, roughness, block
// two-ring, and its state, which the CTA's own corrector wrote; restaged only
// after sources). Tiles without a seat wait in a queue: at the start of a
// launch every active tile (the block list), later the tiles of blocks that
// become active (pushed by the step that first marks them) and the tiles a
// CTA computed besides its seat (pushed back every step, except the first of
// them, which the CTA keeps and stages while its seat computes). CTAs without a seat
// take queued tiles first and seat the first one; a CTA with a seat takes more
// only after computing its seat, and streams those through its second buffer.
// A sparse step's critical path is then a few dependent global accesses (the
// neighbours' states, the two barriers; the seat's activity mark and its dt
// arrive while it computes its fluxes); a dense step spreads the queue over all
// CTAs.
//
// Step control: the last CTA to arrive at a step's final barrier runs it for
// every instance after the others have gone on, and publishes each instance's
// next dt beside that step's epoch as one 64-bit pair (dt words 2..3), which
// the next step's readers wait for (bounded) only where they need the dt.
//
// Activity: a block is active in step n if it was in the launch's start list
// (n = 0) or a wet or forced block of its two-ring marked it with the step's
// epoch E(n) = epoch0 + n + 1 during step n - 1. Marks are exchanged atomically, so
// the first marker of a block that was not active in step n learns that it is
// new and queues its tiles. The CTA that computes a block's first tile sets the
// block's active flag in the predictor phase, before any corrector reads it; a
// CTA that finds a tile of its seat or of the queue inactive clears it. At the
// end of a launch one pass turns the last marks into the flags, block list and
// tile work items the other kernels and the host read.
constexpr uint32_t kExtraCap = 512;  // tiles a CTA computes besides its seat in one step
constexpr uint32_t kRingCache = 96;  // blocks of the seat's two-ring kept in shared memory
constexpr uint32_t kNoTile = 0xFFFFFFFFu;

struct SeatShared {
    uint4 extra[kExtraCap];  // this step's other tiles (their work items)
    uint32_t extra_dt[kExtraCap];
    uint32_t n_extra;
    uint32_t seat;            // the seated tile (kNoTile: none)
    uint32_t staged;          // the tile whose records buffer 0 holds (kNoTile: none)
    uint32_t state_ok;        // buffer 0 holds that tile's current state
    uint4 seat_item;
    uint32_t seat_dt;
    uint32_t seat_active;     // the seat is computed in this step
    uint32_t seat_forced;
    uint32_t ring_n;
    uint32_t ring[kRingCache];
    uint32_t ring_active[kRingCache / 32];  // ring blocks active in this step
    uint32_t ring_ok;         // ring_active holds this step's bits for the seat
    uint32_t qlen;            // tiles queued for this step
    uint32_t take;            // a taken tile (kNoTile: the queue is empty)
    uint4 take_item;
    uint32_t take_dt;
    uint32_t kept;            // the other tile this CTA computed last step, kept for this one (kNoTile: none)
    uint4 kept_item;
    uint32_t kept_ring_block; // the block whose two-ring kept_ring holds (kNoTile: none)
    uint32_t kept_ring_n;
    uint32_t kept_forced;
    uint32_t kept_bits_step;  // step + 1 of the step kept_ring_active describes (0: none)
    uint32_t kept_ring[kRingCache];
    uint32_t kept_ring_active[kRingCache / 32];
};

__device__ __forceinline__ uint4 tile_item(const swe_mesh_t &m, uint32_t t, uint32_t inst) {
    const uint32_t b = t >> 2, q = t & 3u;
    const uint32_t cells = min(static_cast<uint32_t>(kTileCells), m.block_cells[b] - q * kTileCells);
    const uint32_t l0 = m.sub_lcsr_ptr[t];
    return make_item(t, cells, m.sub_ptr[t], l0, m.sub_count[t], m.sub_lcsr_ptr[t + 1] - l0, inst);
}

// The queue of tiles for steps of parity `par` (tile ids; 4 n_blocks each, in the
// second half of the work-item buffer).
__device__ __forceinline__ uint32_t *tile_queue(const swe_mesh_t &m, const swe_state_t &s, uint32_t par) {
    return s.items + 16u * m.n_blocks + par * 4u * m.n_blocks;
}

// Mark block b and its two-ring active for the step of epoch `next` (one warp);
// a block whose old mark is neither `next` nor `cur` (not active now) becomes
// active: its tiles join the next step's queue (parity qpar). ring: the cached
// two-ring, or nullptr to read it from global memory; active: bits of ring
// blocks known to be active now (and block b is), which need no exchange.
__device__ __forceinline__ void mark_ring(const swe_mesh_t &m, const swe_state_t &s, uint32_t b, uint32_t cur,
                                          uint32_t next, uint32_t qpar, const uint32_t *ring, uint32_t ring_n,
                                          const uint32_t *active = nullptr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t k0 = ring ? 0u : m.ring_ptr[b];
    const uint32_t n = ring ? ring_n : m.ring_ptr[b + 1] - k0;
    uint32_t *q = tile_queue(m, s, qpar);
    for (uint32_t k = lane; k <= n; k += 32u) {
        const uint32_t nb = k == 0u ? b : (ring ? ring[k - 1u] : m.ring_idx[k0 + k - 1u]);
        if (active && (k == 0u || ((active[(k - 1u) >> 5] >> ((k - 1u) & 31u)) & 1u))) {
            s.marks[2u * nb] = next;  // active now: no tiles to queue
            continue;
        }
        const uint32_t old = atomicExch(&s.marks[2u * nb], next);
        if (old != next && old != cur) {
            const uint32_t n_tiles = (m.block_cells[nb] + kTileCells - 1u) / kTileCells;
            const uint32_t pos = atomicAdd(&s.sched[kSchedQProd + qpar], n_tiles);
            for (uint32_t t = 0; t < n_tiles; ++t) q[pos + t] = 4u * nb + t;
        }
    }
}

// The same from one thread (sources).
__device__ __forceinline__ void mark_ring_thread(const swe_mesh_t &m, const swe_state_t &s, uint32_t b, uint32_t cur,
                                                 uint32_t next, uint32_t qpar) {
    uint32_t *q = tile_queue(m, s, qpar);
    for (uint32_t k = m.ring_ptr[b], k1 = m.ring_ptr[b + 1]; k <= k1; ++k) {
        const uint32_t nb = k == k1 ? b : m.ring_idx[k];
        const uint32_t old = atomicExch(&s.marks[2u * nb], next);
        if (old != next && old != cur) {
            const uint32_t n_tiles = (m.block_cells[nb] + kTileCells - 1u) / kTileCells;
            const uint32_t pos = atomicAdd(&s.sched[kSchedQProd + qpar], n_tiles);
            for (uint32_t t = 0; t < n_tiles; ++t) q[pos + t] = 4u * nb + t;
        }
    }
}

// Stage the tile of `item` into buffer k (warp 0): everything, or its state only.
template <int STAGE>
__device__ __forceinline__ void seat_issue(const swe_mesh_t &m, const swe_state_t &s, const uint4 item, const TileBuf &B,
                                           bool state_only) {
    const uint32_t lane = threadIdx.x & 31u;
    if (!state_only) {
        tile_issue<STAGE>(m, s, unpack(item), B);
        return;
    }
    const uint32_t c0 = unpack(item).tile * kTileCells;
    if (lane == 0) mbar_expect_tx(B.bar, 4u * 256u);
    __syncwarp();
    if (lane < 4u) {
        const float *src = lane == 0 ? s.h : lane == 1 ? s.hu : lane == 2 ? s.hv : s.h_lo;
        bulk_load(B.c + lane * kTileCells, src + c0, 256u, B.bar);
    }
}

// Wait for buffer k's staged data; on a timeout report error 1 and give the copy
// one more bounded wait. All threads; returns false on the timeout.
__device__ __forceinline__ bool seat_wait(const swe_state_t &s, const TileBuf &B, uint32_t *ph, uint32_t k) {
    const bool ok = mbar_wait(B.bar, ph[k]);
    ph[k] ^= 1u;
    if (__syncthreads_and(ok)) return true;
    if (threadIdx.x == 0) atomicOr(&s.ctrl->error, 1u);
    mbar_wait(B.bar, ph[k]);
    return false;
}

// The dt of instance `inst` in step `step` of epoch `epoch`: from the second step
// of a launch on it is the published pair's (the step control runs after the
// grid's release).
__device__ __forceinline__ uint32_t step_dt(const swe_state_t &s, uint32_t inst, uint32_t step, uint32_t epoch) {
    if (step == 0u) return s.dt_buf[kDtWords * inst];
    const uint64_t *pair = dt_pair(s, inst);
    return published_dt(s, pair, epoch, ld_relaxed_u64(pair));
}

// Take the next tile of this step's queue (thread 0 takes, all threads see it in
// ss.take / take_item / take_dt): skipped are tiles of instances that do not run
// this step and, from the second step on, tiles whose block is no longer active
// (pushed back by the CTA that computed them; their block's flag is cleared).
// In the first step a taken tile's block gets the step's mark.
__device__ __forceinline__ void seat_take(const swe_mesh_t &m, const swe_state_t &s, SeatShared &ss, uint32_t step,
                                          uint32_t epoch, bool all_active) {
    if (threadIdx.x == 0) {
        uint32_t got = kNoTile;
        for (; ss.qlen != 0u;) {  // an empty queue needs no round trip to find so
            uint32_t *taken = step == 0u ? &s.sched[kSchedStartTaken] : &s.sched[kSchedQCons + (step & 1u)];
            const uint32_t idx = atomicAdd(taken, 1u);
            if (idx >= ss.qlen) break;
            const uint32_t t = step == 0u ? unpack(reinterpret_cast<const uint4 *>(s.items)[idx]).tile
                                          : tile_queue(m, s, step & 1u)[idx];
            const uint32_t b = t >> 2, inst = m.block_inst[b];
            const uint32_t dt = step_dt(s, inst, step, epoch);
            if (dt == 0u) continue;  // a no-op step keeps the block's flags
            const bool active = step == 0u || all_active || s.marks[2u * b] == epoch;
            const uint32_t flag = s.blk[kBlkWords * b + kBlkActive];
            if (!active) {
                if ((t & 3u) == 0u && flag != 0u) s.blk[kBlkWords * b + kBlkActive] = 0u;
                continue;
            }
            if (step == 0u) s.marks[2u * b] = epoch;
            if ((t & 3u) == 0u && flag == 0u) s.blk[kBlkWords * b + kBlkActive] = 1u;
            got = t;
            ss.take_item = tile_item(m, t, inst);
            ss.take_dt = dt;
            break;
        }
        ss.take = got;
    }
    __syncthreads();
}

// The predictor of this CTA's tiles in step `step`: its seat if still active,
// then tiles of the queue (the first one seated when the CTA has no seat).
template <bool COMP, bool CLAMP, bool OPEN>
__device__ bool seat_predictor(const swe_mesh_t &m, const swe_state_t &s, const Phys &p, float cfl,
                               unsigned char *smem, TiledShared<kPersistThreads> &sh, SeatShared &ss, uint32_t *ph,
                               uint64_t &computed, uint32_t step, uint32_t epoch, bool all_active, bool sources) {
    const TilePlan L = tile_plan(m.max_sub_edges, m.max_sub_slots, 10u);
    float *F = reinterpret_cast<float *>(smem + L.total);
    const TileBuf B0 = tile_buf(smem, L, 0u), B1 = tile_buf(smem, L, 1u);
    const uint32_t tid = threadIdx.x;
    const uint32_t kept = ss.kept;
    bool kept_issued = false;
    if (!OPEN && step > 0u && ss.seat != kNoTile) {
        // The seat's predictor starts before its activity and dt are known: both arrive
        // while its fluxes are computed (the update of an inactive seat keeps nothing
        // anyone reads). An open mesh's tallies need dt in the flux loop: no early start.
        const Item it = unpack(ss.seat_item);
        const uint32_t b = ss.seat >> 2;
        if (!ss.state_ok || sources) {
            if (tid < 32u) seat_issue<0>(m, s, ss.seat_item, B0, true);
            if (!seat_wait(s, B0, ph, 0u)) return false;
        }
        // the queue's length (final since the last barrier) arrives with them
        const LateDt late{dt_pair(s, it.inst), s.marks + 2u * b, s.sched + kSchedQProd + (step & 1u), epoch,
                          all_active ? 1u : 0u, sh.late};
        // the kept tile's records and state are staged while the seat computes
        kept_issued = kept != kNoTile;
        if (kept_issued && tid < 32u) seat_issue<0>(m, s, ss.kept_item, B1, false);
        tile_compute<0, COMP, CLAMP, kPersistThreads, OPEN>(m, s, p, cfl, B0, it, 0.0f, 0u, 6u, F, L.capE, sh.red,
                                                            computed, true, nullptr, &late);
        fence_proxy_async();
        if (tid == 0) {
            ss.n_extra = 0u;
            ss.qlen = sh.late[2];
            const uint32_t dt = sh.late[1];
            ss.seat_active = sh.late[0] != 0u ? 1u : 0u;
            ss.seat_dt = sh.late[0];
            if (dt != 0u && !ss.seat_active) {
                if ((ss.seat & 3u) == 0u) s.blk[kBlkWords * b + kBlkActive] = 0u;
                ss.seat = kNoTile;  // free for a queued tile; the records stay staged
                ss.state_ok = 0u;   // another CTA may compute the tile before it returns here
            }
        }
        __syncthreads();
    } else if (tid == 0) {
        ss.n_extra = 0u;
        ss.qlen = step == 0u ? *reinterpret_cast<volatile uint32_t *>(s.sched + kSchedItems)
                             : *reinterpret_cast<volatile uint32_t *>(s.sched + kSchedQProd + (step & 1u));
        ss.seat_active = 0u;
        if (ss.seat != kNoTile) {
            const uint32_t b = ss.seat >> 2;
            const uint32_t dt = step_dt(s, unpack(ss.seat_item).inst, step, epoch);
            const bool active = all_active || s.marks[2u * b] == epoch;
            if (dt != 0u && active) {
                ss.seat_active = 1u;
                ss.seat_dt = dt;
            } else {
                if (dt != 0u && (ss.seat & 3u) == 0u) s.blk[kBlkWords * b + kBlkActive] = 0u;
                if (dt != 0u) {
                    ss.seat = kNoTile;  // free for a queued tile; the records stay staged
                    ss.state_ok = 0u;   // another CTA may compute the tile before it returns here
                }
            }
        }
    }
    __syncthreads();
    if (OPEN && ss.seat_active) {
        if (!ss.state_ok || sources) {
            if (tid < 32u) seat_issue<0>(m, s, ss.seat_item, B0, true);
            if (!seat_wait(s, B0, ph, 0u)) return false;
        }
        tile_compute<0, COMP, CLAMP, kPersistThreads, OPEN>(m, s, p, cfl, B0, unpack(ss.seat_item),
                                                            __uint_as_float(ss.seat_dt), 0u, 6u, F, L.capE, sh.red,
                                                            computed, true);
        fence_proxy_async();
        __syncthreads();
    }
    // A seat active from the start of the step keeps its tile all step: which blocks
    // of its two-ring are active now (read beside the first take). A tile seated
    // later has no such bits.
    const bool ring_ok = !OPEN && !all_active && ss.seat_active && ss.ring_n <= kRingCache;
    if (tid == 0) ss.ring_ok = ring_ok ? 1u : 0u;
    if (ring_ok && tid >= 32u && tid < 64u) {
        const uint32_t lane = tid & 31u;
        for (uint32_t w = 0; w * 32u < ss.ring_n; ++w) {
            const uint32_t k = w * 32u + lane;
            const bool act = k < ss.ring_n && s.marks[2u * ss.ring[k]] == epoch;
            const uint32_t bits = __ballot_sync(0xFFFFFFFFu, act);
            if (lane == 0) ss.ring_active[w] = bits;
        }
    }
    // The kept tile first (it is in no queue): computed when it is still active this step,
    // dropped otherwise, with the block flag handled as for a tile taken from the queue.
    if (kept != kNoTile) {
        if (!kept_issued && tid < 32u) seat_issue<0>(m, s, ss.kept_item, B1, false);
        if (tid == 0) {
            const Item ki = unpack(ss.kept_item);
            const uint32_t b = ki.tile >> 2;
            const uint32_t dt = step_dt(s, ki.inst, step, epoch);
            const bool active = all_active || s.marks[2u * b] == epoch;
            const uint32_t flag = s.blk[kBlkWords * b + kBlkActive];
            bool use = false;
            if (dt != 0u) {  // a no-op step keeps the block's flags
                if ((ki.tile & 3u) == 0u && flag != (active ? 1u : 0u)) s.blk[kBlkWords * b + kBlkActive] = active;
                use = active;
            }
            ss.take = use ? ki.tile : kNoTile;
            ss.take_dt = dt;
            ss.kept = kNoTile;
            if (use) {
                ss.extra[ss.n_extra] = ss.kept_item;
                ss.extra_dt[ss.n_extra] = dt;
                ss.n_extra += 1u;
            }
        }
        if (!OPEN && !all_active && tid >= 64u && tid < 96u) {
            // warp 2: the kept tile's block two-ring (read once while the tile stays kept) and
            // which of its blocks are active now, for its corrector's marks as the seat has them
            const uint32_t lane = tid & 31u, b = unpack(ss.kept_item).tile >> 2;
            if (ss.kept_ring_block != b) {
                const uint32_t k0 = m.ring_ptr[b], rn = m.ring_ptr[b + 1] - k0;
                if (rn <= kRingCache)
                    for (uint32_t r = lane; r < rn; r += 32u) ss.kept_ring[r] = m.ring_idx[k0 + r];
                if (lane == 0) {
                    ss.kept_ring_n = rn;
                    ss.kept_forced = s.blk[kBlkWords * b + kBlkForced];
                }
                __syncwarp();
                if (lane == 0) ss.kept_ring_block = b;
            }
            __syncwarp();
            const uint32_t rn = ss.kept_ring_n;
            if (rn <= kRingCache) {
                for (uint32_t w = 0; w * 32u < rn; ++w) {
                    const uint32_t k = w * 32u + lane;
                    const bool act = k < rn && s.marks[2u * ss.kept_ring[k]] == epoch;
                    const uint32_t bits = __ballot_sync(0xFFFFFFFFu, act);
                    if (lane == 0) ss.kept_ring_active[w] = bits;
                }
                if (lane == 0) ss.kept_bits_step = step + 1u;
            }
        }
        if (!seat_wait(s, B1, ph, 1u)) return false;
        if (ss.take != kNoTile) {
            tile_compute<0, COMP, CLAMP, kPersistThreads, OPEN>(m, s, p, cfl, B1, unpack(ss.kept_item),
                                                                __uint_as_float(ss.take_dt), 0u, 6u, F, L.capE,
                                                                sh.red, computed, false);
            fence_proxy_async();
        }
        __syncthreads();
    }
    for (;;) {
        if (ss.seat != kNoTile && ss.n_extra >= kExtraCap) break;
        seat_take(m, s, ss, step, epoch, all_active);
        // every thread reads what decides its path before thread 0 changes it
        const uint32_t t = ss.take;
        const bool seat_free = ss.seat == kNoTile, restage = ss.staged == t;
        __syncthreads();
        if (t == kNoTile) break;
        if (seat_free) {
            // seat it: its records may still be staged from an earlier seat
            if (tid == 0) {
                ss.seat = t;
                ss.seat_item = ss.take_item;
                ss.seat_dt = ss.take_dt;
                ss.seat_active = 1u;
                ss.staged = t;
                ss.state_ok = 1u;
            }
            if (tid < 32u) seat_issue<0>(m, s, ss.take_item, B0, restage);
            if (!restage && tid >= 32u && tid < 64u) {
                // warp 1: the seat's two-ring and forced flag, while the records arrive
                const uint32_t b = t >> 2, lane = tid & 31u;
                const uint32_t k0 = m.ring_ptr[b], rn = m.ring_ptr[b + 1] - k0;
                if (lane == 0) {
                    ss.ring_n = rn;
                    ss.seat_forced = s.blk[kBlkWords * b + kBlkForced];
                }
                if (rn <= kRingCache)
                    for (uint32_t r = lane; r < rn; r += 32u) ss.ring[r] = m.ring_idx[k0 + r];
            }
            if (!seat_wait(s, B0, ph, 0u)) return false;
            tile_compute<0, COMP, CLAMP, kPersistThreads, OPEN>(m, s, p, cfl, B0, unpack(ss.seat_item),
                                                                __uint_as_float(ss.seat_dt), 0u, 6u, F, L.capE, sh.red,
                                                                computed, true);
        } else {
            if (tid == 0) {
                ss.extra[ss.n_extra] = ss.take_item;
                ss.extra_dt[ss.n_extra] = ss.take_dt;
                ss.n_extra += 1u;
            }
            if (tid < 32u) seat_issue<0>(m, s, ss.take_item, B1, false);
            if (!seat_wait(s, B1, ph, 1u)) return false;
            tile_compute<0, COMP, CLAMP, kPersistThreads, OPEN>(m, s, p, cfl, B1, unpack(ss.take_item),
                                                                __uint_as_float(ss.take_dt), 0u, 6u, F, L.capE, sh.red,
                                                                computed, false);
        }
        fence_proxy_async();
        __syncthreads();
    }
    return true;
}

// The corrector of this CTA's tiles: the seat from its kept predictor state (its
// new state stays in buffer 0), the other tiles restaged through buffer 1 and
// pushed back into the next step's queue. Wet or forced tiles mark their
// block's two-ring for the next step.
template <bool COMP, bool CLAMP, bool OPEN>
__device__ bool seat_corrector(const swe_mesh_t &m, const swe_state_t &s, const Phys &p, float cfl,
                               unsigned char *smem, TiledShared<kPersistThreads> &sh, SeatShared &ss, uint32_t *ph,
                               uint64_t &computed, uint32_t step, uint32_t epoch, bool all_active) {
    const TilePlan L = tile_plan(m.max_sub_edges, m.max_sub_slots, 10u);
    float *F = reinterpret_cast<float *>(smem + L.total);
    const TileBuf B0 = tile_buf(smem, L, 0u), B1 = tile_buf(smem, L, 1u);
    const uint32_t tid = threadIdx.x, next = epoch + 1u, qpar = (step + 1u) & 1u;
    const uint32_t n = ss.n_extra;
    // the first other tile's restaging flies while the seat computes (buffer 1 is free)
    if (n && tid < 32u) seat_issue<1>(m, s, ss.extra[0], B1, false);
    if (ss.seat_active) {
        const Item it = unpack(ss.seat_item);
        const bool wet = tile_compute<1, COMP, CLAMP, kPersistThreads, OPEN>(
            m, s, p, cfl, B0, it, __uint_as_float(ss.seat_dt), 6u, 0u, F, L.capE, sh.red, computed, true);
        if (!all_active && tid < 32u && (wet || ss.seat_forced != 0u)) {
            const bool cached = ss.ring_n <= kRingCache;
            mark_ring(m, s, it.tile >> 2, epoch, next, qpar, cached ? ss.ring : nullptr, ss.ring_n,
                      ss.ring_ok ? ss.ring_active : nullptr);
        }
        fence_proxy_async();
        __syncthreads();
    }
    for (uint32_t w = 0; w < n; ++w) {
        if (w > 0u && tid < 32u) seat_issue<1>(m, s, ss.extra[w], B1, false);
        if (!seat_wait(s, B1, ph, 1u)) return false;
        const Item it = unpack(ss.extra[w]);
        const bool wet = tile_compute<1, COMP, CLAMP, kPersistThreads, OPEN>(
            m, s, p, cfl, B1, it, __uint_as_float(ss.extra_dt[w]), 0u, 6u, F, L.capE, sh.red, computed, false);
        // the kept tile's block has its two-ring and this step's active bits cached
        const uint32_t eb = it.tile >> 2;
        const bool cached = ss.kept_ring_block == eb && ss.kept_bits_step == step + 1u && ss.kept_ring_n <= kRingCache;
        if (!all_active && tid < 32u && (wet || (cached ? ss.kept_forced : s.blk[kBlkWords * eb + kBlkForced]) != 0u))
            mark_ring(m, s, eb, epoch, next, qpar, cached ? ss.kept_ring : nullptr, ss.kept_ring_n,
                      cached ? ss.kept_ring_active : nullptr);
        fence_proxy_async();
        __syncthreads();
    }
    // The first other tile stays with this CTA for the next step (checked for activity
    // then); the rest wait in the next step's queue again (checked when taken).
    if (n && tid == 0) {
        ss.kept = unpack(ss.extra[0]).tile;
        ss.kept_item = ss.extra[0];
    }
    if (n > 1u) {
        uint32_t *q = tile_queue(m, s, qpar);
        if (tid == 0) ss.qlen = atomicAdd(&s.sched[kSchedQProd + qpar], n - 1u);
        __syncthreads();
        for (uint32_t w = tid; w + 1u < n; w += blockDim.x) q[ss.qlen + w] = unpack(ss.extra[w + 1u]).tile;
    }
    return true;
}

// The end of a launch: active flags, block list and tile work items of the next
// step from the last marks (what the dilation would have built), for the other
// kernels and the host. Instances that will not run keep their flags, unlisted.
__device__ __forceinline__ void seat_handover(const swe_mesh_t &m, const swe_state_t &s, uint32_t epoch,
                                              bool all_active) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t base = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); base * 32u < m.n_blocks;
         base += warps) {
        const uint32_t b = base * 32u + lane;
        bool listed = false;
        if (b < m.n_blocks && s.dt_buf[kDtWords * m.block_inst[b]] != 0u) {
            listed = all_active || s.marks[2u * b] == epoch;
            s.blk[kBlkWords * b + kBlkActive] = listed ? 1u : 0u;
        }
        const uint32_t mask = __ballot_sync(0xFFFFFFFFu, listed);
        if (!mask) continue;
        const uint32_t cells = listed ? m.block_cells[b] : 0u;
        const uint32_t n_items = (cells + kTileCells - 1u) / kTileCells;
        uint32_t before = n_items;
        for (int d = 1; d < 32; d <<= 1) {  // inclusive scan of the tile counts
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, before, d);
            if (lane >= static_cast<uint32_t>(d)) before += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, before, 31);
        before -= n_items;
        uint32_t pos0 = 0u, ipos0 = 0u;
        if (lane == 0) {
            pos0 = atomicAdd(&s.sched[kSchedActive], __popc(mask));
            ipos0 = atomicAdd(&s.sched[kSchedItems], total);
        }
        pos0 = __shfl_sync(0xFFFFFFFFu, pos0, 0);
        ipos0 = __shfl_sync(0xFFFFFFFFu, ipos0, 0);
        if (listed) {
            s.active_list[pos0 + __popc(mask & ((1u << lane) - 1u))] = b;
            uint4 *items = reinterpret_cast<uint4 *>(s.items);
            const uint32_t inst = m.block_inst[b];
            for (uint32_t q = 0; q < n_items; ++q) items[ipos0 + before + q] = tile_item(m, 4u * b + q, inst);
        }
    }
}

template <bool COMP, bool CLAMP, bool OPEN>
__global__ void __launch_bounds__(kPersistThreads, 1024 / kPersistThreads)
    persistent_steps_kernel(swe_mesh_t m, swe_state_t s, swe_sources_t src, Phys p, float cfl, int all_active,
                            uint32_t n_steps) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ TiledShared<kPersistThreads> sh;
    __shared__ SeatShared ss;
    __shared__ int flag[2];
    __shared__ uint32_t epoch0;
    CountSync g{s.sync, 0u};  // the launch zeroes the counter before the kernel starts
    if (threadIdx.x == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(smem), 1u);
        mbar_init(reinterpret_cast<uint64_t *>(smem) + 1, 1u);
        fence_barrier_init();
        epoch0 = *reinterpret_cast<volatile uint32_t *>(s.sched + kSchedEpoch);  // before any CTA's first barrier
        ss.seat = ss.staged = ss.kept = ss.kept_ring_block = kNoTile;
        ss.kept_bits_step = 0u;
        ss.state_ok = 0u;
        if (blockIdx.x == 0) {  // the queues of this launch start empty (first used after the first barrier)
            for (int k = 0; k < 2; ++k) {
                s.sched[kSchedQProd + k] = 0u;
                s.sched[kSchedQCons + k] = 0u;
            }
        }
    }
    if (blockIdx.x == 0)  // no published dt pair of an earlier run or launch carries an epoch of this one
        for (uint32_t i = threadIdx.x; i < m.n_inst; i += blockDim.x)
            *const_cast<uint64_t *>(dt_pair(s, i)) = 0ull;
    __syncthreads();
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const bool all = all_active != 0;
    auto nothing = [] {};
    uint32_t ph[2] = {0u, 0u};
    uint64_t computed = 0;
    bool ok = true;
    uint32_t step = 0;
    for (; step < n_steps; ++step) {
        // E(n) = epoch0 + n + 1: never the zero the prologue leaves in the marks, never a value
        // of an earlier launch (each leaves its last E(n) + 1 in the epoch word)
        const uint32_t epoch = epoch0 + step + 1u, next_epoch = epoch + 1u;
        if (!(ok = seat_predictor<COMP, CLAMP, OPEN>(m, s, p, cfl, smem, sh, ss, ph, computed, step, epoch, all,
                                                      src.count != 0u)))
            break;
        if (!(ok = count_sync(g, flag, nothing))) break;
        if (!(ok = seat_corrector<COMP, CLAMP, OPEN>(m, s, p, cfl, smem, sh, ss, ph, computed, step, epoch, all)))
            break;
        if (src.count) {
            if (!(ok = count_sync(g, flag, nothing))) break;
            source_apply(m, s, src, p.dry_tol, COMP ? 1 : 0, first, stride);
            if (!(ok = count_sync(g, flag, nothing))) break;
            source_bound(m, s, src, p, cfl, first, stride);
            if (!all) {  // a source that wets its block marks the block's two-ring
                for (uint32_t q = first; q < src.count; q += stride) {
                    const uint32_t b = src.cells[q] >> 8;
                    if (s.blk[kBlkWords * b + kBlkWet] != 0u && s.dt_buf[kDtWords * m.block_inst[b]] != 0u)
                        mark_ring_thread(m, s, b, epoch, next_epoch, (step + 1u) & 1u);
                }
            }
        }
        const bool last_step = step + 1u == n_steps;
        auto control = [&] {
            for (uint32_t i = threadIdx.x; i < m.n_inst; i += blockDim.x) {
                const uint32_t dt = step_control(s.ctrl + i, s.dt_buf + kDtWords * i, 1);
                // readers use the pair's own 64 bits only: no release ordering to wait for
                st_relaxed_u64(const_cast<uint64_t *>(dt_pair(s, i)), (static_cast<uint64_t>(next_epoch) << 32) | dt);
            }
            if (threadIdx.x == blockDim.x - 1u) {  // beside instance 0's control, not after it
                volatile uint32_t *sched = s.sched;
                sched[kSchedEpoch] = next_epoch;
                if (step == 0u) sched[kSchedStartTaken] = 0u;
                // this step's queue is used up: it takes the tiles of the step after next
                sched[kSchedQProd + (step & 1u)] = 0u;
                sched[kSchedQCons + (step & 1u)] = 0u;
                if (last_step) {  // the hand-over lists are counted from zero
                    sched[kSchedActive] = 0u;
                    sched[kSchedItems] = 0u;
                    sched[kSchedNext] = 0u;
                    sched[kSchedNextItems] = 0u;
                    sched[kSchedStartTaken] = 0u;
                }
            }
        };
        // The step control runs after the release, the others wait for its dt pairs
        // only where they need them.
        if (!(ok = count_sync(g, flag, control))) break;
        // the hand-over reads the last step's dt and the lists its control zeroes
        if (last_step && !(ok = count_sync(g, flag, nothing))) break;
    }
    if (ok && step > 0u) seat_handover(m, s, epoch0 + step + 1u, all);
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
    // every tile of a step must find a CTA: one seat and kExtraCap others each
    if (4ull * m->n_blocks > static_cast<uint64_t>(grid) * (1u + kExtraCap)) return SWE_ERR_TOO_LARGE;
    // the barrier's arrival counter (at most four barriers a step, one more at the end) stays below 2^32
    if ((4ull * n_steps + 1ull) * grid >= (1ull << 32)) return SWE_ERR_TOO_LARGE;
    Phys ph{p->g, p->dry_tol};
    float cfl = p->cfl;
    int all_active = p->active_set ? 0 : 1;
    swe_mesh_t mm = *m;
    swe_state_t ss = *s;
    swe_sources_t sc = *src;
    void *args[] = {&mm, &ss, &sc, &ph, &cfl, &all_active, &n_steps};
    // the grid barrier's arrival counter starts from zero in every launch
    if (cudaMemsetAsync(s->sync, 0, sizeof(uint32_t), st) != cudaSuccess) return SWE_ERR_CUDA;
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
    if (!mesh_ok(mesh) || !state_ok(state) || !open_ok(mesh, state) || !params || !sources || params->kernel > 3u)
        return SWE_ERR_ARGUMENT;
    if (n_steps == 0u) return SWE_OK;
    if (params->kernel != 2u) {
        for (uint32_t k = 0; k < n_steps; ++k) {
            const int rc = swe_step(mesh, state, params, sources, stream);
            if (rc) return rc;
        }
        return SWE_OK;
    }
    if (!state->sync || !state->marks || (reinterpret_cast<uintptr_t>(state->dt_buf) & 15u)) return SWE_ERR_ARGUMENT;
    if (mesh->max_sub_edges > 2047u || mesh->max_sub_slots > 2047u || mesh->n_inst > 1023u) return SWE_ERR_TOO_LARGE;
    if (sources->count && (!sources->cells || !sources->rate)) return SWE_ERR_ARGUMENT;
    return mesh->n_open ? dispatch_persistent<true>(mesh, state, params, sources, n_steps, stream)
                        : dispatch_persistent<false>(mesh, state, params, sources, n_steps, stream);
}
