// Sparse sources as device functions over a strided range of sources, shared
// by the source kernels and the persistent step kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "swe_common.cuh"

namespace swe {

// ---------------------------------------------------------------------------
// Sparse sources (resident.py:665-733): all increments, then the bounds.
// A source with a hydrograph adds hscale times the hydrograph's value at the
// start of its instance's step to its rate: t = now_ticks / 2^20 s rounded to
// float, piecewise linear between the knots, the end values outside them.
// (The reference's inflows are constant per phase; this is the product's own
// interpolation, restated by the oracle.)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float hydrograph_at(const swe_sources_t &src, uint32_t j, float t) {
    const uint32_t k0 = src.knot_ptr[j], k1 = src.knot_ptr[j + 1];
    if (k1 <= k0) return 0.0f;
    if (!(t > src.knot_t[k0])) return src.knot_q[k0];
    if (!(t < src.knot_t[k1 - 1])) return src.knot_q[k1 - 1];
    uint32_t k = k0;
    while (k + 2 < k1 && !(t < src.knot_t[k + 1])) ++k;
    const float t0 = src.knot_t[k], t1 = src.knot_t[k + 1];
    const float q0 = src.knot_q[k], q1 = src.knot_q[k + 1];
    return q0 + (q1 - q0) * ((t - t0) / (t1 - t0));
}

__device__ __forceinline__ float clock_seconds(const swe_ctrl_t *c) {
    return static_cast<float>(c->now_ticks) * (1.0f / kTicksPerSecond);
}

__device__ __forceinline__ void source_apply(const swe_mesh_t &m, const swe_state_t &s, const swe_sources_t &src,
                                             float dry_tol, int comp, uint32_t first, uint32_t stride) {
    for (uint32_t k = first; k < src.count; k += stride) {
        const uint32_t i = src.cells[k];
        const uint32_t inst = m.block_inst[i >> 8];
        const uint32_t dt_bits = s.dt_buf[kDtWords * inst];
        if (dt_bits == 0u) continue;
        const float dt = __uint_as_float(dt_bits);
        float rate = src.rate[k];
        if (src.hydro && src.hydro[k] != 0xFFFFFFFFu)
            rate = rate + src.hscale[k] * hydrograph_at(src, src.hydro[k], clock_seconds(s.ctrl + inst));
        const float inc = dt * rate;
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

// One instance's CFL bound from a warp: every lane's (inst, bound), kNoBound for
// none. A warp whose bounds all belong to one instance sends one atomic minimum;
// otherwise every lane sends its own. Called by all 32 lanes.
__device__ __forceinline__ void bound_flush_warp(const swe_state_t &s, uint32_t inst, uint32_t bound) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const bool has = bound != kNoBound;
    const unsigned with = __ballot_sync(kFull, has);
    if (!with) return;
    const int leader = __ffs(with) - 1;
    const uint32_t ref = __shfl_sync(kFull, inst, leader);
    if (__all_sync(kFull, !has || inst == ref)) {
        const uint32_t low = __reduce_min_sync(kFull, bound);
        if (static_cast<int>(threadIdx.x & 31u) == leader) atomicMin(&s.dt_buf[kDtWords * ref + 1], low);
    } else if (has) {
        atomicMin(&s.dt_buf[kDtWords * inst + 1], bound);
    }
}

// The post-source CFL bounds: each thread keeps the minimum of its sources'
// bounds while they belong to one instance, and the warp combines them at the
// end, so the dt word sees few atomics however many sources there are (a
// minimum is the same in any order). Called by every thread of whole warps.
__device__ __forceinline__ void source_bound(const swe_mesh_t &m, const swe_state_t &s, const swe_sources_t &src,
                                             const Phys &p, float cfl, uint32_t first, uint32_t stride) {
    uint32_t acc_inst = 0u, acc = kNoBound;
    for (uint32_t k = first; k < src.count; k += stride) {
        const uint32_t i = src.cells[k];
        const uint32_t inst = m.block_inst[i >> 8];
        if (s.dt_buf[kDtWords * inst] == 0u) continue;
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
        if (!(lam > 1e-30f && A > 1e-10f)) continue;
        const uint32_t b = __float_as_uint(cfl * A / lam);
        if (inst != acc_inst && acc != kNoBound) {
            atomicMin(&s.dt_buf[kDtWords * acc_inst + 1], acc);
            acc = kNoBound;
        }
        acc_inst = inst;
        acc = min(acc, b);
    }
    bound_flush_warp(s, acc_inst, acc);
}

}  // namespace swe
