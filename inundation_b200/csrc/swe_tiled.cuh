// Stage pieces shared by the stage kernels and the persistent step kernel:
// the per-cell Heun update, the per-edge gather words, and the 64-cell tile
// work items staged into shared memory by bulk copies.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "swe_common.cuh"

namespace swe {

// The gather words of a tile's edges in shared memory, laid out so that both
// cells of an edge add what they read: six arrays of `cap` words from P. The
// left cell of edge j adds (P[j], P[cap + j], P[2 cap + j]) = (w0, w1, w2) to
// its sums (sdh, sdhu, sdhv), the right cell (P[3 cap + j], P[4 cap + j],
// P[5 cap + j]) = (-w0, -w3, -w4): adding -w is subtracting w, bit for bit. An
// edge that is not computed (dry on both sides) holds -0.0 in all six, which
// leaves a sum unchanged (x + -0.0 == x for every x, +0.0 included, in
// round-to-nearest), so the gather needs no flag and no branch per slot and its
// sums have the bits of sums that skip such edges. The corrector's CFL word w5,
// which both cells add, sits at Lw[j] (-0.0 when not computed).
struct SideWords {
    float *P;
    float *Lw;
    uint32_t cap;
};

// Edge j's words: the computed ones when `live`, else -0.0 throughout.
template <int STAGE>
__device__ __forceinline__ void put_side_words(const SideWords &S, uint32_t j, bool live, float w0, float w1,
                                               float w2, float w3, float w4, float w5) {
    const float z = -0.0f;
    float *P = S.P + j;
    const uint32_t c = S.cap;
    P[0] = live ? w0 : z;
    P[c] = live ? w1 : z;
    P[2u * c] = live ? w2 : z;
    P[3u * c] = live ? -w0 : z;
    P[4u * c] = live ? -w3 : z;
    P[5u * c] = live ? -w4 : z;
    if (STAGE == 1) S.Lw[j] = live ? w5 : z;
}

// Adds the words of local-CSR slot v (edge v >> 1, side v & 1) to a cell's sums.
template <int STAGE>
__device__ __forceinline__ void add_side_words(const SideWords &S, uint32_t v, float &sdh, float &sdhu, float &sdhv,
                                               float &lam) {
    const float *w = S.P + ((v >> 1) + (v & 1u) * 3u * S.cap);
    sdh += w[0];
    sdhu += w[S.cap];
    sdhv += w[2u * S.cap];
    if (STAGE == 1) lam += S.Lw[v >> 1];
}

// The same words in arrays of their own (the persistent kernel, whose staged
// records stay from step to step): one float4 per local-CSR slot value
// v = 2j + side, (w0, w1, w2, w5) for the left cell of edge j and
// (-w0, -w3, -w4, w5) for the right, -0.0 throughout for an edge that is not
// computed. The sums are those of SideWords, bit for bit, from one 16-byte
// shared load per slot; F holds 8 words per record, 16-byte aligned.
template <int STAGE>
__device__ __forceinline__ void put_slot_words(float *F, uint32_t j, bool live, float w0, float w1, float w2,
                                               float w3, float w4, float w5) {
    const float z = -0.0f;
    float4 *P = reinterpret_cast<float4 *>(F) + 2u * j;
    const float c = (STAGE == 1 && live) ? w5 : z;
    P[0] = live ? make_float4(w0, w1, w2, c) : make_float4(z, z, z, z);
    P[1] = live ? make_float4(-w0, -w3, -w4, c) : make_float4(z, z, z, z);
}

template <int STAGE>
__device__ __forceinline__ void add_slot_words(const float *F, uint32_t v, float &sdh, float &sdhu, float &sdhv,
                                               float &lam) {
    const float4 w = reinterpret_cast<const float4 *>(F)[v];
    sdh += w.x;
    sdhu += w.y;
    sdhv += w.z;
    if (STAGE == 1) lam += w.w;
}

// The compensated Heun update of one cell from its gathered sums (resident.py:354-513).
// keep != nullptr: the new state also goes to shared memory at keep[0], keep[64],
// keep[128], keep[192] (h, hu, hv, h_lo): the predictor's, or the committed one.
template <int STAGE, bool COMP, bool CLAMP>
__device__ __forceinline__ void update_cell(const swe_state_t &s, const Phys &p, float cfl, float dt, uint32_t i,
                                            float A, float n, float hi, float hui, float hvi, float loi, float h0,
                                            float hu0, float hv0, float lo0, float sdh, float sdhu, float sdhv,
                                            float lam, bool &wet, uint32_t &bound, float *keep = nullptr) {
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
    float hu_new = fmaf_rn(-dti, sdhu, hui);
    float hv_new = fmaf_rn(-dti, sdhv, hvi);
    if (CLAMP) s.clamp_mass[i] += 0.5f * A * (h_new - h_raw);
    if (h_new < p.dry_tol) {
        hu_new = 0.0f;
        hv_new = 0.0f;
    }
    if (h_new >= p.dry_tol) {
        const float drag = film_drag(p, h_new, dt);
        hu_new *= drag;
        hv_new *= drag;
        const float inv_h = 1.0f / h_new;
        const float u_ = hu_new * inv_h, v_ = hv_new * inv_h;
        const float spd = sqrtf(fmaf_rn(u_, u_, v_ * v_));
        const float Sf = p.g * n * n * spd * inv_pow43(h_new);
        const float inv_den = 1.0f / fmaf_rn(dt, Sf, 1.0f);
        hu_new = hu_new * inv_den;
        hv_new = hv_new * inv_den;
    }
    if (STAGE == 0) {
        s.h1[i] = h_new;
        if (COMP) s.h1_lo[i] = lo_new;
        s.hu1[i] = hu_new;
        s.hv1[i] = hv_new;
        if (keep) {  // the predictor's state kept in shared memory, columns h, hu, hv, h_lo
            keep[0] = h_new;
            keep[kTileCells] = hu_new;
            keep[2 * kTileCells] = hv_new;
            keep[3 * kTileCells] = lo_new;
        }
        return;
    }
    float hf, lof = 0.0f;
    if (COMP) {
        float sm, em;
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
    if (keep) {
        keep[0] = hf;
        keep[kTileCells] = huf;
        keep[2 * kTileCells] = hvf;
        keep[3 * kTileCells] = lof;
    }
    wet = hf >= p.dry_tol;
    if (lam > 1e-30f && A > 1e-10f) bound = __float_as_uint(cfl * A / lam);
}

// The edge flux with the two sides of every symmetric step in the two lanes of a
// float2 (lane x the left side, lane y the right): Blackwell's paired float32
// instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn) round each lane exactly as
// the scalar operation would, so face_flux_pair gives the values of face_states +
// hllc (swe_math.cuh) bit for bit, in fewer instructions. A difference x - y is
// written x + (-y) or fma(-1, y, x), which round to the same value.
__device__ __forceinline__ float2 pr(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// safe_vel2 of both sides: the velocities of momenta q1, q2 at depth h, per lane.
__device__ __forceinline__ void safe_vel_pair(const Phys &p, float2 h, float2 q1, float2 q2, float2 &v1, float2 &v2) {
    const float e = kFilmDepths * p.dry_tol;
    const float2 hh = mul2(h, h);
    const float2 den = add2(hh, pr(gmax(hh.x, e * e), gmax(hh.y, e * e)));
    const float2 inv = pr(1.0f / den.x, 1.0f / den.y);
    const float2 twice = mul2(pr(2.0f, 2.0f), h);
    v1 = mul2(mul2(twice, q1), inv);
    v2 = mul2(mul2(twice, q2), inv);
    if (!(h.x > p.dry_tol)) v1.x = v2.x = 0.0f;
    if (!(h.y > p.dry_tol)) v1.y = v2.y = 0.0f;
}

// face_states + hllc: the reconstructed depths hs and the face-frame HLLC flux and speed bound.
__device__ __forceinline__ void face_flux_pair(const Phys &p, float nx, float ny, float2 dz, float2 h, float2 hu,
                                               float2 hv, float2 &hs, float &Fh, float &Fhn, float &Fht,
                                               float &smax) {
    const float2 dh = add2(h, pr(-dz.x, -dz.y));
    hs = pr(gmax(0.0f, dh.x), gmax(0.0f, dh.y));
    float2 u, v;
    safe_vel_pair(p, h, hu, hv, u, v);
    const float2 hus = mul2(hs, u), hvs = mul2(hs, v);
    const float2 qn = fma2(hus, pr(nx, nx), mul2(hvs, pr(ny, ny)));
    const float2 qt = fma2(hvs, pr(nx, nx), mul2(hus, pr(-ny, -ny)));
    float2 un, ut;
    safe_vel_pair(p, hs, qn, qt, un, ut);
    const float sqL = sqrtf(gmax(hs.x, 0.0f)), sqR = sqrtf(gmax(hs.y, 0.0f));
    const float root_g = sqrtf(p.g);
    const float2 c = mul2(pr(root_g, root_g), pr(sqL, sqR));
    const float den = sqL + sqR;
    const float u_roe = (den > 1e-12f) ? fmaf_rn(sqL, un.x, sqR * un.y) / den : 0.0f;
    const float c_roe = sqrtf(p.g * 0.5f * (hs.x + hs.y));
    const float2 a = fma2(pr(-1.0f, 1.0f), c, un);
    const float2 b = fma2(pr(-1.0f, 1.0f), pr(c_roe, c_roe), pr(u_roe, u_roe));
    const float SL0 = gmin(a.x, b.x), SR0 = gmax(a.y, b.y);
    const float wetL = wet_blend(p, hs.x), wetR = wet_blend(p, hs.y);
    const float2 dry = mul2(add2(pr(1.0f, 1.0f), pr(-wetL, -wetR)), pr(wetR, wetL));
    const float roe = 1.0f - dry.x - dry.y;
    const float2 m1 = fma2(pr(-2.0f, 1.0f), pr(c.y, c.y), pr(un.y, un.y));
    const float2 m2 = fma2(pr(-1.0f, 2.0f), pr(c.x, c.x), pr(un.x, un.x));
    const float2 S = fma2(pr(roe, roe), pr(SL0, SR0), fma2(pr(dry.x, dry.x), m1, mul2(pr(dry.y, dry.y), m2)));
    const float SL = S.x, SR = S.y;
    smax = gmax(fabsf(SL), fabsf(SR));
    const float2 aRL = mul2(pr(hs.y, hs.x), add2(pr(un.y, un.x), pr(-SR, -SL)));
    const float num_sm = fmaf_rn(SL, aRL.x, -(SR * aRL.y));
    const float den_sm = aRL.x - aRL.y;
    const float SM = (fabsf(den_sm) > 1e-12f) ? num_sm / den_sm : 0.0f;
    const bool left = (SL >= 0.0f) || (SM >= 0.0f);
    const bool star = !(SL >= 0.0f) && (left || SR >= 0.0f);
    const float hX = left ? hs.x : hs.y, unX = left ? un.x : un.y, utX = left ? ut.x : ut.y;
    const float q = hX * unX;
    Fh = q;
    Fhn = fmaf_rn(q, unX, 0.5f * p.g * hX * hX);
    Fht = q * utX;
    if (star) {
        const float Sx = left ? SL : SR;
        const float dS = Sx - SM;
        const float k = hX * (Sx - unX) / ((fabsf(dS) > 1e-14f) ? dS : 1e-14f);
        Fh = fmaf_rn(Sx, k - hX, q);
        Fhn = fmaf_rn(Sx, fmaf_rn(k, SM, -q), Fhn);
        Fht = fmaf_rn(Sx, (k - hX) * utX, Fht);
    }
}

// Flux of one edge from its two cell states: the five gather words and the
// corrector's CFL word (resident.py:254-284). On an open edge (cR < -1,
// condition kind/value) the mass flux follows the condition, and an
// outflow-only edge whose flux would draw water in is redone as a wall, its
// momentum included (flux.py:284-294). OPEN: the mesh may have open edges.
template <bool OPEN>
__device__ __forceinline__ void edge_words(const Phys &p, int cR, float nx, float ny, float len, float dzL,
                                           float dzR, float hL, float huL, float hvL, float hR, float huR,
                                           float hvR, float &w0, float &w1, float &w2, float &w3, float &w4,
                                           float &w5, uint32_t kind = kOpenWall, float value = 0.0f) {
    float2 hs;
    float Fh, Fhn, Fht, smax;
    face_flux_pair(p, nx, ny, pr(dzL, dzR), pr(hL, hR), pr(huL, huR), pr(hvL, hvR), hs, Fh, Fhn, Fht, smax);
    if (OPEN && cR < -1) {
        if ((kind == kOpenFree || kind == kOpenNormal) && Fh < 0.0f) {
            ghost_state(p, kOpenWall, 0.0f, hL, huL, hvL, nx, ny, hR, huR, hvR);
            face_flux_pair(p, nx, ny, pr(dzL, dzR), pr(hL, hR), pr(huL, huR), pr(hvL, hvR), hs, Fh, Fhn, Fht, smax);
            Fh = 0.0f;
        } else {
            Fh = boundary_mass_flux(kind, value, Fh);
        }
    } else if (cR < 0) {
        Fh = 0.0f;  // a wall passes no mass
    }
    const float2 F = fma2(pr(Fhn, Fhn), pr(nx, ny), mul2(pr(Fht, Fht), pr(-ny, nx)));
    const float2 hs2 = mul2(hs, hs);
    const float2 hyd = mul2(pr(0.5f * p.g, 0.5f * p.g), fma2(pr(hL, hR), pr(hL, hR), pr(-hs2.x, -hs2.y)));
    const float2 wn = mul2(fma2(hyd, pr(nx, nx), pr(F.x, F.x)), pr(len, len));
    const float2 wt = mul2(fma2(hyd, pr(ny, ny), pr(F.y, F.y)), pr(len, len));
    w0 = Fh * len;
    w1 = wn.x;
    w2 = wt.x;
    w3 = wn.y;
    w4 = wt.y;
    w5 = smax * len;
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

// Shared words of a tile pass besides the staged buffers.
template <int TPB>
struct TiledShared {
    uint32_t late[3];  // LateDt's slots
    uint32_t red[2 * TPB / 32];
    uint4 items[2];
    uint32_t dts[2];
    uint32_t count;
};

// A predictor started before its dt and the tile's activity are known (the
// persistent kernel's seat): thread 0 loads both at the start, and after the
// fluxes, which need neither, publishes in slot[0] the dt the update uses (0
// when the tile turns out inactive or its instance does not run: the update is
// then skipped) and in slot[1] the instance's dt. The dt comes from the pair
// the step control publishes, which may still be on its way.
struct LateDt {
    const uint64_t *dt;    // the instance's published (dt, epoch) pair
    const uint32_t *mark;  // the block's epoch word
    const uint32_t *queue; // a word read beside them (the length of this step's tile queue)
    uint32_t epoch;        // this step's epoch: of an active block, and of the pair
    uint32_t all;          // every block is active
    uint32_t *slot;        // three shared words: dt if active (else 0), dt, the queue word
};

// Shared-memory bytes of a tile pass: two staged buffers, and with `keep` (the
// persistent kernel, whose buffers keep their records from step to step) the
// flux words in arrays of their own (8 per record: two float4 slot words).
__host__ __device__ inline size_t tiled_smem_bytes(uint32_t max_edges, uint32_t max_slots, bool keep) {
    const TilePlan L = tile_plan(max_edges, max_slots, 10u);
    return keep ? L.total + 8u * L.capE * 4u : L.total;
}

// Fluxes, gather and update of one staged tile. The stage's input state is in
// columns in_col..in_col+3 of B.c (h, hu, hv, h_lo), the committed state of the
// corrector in com_col..com_col+3. F == nullptr: the flux words overwrite the
// consumed records (side words); otherwise they go to F (8 x capE words, slot words) and the records stay.
// keep_pred: the new state also goes to columns 6..9 (predictor) or 0..3
// (corrector). Returns, in the corrector and to warp 0, whether a cell of the tile is wet.
// OPEN: the mesh has open edges (right cell -2 - k), with ghosts and tallies.
template <int STAGE, bool COMP, bool CLAMP, int TPB, bool OPEN>
__device__ __forceinline__ bool tile_compute(const swe_mesh_t &m, const swe_state_t &s, const Phys &p, float cfl,
                                             const TileBuf &B, const Item &it, float dt, uint32_t in_col,
                                             uint32_t com_col, float *F, uint32_t capE, uint32_t *red,
                                             uint64_t &computed, bool keep_pred, float *sums = nullptr,
                                             const LateDt *late = nullptr) {
    const uint32_t tid = threadIdx.x;
    const uint32_t b = it.tile >> 2;
    uint64_t late_pair = 0u;
    uint32_t late_mark = 0u, late_queue = 0u;
    if (late && tid == 0) {  // in flight while the fluxes are computed
        late_pair = ld_relaxed_u64(late->dt);
        late_mark = *late->mark;
        late_queue = *reinterpret_cast<const volatile uint32_t *>(late->queue);
    }
    if (STAGE == 0 && !late && (it.tile & 3u) == 0u && tid == 0) s.blk[kBlkWords * b + kBlkWet] = 0u;
    const float *C0 = B.c + in_col * kTileCells, *C1 = C0 + kTileCells, *C2 = C0 + 2 * kTileCells;
    const int base = static_cast<int>(it.tile * kTileCells);
    // without F: the side words over the records cr..dzr (six arrays of capE words from B.cr), the CFL word over cl
    const SideWords S{reinterpret_cast<float *>(B.cr), reinterpret_cast<float *>(B.cl), capE};

    // Edge fluxes.
    for (uint32_t j = tid; j < it.ne; j += TPB) {
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
            if (lR < static_cast<uint32_t>(kTileCells)) {
                hR = C0[lR];
                huR = C1[lR];
                hvR = C2[lR];
            } else {
                load_state<STAGE>(s, cR, hR, huR, hvR);
            }
        }
        const bool live = !(hL < p.dry_tol && hR < p.dry_tol) || (OPEN && open_forced(kind, value));
        const float len = B.len[j], dzl = B.dzl[j], dzr = B.dzr[j];
        float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f, w4 = 0.0f, w5 = 0.0f;
        if (live) {
            edge_words<OPEN>(p, cR, nx, ny, len, dzl, dzr, hL, huL, hvL, hR, huR, hvR, w0, w1, w2, w3, w4, w5, kind,
                             value);
            if (OPEN && cR < -1) tally_open(s.open_vol, static_cast<uint32_t>(-2 - cR), (0.5f * dt) * w0);
        }
        if (F)
            put_slot_words<STAGE>(F, j, live, w0, w1, w2, w3, w4, w5);
        else
            put_side_words<STAGE>(S, j, live, w0, w1, w2, w3, w4, w5);
    }
    if (late && tid == 0) {
        const uint32_t late_dt = published_dt(s, late->dt, late->epoch, late_pair);
        const bool active = late->all || late_mark == late->epoch;
        late->slot[0] = active ? late_dt : 0u;
        late->slot[1] = late_dt;
        late->slot[2] = late_queue;
        if (STAGE == 0 && active && late_dt != 0u && (it.tile & 3u) == 0u) s.blk[kBlkWords * b + kBlkWet] = 0u;
    }
    __syncthreads();
    if (late) {
        if (late->slot[0] == 0u) return false;
        dt = __uint_as_float(late->slot[0]);
    }

    bool wet = false;
    uint32_t bound = kNoBound;
    if (tid < it.cells) {
        float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
        const uint32_t k0 = B.cptr[tid] - B.cptr[0], k1 = B.cptr[tid + 1] - B.cptr[0];
        if (F) {
#pragma unroll 1  // unrolled, the float4 loads in flight spill the persistent kernel's registers
            for (uint32_t q = k0; q < k1; ++q) add_slot_words<STAGE>(F, B.lcsr[q], sdh, sdhu, sdhv, lam);
        } else {
            for (uint32_t q = k0; q < k1; ++q) add_side_words<STAGE>(S, B.lcsr[q], sdh, sdhu, sdhv, lam);
        }
        if (sums) {  // the record the adjoint reverses
            const uint32_t n = m.n_blocks * kBlockCells, i = base + tid;
            sums[i] = sdh;
            sums[n + i] = sdhu;
            sums[2 * n + i] = sdhv;
        }
        const float *c = B.c;
        const float *ci = c + in_col * kTileCells, *cc = c + com_col * kTileCells;
        update_cell<STAGE, COMP, CLAMP>(s, p, cfl, dt, base + tid, c[4 * kTileCells + tid], c[5 * kTileCells + tid],
                                        ci[tid], ci[kTileCells + tid], ci[2 * kTileCells + tid],
                                        ci[3 * kTileCells + tid], STAGE ? cc[tid] : 0.0f,
                                        STAGE ? cc[kTileCells + tid] : 0.0f, STAGE ? cc[2 * kTileCells + tid] : 0.0f,
                                        STAGE ? cc[3 * kTileCells + tid] : 0.0f, sdh, sdhu, sdhv, lam, wet, bound,
                                        keep_pred ? B.c + (STAGE ? 0 : 6) * kTileCells + tid : nullptr);
    }
    if (STAGE == 1) {
        bool any_wet;
        uint32_t bmin;
        tile_outcome(wet, bound, red, any_wet, bmin);
        if (tid == 0) {
            if (any_wet) s.blk[kBlkWords * b + kBlkWet] = 1u;
            if (bmin != kNoBound) atomicMin(&s.dt_buf[kDtWords * it.inst + 1], bmin);
            computed += it.cells;
        }
        return any_wet;  // valid in warp 0
    }
    return false;
}

// One stage over the current tile work items: items blockIdx.x, + gridDim.x, ...
// `smem` holds the two mbarriers (initialised by the caller) and the two staged
// buffers; `k` counts this CTA's buffer uses across calls (their mbarrier
// phases); computed cells of the corrector accumulate in `computed`.
// Returns false when staged data did not arrive within the wait bound (the
// copies in flight have had one more bounded wait; the caller must stop).
template <int STAGE, bool COMP, bool CLAMP, int TPB, bool OPEN>
__device__ bool tiled_pass(const swe_mesh_t &m, const swe_state_t &s, const Phys &p, float cfl, unsigned char *smem,
                           TiledShared<TPB> &sh, uint32_t &k, uint64_t &computed, float *sums = nullptr) {
    constexpr uint32_t nc = STAGE ? 10u : 6u;
    const TilePlan L = tile_plan(m.max_sub_edges, m.max_sub_slots, nc);
    uint32_t *red = sh.red;
    uint4 *items = sh.items;
    uint32_t *dts = sh.dts;
    const uint4 *work = reinterpret_cast<const uint4 *>(s.items);
    const uint32_t tid = threadIdx.x;

    if (tid < 32u) {
        // The item count and this CTA's first item in one round trip (the item buffer
        // holds four per block, so the read stays inside it even past the count).
        uint32_t cnt = 0u;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (tid == 0) {
            cnt = *reinterpret_cast<volatile const uint32_t *>(s.sched + kSchedItems);
            if (blockIdx.x < 4u * m.n_blocks) v = work[blockIdx.x];
        }
        cnt = __shfl_sync(0xFFFFFFFFu, cnt, 0);
        v.x = __shfl_sync(0xFFFFFFFFu, v.x, 0);
        v.y = __shfl_sync(0xFFFFFFFFu, v.y, 0);
        v.z = __shfl_sync(0xFFFFFFFFu, v.z, 0);
        v.w = __shfl_sync(0xFFFFFFFFu, v.w, 0);
        if (tid == 0) sh.count = cnt;
        if (blockIdx.x < cnt) {
            const Item it = unpack(v);
            if (tid == 0) {
                items[k & 1u] = v;
                dts[k & 1u] = s.dt_buf[kDtWords * it.inst];
            }
            tile_issue<STAGE>(m, s, it, tile_buf(smem, L, k & 1u));
        }
    }
    __syncthreads();
    const uint32_t count = sh.count;
    if (blockIdx.x >= count) return true;

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
            return false;
        }
        const uint32_t dt_bits = dts[k & 1u];
        if (dt_bits != 0u)
            tile_compute<STAGE, COMP, CLAMP, TPB, OPEN>(m, s, p, cfl, B, unpack(items[k & 1u]), __uint_as_float(dt_bits), 0u,
                                                  6u, nullptr, L.capE, red, computed, false, sums);
        // This buffer is refilled by bulk copies two items on.
        fence_proxy_async();
        __syncthreads();
    }
    return true;
}

}  // namespace swe
