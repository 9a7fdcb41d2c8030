// Adjoint (reverse mode) of the resident shallow-water step, dt frozen.
//
// Differentiates the discrete step the forward kernels compute -- the edge
// flux (hydrostatic reconstruction, Kurganov-Petrova velocities, HLLC with
// dry-bed wave speeds), the fixed-order gather, the Heun stages with film
// drag and semi-implicit Manning friction, the sources with hydrograph
// discharge -- with every step's dt held at its forward value. Non-smooth
// points (clamps, dry thresholds, HLLC regions, the higher of two beds) take
// the derivative of the branch the forward took; the forward's branch
// decisions are reproduced exactly by recomputing the primal with the same
// expressions from the taped state and stage sums.
//
// Per step, reversed over that step's active blocks (every live edge joins
// two cells of active blocks, so nothing outside them has a derivative):
//   boundary    the misfit's gradient at the state after the step; knot
//               gradients of the hydrograph sources
//   cell1       the Heun average and the corrector's cell update: adjoint of
//               the corrector sums and of the predictor state (local part)
//   edge<1>     the corrector's edges: adjoint of the predictor state through
//               the fluxes, gathered per cell in CSR order (no float atomics)
//   cell0       the predictor's cell update
//   edge<0>     the predictor's edges, into the adjoint of the step's start state
// Parameter gradients: Manning n in the cell kernels, the bed through the
// edges' face steps dzL = max(zL, zR) - zL, dzR = max(zL, zR) - zR.
// No counterpart in the reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "swe_grid.cuh"

namespace swe {

// -- primal pieces that report their branch ---------------------------------------------------------
// add_compensated, also telling whether the clamp at zero was taken.
__device__ __forceinline__ bool add_compensated_clamped(float hi, float lo, float inc, float &h_new, float &lo_new) {
    float s, e;
    two_sum(hi, inc, s, e);
    e += lo;
    two_sum(s, e, h_new, lo_new);
    if (h_new < 0.0f || (h_new == 0.0f && lo_new < 0.0f)) {
        h_new = 0.0f;
        lo_new = 0.0f;
        return true;
    }
    return false;
}

// One cell's Heun-stage update (the forward's update_cell without the stores),
// with the values its reverse needs.
struct CellFwd {
    float h_new, lo_new, hu_new, hv_new;  // outputs
    float hu_a, hv_a;                     // momenta before drag and friction
    float drag, hu_b, hv_b;               // after drag
    float spd, Q, Sf, den, u, v;          // friction (Q = h^(-4/3))
    bool clamped, wet;
};

__device__ __forceinline__ CellFwd cell_forward(const Phys &p, float dt, float A, float n, float hi, float loi,
                                                float hui, float hvi, float sdh, float sdhu, float sdhv) {
    CellFwd c;
    const float dti = dt / A;
    c.clamped = add_compensated_clamped(hi, loi, -dti * sdh, c.h_new, c.lo_new);
    c.hu_a = fmaf_rn(-dti, sdhu, hui);
    c.hv_a = fmaf_rn(-dti, sdhv, hvi);
    c.wet = !(c.h_new < p.dry_tol);
    c.drag = 1.0f;
    c.hu_b = c.hu_a;
    c.hv_b = c.hv_a;
    c.spd = c.Q = c.Sf = c.u = c.v = 0.0f;
    c.den = 1.0f;
    if (!c.wet) {
        c.hu_new = 0.0f;
        c.hv_new = 0.0f;
        return c;
    }
    c.drag = film_drag(p, c.h_new, dt);
    c.hu_b = c.hu_a * c.drag;
    c.hv_b = c.hv_a * c.drag;
    const float inv_h = 1.0f / c.h_new;
    c.u = c.hu_b * inv_h;
    c.v = c.hv_b * inv_h;
    c.spd = sqrtf(fmaf_rn(c.u, c.u, c.v * c.v));
    c.Q = inv_pow43(c.h_new);
    c.Sf = p.g * n * n * c.spd * c.Q;
    c.den = fmaf_rn(dt, c.Sf, 1.0f);
    const float inv_den = 1.0f / c.den;
    c.hu_new = c.hu_b * inv_den;
    c.hv_new = c.hv_b * inv_den;
    return c;
}

// Reverse of cell_forward: output adjoints (gH on the total depth, gHU, gHV)
// to the adjoints of the inputs (state, sums) and of n.
__device__ __forceinline__ void cell_reverse(const Phys &p, float dt, float A, float n, const CellFwd &c, float gH,
                                             float gHU, float gHV, float &g_h, float &g_hu, float &g_hv, float &g_sdh,
                                             float &g_sdhu, float &g_sdhv, float &g_n, bool cut_in, float cut) {
    const float dti = dt / A;
    float g_hua = 0.0f, g_hva = 0.0f;
    if (c.wet) {
        const float h = c.h_new;
        const bool thin = h < cut;  // friction and drag depth held constant
        float g_hub = gHU / c.den, g_hvb = gHV / c.den;
        const float g_den = -(gHU * c.hu_new + gHV * c.hv_new) / c.den;
        const float g_Sf = g_den * dt;
        g_n += g_Sf * 2.0f * p.g * n * c.spd * c.Q;
        const float g_spd = g_Sf * p.g * n * n * c.Q;
        // Sf is proportional to h^(-4/3): d Sf / dh = -(4/3) Sf / h
        if (!thin) gH -= g_Sf * c.Sf * (4.0f / 3.0f) / h;
        if (c.spd > 0.0f) {
            const float g_u = g_spd * c.u / c.spd, g_v = g_spd * c.v / c.spd;
            g_hub += g_u / h;
            g_hvb += g_v / h;
            if (!thin) gH -= (g_u * c.u + g_v * c.v) / h;
        }
        g_hua = g_hub * c.drag;
        g_hva = g_hvb * c.drag;
        const float e = kFilmDepths * p.dry_tol;
        if (h < e && !thin) {
            // drag = 1 / (1 + dt rate), rate = (e^2 - h^2) / (2 h^2) sqrt(g / e): d drag / dh = dt e^2 / h^3 sqrt(g/e) drag^2
            const float g_drag = g_hub * c.hu_a + g_hvb * c.hv_a;
            gH += g_drag * dt * e * e / (h * h * h) * sqrtf(p.g / e) * c.drag * c.drag;
        }
    }
    if (!c.clamped) {
        if (!cut_in) g_h += gH;
        g_sdh = -dti * gH;
    } else {
        g_sdh = 0.0f;
    }
    if (!cut_in) {
        g_hu += g_hua;
        g_hv += g_hva;
    }
    g_sdhu = -dti * g_hua;
    g_sdhv = -dti * g_hva;
}

// -- edge reverse ---------------------------------------------------------------------------------
__device__ __forceinline__ void safe_vel_rev(const Phys &p, float h, float q, float gu, float &gh, float &gq) {
    if (!(h > p.dry_tol) || gu == 0.0f) return;
    const float e = kFilmDepths * p.dry_tol;
    const float h2 = h * h, e2 = e * e;
    const bool big = !(h2 < e2);  // gmax(h2, e2)
    const float D = h2 + (big ? h2 : e2);
    const float dD = big ? 4.0f * h : 2.0f * h;
    gq += gu * 2.0f * h / D;
    gh += gu * (2.0f * q / D - 2.0f * h * q * dD / (D * D));
}

__device__ __forceinline__ float wet_blend_d(const Phys &p, float h) {
    return (h > p.dry_tol && h < 2.0f * p.dry_tol) ? 1.0f / p.dry_tol : 0.0f;
}

struct EdgeGrad {
    float hL, huL, hvL, hR, huR, hvR, dzL, dzR;
};

// Adjoint of the five gather words of edge_words (w0 .. w4) with respect to
// the two cell states and the two bed steps. The primal is recomputed with
// the forward's expressions, so every branch is the one the forward took.
__device__ EdgeGrad edge_words_rev(const Phys &p, bool wall, float nx, float ny, float len, float dzL, float dzR,
                                   float hL, float huL, float hvL, float hR, float huR, float hvR, float g0, float g1,
                                   float g2, float g3, float g4, float cut) {
    // ---- primal (face_states, hllc_speeds_fast, hllc) ----
    const float hLs = gmax(0.0f, hL - dzL);
    const float hRs = gmax(0.0f, hR - dzR);
    float uL, vL, uR, vR;
    safe_vel2(p, hL, huL, hvL, uL, vL);
    safe_vel2(p, hR, huR, hvR, uR, vR);
    const float huLs = hLs * uL, hvLs = hLs * vL, huRs = hRs * uR, hvRs = hRs * vR;
    const float hqnL = fmaf_rn(huLs, nx, hvLs * ny);
    const float hqtL = fmaf_rn(hvLs, nx, -(huLs * ny));
    const float hqnR = fmaf_rn(huRs, nx, hvRs * ny);
    const float hqtR = fmaf_rn(hvRs, nx, -(huRs * ny));
    float unL, utL, unR, utR;
    safe_vel2(p, hLs, hqnL, hqtL, unL, utL);
    safe_vel2(p, hRs, hqnR, hqtR, unR, utR);
    const float sqL = sqrtf(gmax(hLs, 0.0f));
    const float sqR = sqrtf(gmax(hRs, 0.0f));
    const float root_g = sqrtf(p.g);
    const float cL = root_g * sqL;
    const float cR = root_g * sqR;
    const float den = sqL + sqR;
    const bool roe_ok = den > 1e-12f;
    const float u_roe = roe_ok ? fmaf_rn(sqL, unL, sqR * unR) / den : 0.0f;
    const float c_roe = sqrtf(p.g * 0.5f * (hLs + hRs));
    const float aL = unL - cL, bL = u_roe - c_roe;
    const bool selL = bL < aL;
    const float SL0 = selL ? bL : aL;
    const float aR = unR + cR, bR = u_roe + c_roe;
    const bool selR = aR < bR;
    const float SR0 = selR ? bR : aR;
    const float wetL = wet_blend(p, hLs);
    const float wetR = wet_blend(p, hRs);
    const float dryLeft = (1.0f - wetL) * wetR;
    const float dryRight = (1.0f - wetR) * wetL;
    const float roe = 1.0f - dryLeft - dryRight;
    const float SL = fmaf_rn(roe, SL0, fmaf_rn(dryLeft, fmaf_rn(-2.0f, cR, unR), dryRight * (unL - cL)));
    const float SR = fmaf_rn(roe, SR0, fmaf_rn(dryLeft, unR + cR, dryRight * fmaf_rn(2.0f, cL, unL)));
    const float aRs = hRs * (unR - SR), aLs = hLs * (unL - SL);
    const float num_sm = fmaf_rn(SL, aRs, -(SR * aLs));
    const float den_sm = aRs - aLs;
    const bool sm_ok = fabsf(den_sm) > 1e-12f;
    const float SM = sm_ok ? num_sm / den_sm : 0.0f;
    const int branch = (SL >= 0.0f) ? 0 : (SM >= 0.0f) ? 1 : (SR >= 0.0f) ? 2 : 3;

    // ---- reverse ----
    const float gFh = wall ? 0.0f : g0 * len;
    const float gFhu = (g1 + g3) * len, gFhv = (g2 + g4) * len;
    const float gSLg = (g1 * nx + g2 * ny) * len, gSRg = (g3 * nx + g4 * ny) * len;
    EdgeGrad G{};
    G.hL = gSLg * p.g * hL;
    G.hR = gSRg * p.g * hR;
    float ghLs = -gSLg * p.g * hLs, ghRs = -gSRg * p.g * hRs;
    const float gFhn = gFhu * nx + gFhv * ny;
    const float gFht = -gFhu * ny + gFhv * nx;
    float gunL = 0.0f, gutL = 0.0f, gunR = 0.0f, gutR = 0.0f, gSL = 0.0f, gSR = 0.0f, gSM = 0.0f;
    if (branch == 0) {
        ghLs += gFh * unL + gFhn * (unL * unL + p.g * hLs) + gFht * unL * utL;
        gunL += gFh * hLs + gFhn * 2.0f * hLs * unL + gFht * hLs * utL;
        gutL += gFht * hLs * unL;
    } else if (branch == 3) {
        ghRs += gFh * unR + gFhn * (unR * unR + p.g * hRs) + gFht * unR * utR;
        gunR += gFh * hRs + gFhn * 2.0f * hRs * unR + gFht * hRs * utR;
        gutR += gFht * hRs * unR;
    } else if (branch == 1) {
        const float dSL = SL - SM;
        const bool dok = fabsf(dSL) > 1e-14f;
        const float d = dok ? dSL : 1e-14f;
        const float kL = hLs * (SL - unL) / d;
        gSL += gFh * (kL - hLs) + gFhn * (kL * SM - hLs * unL) + gFht * (kL * utL - hLs * utL);
        const float gkL = gFh * SL + gFhn * SL * SM + gFht * SL * utL;
        gSM += gFhn * SL * kL;
        ghLs += gFh * (unL - SL) + gFhn * (unL * unL + p.g * hLs - SL * unL) + gFht * (unL * utL - SL * utL);
        gunL += gFh * hLs + gFhn * (2.0f * hLs * unL - SL * hLs) + gFht * hLs * utL;
        gutL += gFht * (hLs * unL + SL * kL - SL * hLs);
        ghLs += gkL * (SL - unL) / d;
        gSL += gkL * hLs / d;
        gunL -= gkL * hLs / d;
        if (dok) {
            const float gd = -gkL * kL / d;
            gSL += gd;
            gSM -= gd;
        }
    } else {
        const float dSR = SR - SM;
        const bool dok = fabsf(dSR) > 1e-14f;
        const float d = dok ? dSR : 1e-14f;
        const float kR = hRs * (SR - unR) / d;
        gSR += gFh * (kR - hRs) + gFhn * (kR * SM - hRs * unR) + gFht * (kR * utR - hRs * utR);
        const float gkR = gFh * SR + gFhn * SR * SM + gFht * SR * utR;
        gSM += gFhn * SR * kR;
        ghRs += gFh * (unR - SR) + gFhn * (unR * unR + p.g * hRs - SR * unR) + gFht * (unR * utR - SR * utR);
        gunR += gFh * hRs + gFhn * (2.0f * hRs * unR - SR * hRs) + gFht * hRs * utR;
        gutR += gFht * (hRs * unR + SR * kR - SR * hRs);
        ghRs += gkR * (SR - unR) / d;
        gSR += gkR * hRs / d;
        gunR -= gkR * hRs / d;
        if (dok) {
            const float gd = -gkR * kR / d;
            gSR += gd;
            gSM -= gd;
        }
    }
    if (sm_ok && gSM != 0.0f) {
        const float gnum = gSM / den_sm, gden = -gSM * SM / den_sm;
        gSL += gnum * (hRs * (unR - SR) + SR * hLs) + gden * hLs;
        gSR += gnum * (-SL * hRs - hLs * (unL - SL)) - gden * hRs;
        ghRs += gnum * SL * (unR - SR) + gden * (unR - SR);
        ghLs -= gnum * SR * (unL - SL) + gden * (unL - SL);
        gunR += gnum * SL * hRs + gden * hRs;
        gunL -= gnum * SR * hLs + gden * hLs;
    }
    // wave speeds
    const float groe = gSL * SL0 + gSR * SR0;
    const float gSL0 = gSL * roe, gSR0 = gSR * roe;
    const float gdryLeft = gSL * (unR - 2.0f * cR) + gSR * (unR + cR) - groe;
    const float gdryRight = gSL * (unL - cL) + gSR * (unL + 2.0f * cL) - groe;
    gunR += (gSL + gSR) * dryLeft;
    float gcR = (-2.0f * gSL + gSR) * dryLeft;
    gunL += (gSL + gSR) * dryRight;
    float gcL = (-gSL + 2.0f * gSR) * dryRight;
    const float gwetL = -gdryLeft * wetR + gdryRight * (1.0f - wetR);
    const float gwetR = gdryLeft * (1.0f - wetL) - gdryRight * wetL;
    ghLs += gwetL * wet_blend_d(p, hLs);
    ghRs += gwetR * wet_blend_d(p, hRs);
    float gu_roe = 0.0f, gc_roe = 0.0f;
    if (selL) {
        gu_roe += gSL0;
        gc_roe -= gSL0;
    } else {
        gunL += gSL0;
        gcL -= gSL0;
    }
    if (selR) {
        gu_roe += gSR0;
        gc_roe += gSR0;
    } else {
        gunR += gSR0;
        gcR += gSR0;
    }
    if (c_roe > 0.0f) {
        const float t = gc_roe * 0.25f * p.g / c_roe;
        ghLs += t;
        ghRs += t;
    }
    if (roe_ok) {
        const float gsqL = gu_roe * (unL - u_roe) / den, gsqR = gu_roe * (unR - u_roe) / den;
        gunL += gu_roe * sqL / den;
        gunR += gu_roe * sqR / den;
        if (sqL > 0.0f) ghLs += gsqL * 0.5f / sqL;
        if (sqR > 0.0f) ghRs += gsqR * 0.5f / sqR;
    }
    if (cL > 0.0f) ghLs += gcL * 0.5f * p.g / cL;
    if (cR > 0.0f) ghRs += gcR * 0.5f * p.g / cR;
    // face-frame velocities
    float ghqnL = 0.0f, ghqtL = 0.0f, ghqnR = 0.0f, ghqtR = 0.0f;
    safe_vel_rev(p, hLs, hqnL, gunL, ghLs, ghqnL);
    safe_vel_rev(p, hLs, hqtL, gutL, ghLs, ghqtL);
    safe_vel_rev(p, hRs, hqnR, gunR, ghRs, ghqnR);
    safe_vel_rev(p, hRs, hqtR, gutR, ghRs, ghqtR);
    const float ghuLs = ghqnL * nx - ghqtL * ny, ghvLs = ghqnL * ny + ghqtL * nx;
    const float ghuRs = ghqnR * nx - ghqtR * ny, ghvRs = ghqnR * ny + ghqtR * nx;
    ghLs += ghuLs * uL + ghvLs * vL;
    ghRs += ghuRs * uR + ghvRs * vR;
    safe_vel_rev(p, hL, huL, ghuLs * hLs, G.hL, G.huL);
    safe_vel_rev(p, hL, hvL, ghvLs * hLs, G.hL, G.hvL);
    safe_vel_rev(p, hR, huR, ghuRs * hRs, G.hR, G.huR);
    safe_vel_rev(p, hR, hvR, ghvRs * hRs, G.hR, G.hvR);
    // hydrostatic reconstruction h* = max(0, h - dz)
    if (0.0f < hL - dzL && !(hLs < cut)) {
        G.hL += ghLs;
        G.dzL = -ghLs;
    }
    if (0.0f < hR - dzR && !(hRs < cut)) {
        G.hR += ghRs;
        G.dzR = -ghRs;
    }
    if (hR < cut) G.hR = G.huR = G.hvR = G.dzR = 0.0f;
    if (hL < cut) {
        G.hL = G.huL = G.hvL = G.dzL = 0.0f;
        if (wall) G.hR = G.huR = G.hvR = G.dzR = 0.0f;  // the ghost is the (held) left state
    }
    if (wall) {
        // the ghost is the left state mirrored; a wall's bed steps are fixed at zero
        G.hL += G.hR;
        G.huL += G.huR * (1.0f - 2.0f * nx * nx) - G.hvR * 2.0f * nx * ny;
        G.hvL += -G.huR * 2.0f * nx * ny + G.hvR * (1.0f - 2.0f * ny * ny);
        G.hR = G.huR = G.hvR = 0.0f;
        G.dzL = G.dzR = 0.0f;
    }
    return G;
}

// -- kernels ------------------------------------------------------------------------------------------
struct Slot {
    const float *h, *hu, *hv, *lo;         // the state at the start of the step
    const float *h_next, *lo_next;         // the state after it
    const float *s0, *s1;                  // stage sums
    const uint32_t *list;
    uint32_t count;
};

__device__ __forceinline__ Slot slot_of(const swe_tape_t &T, uint32_t k, uint32_t n, uint32_t n_blocks) {
    Slot s;
    const size_t o = static_cast<size_t>(k) * n, o1 = o + n;
    s.h = T.h + o;
    s.hu = T.hu + o;
    s.hv = T.hv + o;
    s.lo = T.h_lo + o;
    s.h_next = T.h + o1;
    s.lo_next = T.h_lo + o1;
    s.s0 = T.s0 + 3 * o;
    s.s1 = T.s1 + 3 * o;
    s.list = T.list + static_cast<size_t>(k) * n_blocks;
    s.count = 0;
    return s;
}

// The misfit's gradient at the state after the step, then the hydrograph knots' gradients.
__device__ void adj_boundary(const swe_tape_t &T, const swe_adjoint_t &a, const swe_sources_t &src,
                             const swe_gauges_t &gg, uint32_t k, uint32_t n, uint32_t row) {
    const float *h1 = T.h + static_cast<size_t>(k + 1) * n, *lo1 = T.h_lo + static_cast<size_t>(k + 1) * n;
    if (gg.count && row < gg.steps) {
        const float *obs = gg.obs + static_cast<size_t>(row) * gg.count;
        for (uint32_t g = threadIdx.x; g < gg.count; g += blockDim.x) {
            const uint32_t c = gg.cells[g];
            a.lh[c] += 2.0f * ((h1[c] + lo1[c]) - obs[g]);
        }
    }
    __syncthreads();
    const uint32_t dt_bits = T.dt[k];
    if (threadIdx.x != 0 || dt_bits == 0u || !src.hydro || !a.gq) return;
    const float dt = __uint_as_float(dt_bits), t = T.t[k];
    for (uint32_t q = 0; q < src.count; ++q) {
        const uint32_t j = src.hydro[q];
        if (j == 0xFFFFFFFFu) continue;
        const double w = static_cast<double>(a.lh[src.cells[q]]) * dt * src.hscale[q];
        const uint32_t k0 = src.knot_ptr[j], k1 = src.knot_ptr[j + 1];
        if (k1 <= k0) continue;
        if (!(t > src.knot_t[k0])) {
            a.gq[k0] += w;
        } else if (!(t < src.knot_t[k1 - 1])) {
            a.gq[k1 - 1] += w;
        } else {
            uint32_t i = k0;
            while (i + 2 < k1 && !(t < src.knot_t[i + 1])) ++i;
            const float f = (t - src.knot_t[i]) / (src.knot_t[i + 1] - src.knot_t[i]);
            a.gq[i] += w * (1.0 - f);
            a.gq[i + 1] += w * f;
        }
    }
}

// The Heun average and the corrector's cell update, reversed; also the
// predictor state (recomputed) and the block marks of this step.
__device__ void adj_cell1(const swe_mesh_t &m, const swe_tape_t &T, const swe_adjoint_t &a, const Phys &p, uint32_t k,
                          uint32_t tag) {
    const uint32_t n = m.n_blocks * kBlockCells;
    const uint32_t count = T.count[k];
    const Slot S = slot_of(T, k, n, m.n_blocks);
    const float dt = __uint_as_float(T.dt[k]);
    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        const uint32_t b = S.list[w];
        if (threadIdx.x == 0) a.mark[b] = tag;
        if (threadIdx.x >= m.block_cells[b]) continue;
        const uint32_t i = b * kBlockCells + threadIdx.x;
        const float A = m.area[i], nm = m.n_mann[i];
        const float h0 = S.h[i], lo0 = S.lo[i], hu0 = S.hu[i], hv0 = S.hv[i];
        const CellFwd c0 = cell_forward(p, dt, A, nm, h0, lo0, hu0, hv0, S.s0[i], S.s0[n + i], S.s0[2 * n + i]);
        a.uh[i] = c0.h_new;
        a.ulo[i] = c0.lo_new;
        a.uhu[i] = c0.hu_new;
        a.uhv[i] = c0.hv_new;
        const CellFwd c1 = cell_forward(p, dt, A, nm, c0.h_new, c0.lo_new, c0.hu_new, c0.hv_new, S.s1[i], S.s1[n + i],
                                        S.s1[2 * n + i]);
        float sm, em, hf, lof;
        two_sum(h0, c1.h_new, sm, em);
        em += lo0 + c1.lo_new;
        two_sum(0.5f * sm, 0.5f * em, hf, lof);
        const float mom = (hf < p.dry_tol) ? 0.0f : 1.0f;
        const float gH = a.lh[i], gHU = a.lhu[i] * mom, gHV = a.lhv[i] * mom;
        float g_h = 0.0f, g_hu = 0.0f, g_hv = 0.0f, g_sh, g_su, g_sv, g_n = 0.0f;
        cell_reverse(p, dt, A, nm, c1, 0.5f * gH, 0.5f * gHU, 0.5f * gHV, g_h, g_hu, g_hv, g_sh, g_su, g_sv, g_n,
                     c0.h_new < a.cut_depth, a.cut_depth);
        a.ls[i] = g_sh;
        a.ls[n + i] = g_su;
        a.ls[2 * n + i] = g_sv;
        a.lsh[i] = g_h;
        a.lshu[i] = g_hu;
        a.lshv[i] = g_hv;
        a.lh[i] = 0.5f * gH;
        a.lhu[i] = 0.5f * gHU;
        a.lhv[i] = 0.5f * gHV;
        a.gn[i] += g_n;
    }
}

// The predictor's cell update, reversed.
__device__ void adj_cell0(const swe_mesh_t &m, const swe_tape_t &T, const swe_adjoint_t &a, const Phys &p, uint32_t k) {
    const uint32_t n = m.n_blocks * kBlockCells;
    const uint32_t count = T.count[k];
    const Slot S = slot_of(T, k, n, m.n_blocks);
    const float dt = __uint_as_float(T.dt[k]);
    for (uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        const uint32_t b = S.list[w];
        if (threadIdx.x >= m.block_cells[b]) continue;
        const uint32_t i = b * kBlockCells + threadIdx.x;
        const float A = m.area[i], nm = m.n_mann[i];
        const CellFwd c0 =
            cell_forward(p, dt, A, nm, S.h[i], S.lo[i], S.hu[i], S.hv[i], S.s0[i], S.s0[n + i], S.s0[2 * n + i]);
        float g_h = 0.0f, g_hu = 0.0f, g_hv = 0.0f, g_sh, g_su, g_sv, g_n = 0.0f;
        cell_reverse(p, dt, A, nm, c0, a.lsh[i], a.lshu[i], a.lshv[i], g_h, g_hu, g_hv, g_sh, g_su, g_sv, g_n,
                     S.h[i] < a.cut_depth, a.cut_depth);
        a.ls[i] = g_sh;
        a.ls[n + i] = g_su;
        a.ls[2 * n + i] = g_sv;
        a.lh[i] += g_h;
        a.lhu[i] += g_hu;
        a.lhv[i] += g_hv;
        a.gn[i] += g_n;
    }
}

// Edge adjoints of one stage, gathered per cell in the forward's CSR order.
// STAGE 1: the corrector (inputs: the predictor state in blocks of this step,
// the start state elsewhere; adds into the predictor's adjoint). STAGE 0: the
// predictor (inputs: the start state; adds into the start state's adjoint).
template <int STAGE>
__device__ void adj_edge(const swe_mesh_t &m, const swe_tape_t &T, const swe_adjoint_t &a, const Phys &p, uint32_t k,
                         uint32_t tag, float *G) {
    const uint32_t count = T.count[k];
    const uint32_t cap = (m.max_sub_edges + 3u) & ~3u;
    const uint32_t n = m.n_blocks * kBlockCells;
    const Slot S = slot_of(T, k, n, m.n_blocks);
    // one 64-cell tile per CTA pass: four per active block, one edge record per thread
    for (uint32_t w = blockIdx.x; w < 4u * count; w += gridDim.x) {
        const uint32_t b = S.list[w >> 2], q4 = w & 3u;
        const uint32_t cells = m.block_cells[b];
        if (q4 * kTileCells >= cells) continue;
        const uint32_t t = 4u * b + q4;
        const uint32_t base = m.sub_ptr[t], ne = m.sub_count[t];
        for (uint32_t j = threadIdx.x; j < ne; j += kThreads) {
            const uint32_t e = base + j;
            const int cL = m.sub_cl[e], cR = m.sub_cr[e];
            const float nx = m.sub_nx[e], ny = m.sub_ny[e];
            const bool actL = a.mark[static_cast<uint32_t>(cL) >> 8] == tag;
            float hL, huL, hvL, hR = 0.0f, huR = 0.0f, hvR = 0.0f;
            if (STAGE == 1 && actL) {
                hL = a.uh[cL];
                huL = a.uhu[cL];
                hvL = a.uhv[cL];
            } else {
                hL = S.h[cL];
                huL = S.hu[cL];
                hvL = S.hv[cL];
            }
            bool actR = false;
            if (cR < 0) {
                hR = hL;
                wall_mirror(huL, hvL, nx, ny, huR, hvR);
            } else {
                actR = a.mark[static_cast<uint32_t>(cR) >> 8] == tag;
                if (STAGE == 1 && actR) {
                    hR = a.uh[cR];
                    huR = a.uhu[cR];
                    hvR = a.uhv[cR];
                } else {
                    hR = S.h[cR];
                    huR = S.hu[cR];
                    hvR = S.hv[cR];
                }
            }
            EdgeGrad eg{};
            if (!(hL < p.dry_tol && hR < p.dry_tol)) {
                const float lhL = actL ? a.ls[cL] : 0.0f, luL = actL ? a.ls[n + cL] : 0.0f,
                            lvL = actL ? a.ls[2 * n + cL] : 0.0f;
                const float lhR = actR ? a.ls[cR] : 0.0f, luR = actR ? a.ls[n + cR] : 0.0f,
                            lvR = actR ? a.ls[2 * n + cR] : 0.0f;
                eg = edge_words_rev(p, cR < 0, nx, ny, m.sub_len[e], m.sub_dzl[e], m.sub_dzr[e], hL, huL, hvL, hR,
                                    huR, hvR, lhL - lhR, luL, lvL, -luR, -lvR, a.cut_depth);
            }
            const bool face_left = m.sub_dzl[e] == 0.0f;  // the face sits on the left bed
            G[j] = eg.hL;
            G[cap + j] = eg.huL;
            G[2 * cap + j] = eg.hvL;
            G[3 * cap + j] = eg.hR;
            G[4 * cap + j] = eg.huR;
            G[5 * cap + j] = eg.hvR;
            G[6 * cap + j] = face_left ? eg.dzR : -eg.dzL;  // d loss / d zL through this edge
            G[7 * cap + j] = face_left ? -eg.dzR : eg.dzL;  // d loss / d zR
        }
        __syncthreads();
        if (threadIdx.x < min(static_cast<uint32_t>(kTileCells), cells - q4 * kTileCells)) {
            const uint32_t i = t * kTileCells + threadIdx.x;
            const uint32_t l0 = m.sub_lcsr_ptr[t], c0 = m.cptr[t * kTileCells];
            float sh = 0.0f, su = 0.0f, sv = 0.0f, sz = 0.0f;
            for (uint32_t q = m.cptr[i], q1 = m.cptr[i + 1]; q < q1; ++q) {
                const uint32_t v = m.sub_lcsr[l0 + q - c0];
                const uint32_t j = v >> 1;
                if (v & 1u) {
                    sh += G[3 * cap + j];
                    su += G[4 * cap + j];
                    sv += G[5 * cap + j];
                    sz += G[7 * cap + j];
                } else {
                    sh += G[j];
                    su += G[cap + j];
                    sv += G[2 * cap + j];
                    sz += G[6 * cap + j];
                }
            }
            if (STAGE == 1) {
                a.lsh[i] += sh;
                a.lshu[i] += su;
                a.lshv[i] += sv;
            } else {
                a.lh[i] += sh;
                a.lhu[i] += su;
                a.lhv[i] += sv;
            }
            a.gz[i] += sz;
        }
        __syncthreads();
    }
}

__global__ void adj_boundary_kernel(swe_tape_t T, swe_adjoint_t a, swe_sources_t src, swe_gauges_t gg, uint32_t k,
                                    uint32_t n, uint32_t row) {
    adj_boundary(T, a, src, gg, k, n, row);
}

__global__ void __launch_bounds__(kThreads)
    adj_cell1_kernel(swe_mesh_t m, swe_tape_t T, swe_adjoint_t a, Phys p, uint32_t k, uint32_t tag) {
    adj_cell1(m, T, a, p, k, tag);
}

__global__ void __launch_bounds__(kThreads) adj_cell0_kernel(swe_mesh_t m, swe_tape_t T, swe_adjoint_t a, Phys p, uint32_t k) {
    adj_cell0(m, T, a, p, k);
}

template <int STAGE>
__global__ void __launch_bounds__(kThreads)
    adj_edge_kernel(swe_mesh_t m, swe_tape_t T, swe_adjoint_t a, Phys p, uint32_t k, uint32_t tag) {
    extern __shared__ float4 smem4[];
    adj_edge<STAGE>(m, T, a, p, k, tag, reinterpret_cast<float *>(smem4));
}

// The reverse of a whole segment in one cooperative launch: the five phases of
// every step, slot by slot from the last, separated by grid barriers instead of
// kernel boundaries. A barrier wait past its bound sets a.sync[40] and stops.
__global__ void __launch_bounds__(kThreads)
    adj_persistent_kernel(swe_mesh_t m, swe_tape_t T, swe_adjoint_t a, swe_sources_t src, swe_gauges_t gg, Phys p,
                          uint32_t slots, uint32_t row0, uint32_t tag0) {
    extern __shared__ float4 smem4[];
    float *G = reinterpret_cast<float *>(smem4);
    __shared__ int flag[2];
    GridSync g{a.sync, a.sync + 32, 0u, 0u};
    if (threadIdx.x == 0) g.epoch = ld_acquire_u32(g.gen);
    __syncthreads();
    const uint32_t n = m.n_blocks * kBlockCells;
    auto nothing = [] {};
    bool ok = true;
    for (uint32_t kk = slots; kk-- > 0 && ok;) {
        const uint32_t tag = tag0 + kk + 1;
        if (blockIdx.x == 0) adj_boundary(T, a, src, gg, kk, n, row0 + kk);
        if (!(ok = grid_sync(g, flag, nothing))) break;
        adj_cell1(m, T, a, p, kk, tag);
        if (!(ok = grid_sync(g, flag, nothing))) break;
        adj_edge<1>(m, T, a, p, kk, tag, G);
        if (!(ok = grid_sync(g, flag, nothing))) break;
        adj_cell0(m, T, a, p, kk);
        if (!(ok = grid_sync(g, flag, nothing))) break;
        adj_edge<0>(m, T, a, p, kk, tag, G);
        ok = grid_sync(g, flag, nothing);
    }
    if (!ok && threadIdx.x == 0) atomicOr(a.sync + 40, 1u);
}

// Tape record at the start of a step (or the end state at slot == capacity).
__global__ void tape_record_kernel(swe_mesh_t m, swe_state_t s, swe_tape_t T, uint32_t k) {
    const uint32_t n = m.n_blocks * kBlockCells;
    const size_t o = static_cast<size_t>(k) * n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T.h[o + i] = s.h[i];
        T.hu[o + i] = s.hu[i];
        T.hv[o + i] = s.hv[i];
        T.h_lo[o + i] = s.h_lo[i];
    }
    if (k >= T.capacity) return;
    const uint32_t count = s.sched[kSchedActive];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        T.list[static_cast<size_t>(k) * m.n_blocks + i] = s.active_list[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        T.count[k] = count;
        T.dt[k] = s.dt_buf[0];
        T.t[k] = static_cast<float>(s.ctrl->now_ticks) * (1.0f / kTicksPerSecond);
    }
}

// Gauge record (record = 1) or misfit accumulation, after a step.
__global__ void __launch_bounds__(kThreads) gauge_kernel(swe_state_t s, swe_gauges_t gg, int record) {
    __shared__ double acc[kThreads];
    const uint64_t done = s.ctrl->steps;
    double sum = 0.0;
    if (done >= 1 && done <= gg.steps) {
        float *row = gg.obs + static_cast<size_t>(done - 1) * gg.count;
        for (uint32_t g = threadIdx.x; g < gg.count; g += kThreads) {
            const uint32_t c = gg.cells[g];
            const float H = s.h[c] + s.h_lo[c];
            if (record) {
                row[g] = H;
            } else {
                const double d = static_cast<double>(H) - static_cast<double>(row[g]);
                sum += d * d;
            }
        }
    }
    if (record) return;
    acc[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) acc[threadIdx.x] += acc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *gg.loss += acc[0];
}

__global__ void bed_steps_kernel(const int32_t *cl, const int32_t *cr, const float *z, float *dzl, float *dzr,
                                 uint32_t records) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < records; e += gridDim.x * blockDim.x) {
        const double zl = z[cl[e]];
        const double zr = cr[e] >= 0 ? static_cast<double>(z[cr[e]]) : zl;
        const double face = zl < zr ? zr : zl;
        dzl[e] = static_cast<float>(face - zl);
        dzr[e] = static_cast<float>(face - zr);
    }
}

inline size_t edge_adj_smem(uint32_t max_sub_edges) { return ((max_sub_edges + 3u) & ~3u) * 8 * sizeof(float); }

}  // namespace swe

using namespace swe;

extern "C" {

int swe_bed_steps(const swe_mesh_t *mesh, const float *z, float *tile_dzl, float *tile_dzr, uint32_t tile_records,
                  float *sub_dzl, float *sub_dzr, uint32_t sub_records, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !z || !tile_dzl || !tile_dzr || !sub_dzl || !sub_dzr) return SWE_ERR_ARGUMENT;
    if (tile_records) {
        bed_steps_kernel<<<min((tile_records + 255u) / 256u, 4096u), 256, 0, stream>>>(mesh->tile_cl, mesh->tile_cr, z,
                                                                                    tile_dzl, tile_dzr, tile_records);
        int rc = check_launch();
        if (rc) return rc;
    }
    if (sub_records) {
        bed_steps_kernel<<<min((sub_records + 255u) / 256u, 4096u), 256, 0, stream>>>(mesh->sub_cl, mesh->sub_cr, z,
                                                                                   sub_dzl, sub_dzr, sub_records);
        return check_launch();
    }
    return SWE_OK;
}

int swe_tape_record(const swe_mesh_t *mesh, const swe_state_t *state, const swe_tape_t *tape, uint32_t slot,
                    swe_stream_t stream) {
    if (!mesh_ok(mesh) || !state_ok(state) || !tape || slot > tape->capacity || mesh->n_inst != 1u)
        return SWE_ERR_ARGUMENT;
    tape_record_kernel<<<min(mesh->n_blocks, 148u * 4u), 256, 0, stream>>>(*mesh, *state, *tape, slot);
    return check_launch();
}

int swe_gauge_misfit(const swe_state_t *state, const swe_gauges_t *gauges, int record, swe_stream_t stream) {
    if (!state_ok(state) || !gauges || !gauges->cells || !gauges->obs || (!record && !gauges->loss)) return SWE_ERR_ARGUMENT;
    if (gauges->count == 0u) return SWE_OK;
    gauge_kernel<<<1, kThreads, 0, stream>>>(*state, *gauges, record);
    return check_launch();
}

int swe_adjoint_segment(const swe_mesh_t *mesh, const swe_params_t *params, const swe_tape_t *tape,
                        const swe_adjoint_t *adj, const swe_sources_t *sources, const swe_gauges_t *gauges,
                        uint32_t slots, uint32_t row0, uint32_t tag0, swe_stream_t stream) {
    if (!mesh_ok(mesh) || !params || !tape || !adj || !sources || !gauges || slots > tape->capacity ||
        mesh->n_inst != 1u || !params->compensated || mesh->n_open)
        return SWE_ERR_ARGUMENT;
    const size_t bytes = edge_adj_smem(mesh->max_sub_edges);
    int rc = set_smem(adj_edge_kernel<0>, bytes);
    if (!rc) rc = set_smem(adj_edge_kernel<1>, bytes);
    if (rc) return rc;
    const Phys ph{params->g, params->dry_tol};
    const uint32_t n = mesh->n_blocks * kBlockCells;
    if (adj->sync) {
        auto kern = adj_persistent_kernel;
        if ((rc = set_smem(kern, bytes))) return rc;
        int per_sm = 0, dev = 0, sms = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, bytes) != cudaSuccess)
            return SWE_ERR_CUDA;
        if (per_sm < 1) return SWE_ERR_TOO_LARGE;
        const uint32_t fit = static_cast<uint32_t>(per_sm) * static_cast<uint32_t>(sms);
        const uint32_t pgrid = (params->grid == 0u || params->grid > fit) ? fit : params->grid;
        swe_mesh_t mm = *mesh;
        swe_tape_t tt = *tape;
        swe_adjoint_t aa = *adj;
        swe_sources_t sc = *sources;
        swe_gauges_t gg = *gauges;
        Phys ph{params->g, params->dry_tol};
        uint32_t sl = slots, r0 = row0, t0 = tag0;
        void *args[] = {&mm, &tt, &aa, &sc, &gg, &ph, &sl, &r0, &t0};
        if (cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(pgrid), dim3(kThreads), args, bytes,
                                        stream) != cudaSuccess)
            return SWE_ERR_CUDA;
        return SWE_OK;
    }
    // Every kernel takes the slot's active count from the tape (device memory) and
    // strides over that many list entries with a persistent grid.
    const uint32_t grid = (params->grid == 0u || params->grid > mesh->n_blocks) ? mesh->n_blocks : params->grid;
    for (uint32_t kk = slots; kk-- > 0;) {
        const uint32_t tag = tag0 + kk + 1;
        adj_boundary_kernel<<<1, kThreads, 0, stream>>>(*tape, *adj, *sources, *gauges, kk, n, row0 + kk);
        if ((rc = check_launch())) return rc;
        adj_cell1_kernel<<<grid, kThreads, 0, stream>>>(*mesh, *tape, *adj, ph, kk, tag);
        if ((rc = check_launch())) return rc;
        adj_edge_kernel<1><<<grid, kThreads, bytes, stream>>>(*mesh, *tape, *adj, ph, kk, tag);
        if ((rc = check_launch())) return rc;
        adj_cell0_kernel<<<grid, kThreads, 0, stream>>>(*mesh, *tape, *adj, ph, kk);
        if ((rc = check_launch())) return rc;
        adj_edge_kernel<0><<<grid, kThreads, bytes, stream>>>(*mesh, *tape, *adj, ph, kk, tag);
        if ((rc = check_launch())) return rc;
    }
    return SWE_OK;
}

}  // extern "C"
