// Device arithmetic of the shallow-water step, in float32.
//
// Each function evaluates the reference's GLSL expression
// (inundation/vulkan/shaders/flux.py:43-182 and 301-319) in a stated order:
// contraction is off (--fmad=false), so the only fused multiply-adds are the
// explicit fmaf_rn() calls, and division and square root are IEEE. The FP32
// oracle (oracle/fp32_resident.c) evaluates the same expressions with C's
// fmaf, sqrtf and division, so every result is reproducible bit for bit.
// GLSL contracts a*b+c freely outside `precise` blocks, so a fused site is a
// value the reference admits. GLSL min/max/clamp are written with their
// specified comparisons: min(x,y) = y<x ? y : x, max(x,y) = x<y ? y : x.
#pragma once
#include <cstdint>

namespace swe {

constexpr float kFilmDepths = 4.0f;
constexpr float kTicksPerSecond = 1048576.0f;
constexpr float kDtSentinel = 1e30f;

struct Phys {
    float g;
    float dry_tol;
};

__device__ __forceinline__ float fmaf_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }
__device__ __forceinline__ float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }

// Divisions: GLSL divides to within 2.5 ulp, so a product by a correctly
// rounded reciprocal (or by the float 1/3) is a quotient the reference admits.
// Quotients that share a denominator use one reciprocal; host and device
// evaluate the same expressions.
constexpr float kOneThird = 1.0f / 3.0f;

// x^(-4/3) for x > 0, the depth power of Manning's friction slope (Sf = g n^2 |u| / h^(4/3)),
// without a division: y = x^(-1/3) by Newton's iteration for 1/y^3 = x,
//   y <- y + (y/3)(1 - x y^3),
// from the exponent-thirds estimate bits(y) = (4/3)*127*2^23 - bits(x)/3; four steps
// converge from that estimate's error, then x^(-4/3) = (y^2)^2. Within 6 ulp of the exact
// power over [1e-12, 1e6]. Multiplies and fused multiply-adds only, so host and device agree.
__device__ __forceinline__ float inv_pow43(float x) {
    float y = __uint_as_float(0x54AAAAAAu - __float_as_uint(x) / 3u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float t = x * (y * y);
        y = fmaf_rn(y * kOneThird, fmaf_rn(-t, y, 1.0f), y);
    }
    const float y2 = y * y;
    return y2 * y2;
}

// Desingularised velocity (Kurganov & Petrova 2007): hq/h above the film depth.
__device__ __forceinline__ float safe_vel(const Phys &p, float h, float hq) {
    const float e = kFilmDepths * p.dry_tol;
    return (h > p.dry_tol) ? 2.0f * h * hq / (h * h + gmax(h * h, e * e)) : 0.0f;
}

// safe_vel of two momenta of one depth, with one reciprocal of their denominator.
__device__ __forceinline__ void safe_vel2(const Phys &p, float h, float hq1, float hq2, float &v1, float &v2) {
    if (h > p.dry_tol) {
        const float e = kFilmDepths * p.dry_tol;
        const float inv = 1.0f / (h * h + gmax(h * h, e * e));
        v1 = 2.0f * h * hq1 * inv;
        v2 = 2.0f * h * hq2 * inv;
    } else {
        v1 = 0.0f;
        v2 = 0.0f;
    }
}

// HLLC wave-speed bounds: Roe average, blended continuously into Toro's
// dry-bed speeds u -+ 2c as a side goes from one to two dry_tol deep.
__device__ __forceinline__ void hllc_speeds(const Phys &p, float hL, float unL, float hR, float unR, float &SLo,
                                            float &SRo) {
    const float sqL = sqrtf(gmax(hL, 0.0f));
    const float sqR = sqrtf(gmax(hR, 0.0f));
    const float root_g = sqrtf(p.g);  // loop-invariant: hoisted out of the callers' edge loops
    const float cL = root_g * sqL;
    const float cR = root_g * sqR;
    const float den = sqL + sqR;
    const float u_roe = (den > 1e-12f) ? fmaf_rn(sqL, unL, sqR * unR) / den : 0.0f;
    const float c_roe = sqrtf(p.g * 0.5f * (hL + hR));
    const float SL = gmin(unL - cL, u_roe - c_roe);
    const float SR = gmax(unR + cR, u_roe + c_roe);
    const float wetL = gclamp(hL / p.dry_tol - 1.0f, 0.0f, 1.0f);
    const float wetR = gclamp(hR / p.dry_tol - 1.0f, 0.0f, 1.0f);
    const float dryLeft = (1.0f - wetL) * wetR;
    const float dryRight = (1.0f - wetR) * wetL;
    const float roe = 1.0f - dryLeft - dryRight;
    SLo = fmaf_rn(roe, SL, fmaf_rn(dryLeft, fmaf_rn(-2.0f, cR, unR), dryRight * (unL - cL)));
    SRo = fmaf_rn(roe, SR, fmaf_rn(dryLeft, unR + cR, dryRight * fmaf_rn(2.0f, cL, unL)));
}

// clamp(h / dry_tol - 1, 0, 1) without the division where its value is known:
// division is correctly rounded and monotone, so h >= 2 dry_tol gives exactly
// 1 and h <= dry_tol exactly +0. NaN falls through to the full expression.
__device__ __forceinline__ float wet_blend(const Phys &p, float h) {
    if (h >= 2.0f * p.dry_tol) return 1.0f;
    if (h <= p.dry_tol) return 0.0f;
    return gclamp(h / p.dry_tol - 1.0f, 0.0f, 1.0f);
}

// hllc_speeds with wet_blend for the two blend weights: the same values, bit for bit.
__device__ __forceinline__ void hllc_speeds_fast(const Phys &p, float hL, float unL, float hR, float unR, float &SLo,
                                                 float &SRo) {
    const float sqL = sqrtf(gmax(hL, 0.0f));
    const float sqR = sqrtf(gmax(hR, 0.0f));
    const float root_g = sqrtf(p.g);  // loop-invariant: hoisted out of the callers' edge loops
    const float cL = root_g * sqL;
    const float cR = root_g * sqR;
    const float den = sqL + sqR;
    const float u_roe = (den > 1e-12f) ? fmaf_rn(sqL, unL, sqR * unR) / den : 0.0f;
    const float c_roe = sqrtf(p.g * 0.5f * (hL + hR));
    const float SL = gmin(unL - cL, u_roe - c_roe);
    const float SR = gmax(unR + cR, u_roe + c_roe);
    const float wetL = wet_blend(p, hL);
    const float wetR = wet_blend(p, hR);
    const float dryLeft = (1.0f - wetL) * wetR;
    const float dryRight = (1.0f - wetR) * wetL;
    const float roe = 1.0f - dryLeft - dryRight;
    SLo = fmaf_rn(roe, SL, fmaf_rn(dryLeft, fmaf_rn(-2.0f, cR, unR), dryRight * (unL - cL)));
    SRo = fmaf_rn(roe, SR, fmaf_rn(dryLeft, unR + cR, dryRight * fmaf_rn(2.0f, cL, unL)));
}

// HLLC flux in the face frame (Toro 2001); smax is the largest speed assumed.
__device__ __forceinline__ void hllc(const Phys &p, float hL, float hqnL, float hqtL, float hR, float hqnR,
                                     float hqtR, float &Fh, float &Fhn, float &Fht, float &smax) {
    float unL, utL, unR, utR;
    safe_vel2(p, hL, hqnL, hqtL, unL, utL);
    safe_vel2(p, hR, hqnR, hqtR, unR, utR);
    float SL, SR;
    hllc_speeds_fast(p, hL, unL, hR, unR, SL, SR);
    smax = gmax(fabsf(SL), fabsf(SR));
    const float aR = hR * (unR - SR), aL = hL * (unL - SL);
    const float num_sm = fmaf_rn(SL, aR, -(SR * aL));
    const float den_sm = aR - aL;
    const float SM = (fabsf(den_sm) > 1e-12f) ? num_sm / den_sm : 0.0f;
    // The four regions (SL >= 0: left; SM >= 0: left star; SR >= 0: right star; else right)
    // share one side's plain flux and, in the star regions, one correction: the side is
    // selected first, so a warp whose edges fall in both star regions runs the star
    // arithmetic once, with the same operations on the same values as per region.
    const bool left = (SL >= 0.0f) || (SM >= 0.0f);
    const bool star = !(SL >= 0.0f) && (left || SR >= 0.0f);
    const float h = left ? hL : hR, un = left ? unL : unR, ut = left ? utL : utR;
    const float q = h * un;
    Fh = q;
    Fhn = fmaf_rn(q, un, 0.5f * p.g * h * h);
    Fht = q * ut;
    if (star) {
        const float S = left ? SL : SR;
        const float dS = S - SM;
        const float k = h * (S - un) / ((fabsf(dS) > 1e-14f) ? dS : 1e-14f);
        Fh = fmaf_rn(S, k - h, q);
        Fhn = fmaf_rn(S, fmaf_rn(k, SM, -q), Fhn);
        Fht = fmaf_rn(S, (k - h) * ut, Fht);
    }
}

// Audusse hydrostatic reconstruction: depths at the face elevation, momenta
// rebuilt from the cells' velocities, rotated into the face frame.
__device__ __forceinline__ void face_states(const Phys &p, float hL, float huL, float hvL, float dzL, float hR,
                                            float huR, float hvR, float dzR, float nx, float ny, float &hLs,
                                            float &hqnL, float &hqtL, float &hRs, float &hqnR, float &hqtR) {
    hLs = gmax(0.0f, hL - dzL);
    hRs = gmax(0.0f, hR - dzR);
    float uL, vL, uR, vR;
    safe_vel2(p, hL, huL, hvL, uL, vL);
    safe_vel2(p, hR, huR, hvR, uR, vR);
    const float huLs = hLs * uL, hvLs = hLs * vL, huRs = hRs * uR, hvRs = hRs * vR;
    hqnL = fmaf_rn(huLs, nx, hvLs * ny);
    hqtL = fmaf_rn(hvLs, nx, -(huLs * ny));
    hqnR = fmaf_rn(huRs, nx, hvRs * ny);
    hqtR = fmaf_rn(hvRs, nx, -(huRs * ny));
}

// The CFL wave speed the flux would assume on an edge.
__device__ __forceinline__ float wave_bound(const Phys &p, float hL, float huL, float hvL, float dzL, float hR,
                                            float huR, float hvR, float dzR, float nx, float ny) {
    float hLs, hqnL, hqtL, hRs, hqnR, hqtR, SL, SR;
    face_states(p, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx, ny, hLs, hqnL, hqtL, hRs, hqnR, hqtR);
    hllc_speeds(p, hLs, safe_vel(p, hLs, hqnL), hRs, safe_vel(p, hRs, hqnR), SL, SR);
    return gmax(fabsf(SL), fabsf(SR));
}

// Wall ghost: the left state mirrored in the normal direction.
__device__ __forceinline__ void wall_mirror(float huL, float hvL, float nx, float ny, float &huR, float &hvR) {
    const float twice = -2.0f * fmaf_rn(huL, nx, hvL * ny);
    huR = fmaf_rn(twice, nx, huL);
    hvR = fmaf_rn(twice, ny, hvL);
}

// -- open boundaries (flux.py:187-294) ----------------------------------------------------------
// Open edge k has cR = -2 - k; its condition is the word pair (kind, value bits).
constexpr uint32_t kOpenWall = 0u, kOpenFree = 1u, kOpenNormal = 2u, kOpenStage = 3u, kOpenInflow = 4u;
constexpr int kOpenNewtonSteps = 4;

// Cube root of x >= 0 by Newton's iteration r <- (2r + x/r^2)/3 from the exponent-thirds
// estimate, four steps (no fixed-rounding pow is assumed; this is one value GLSL's
// pow(x, 1/3) admits).
__device__ __forceinline__ float cbrt_newton(float x) {
    if (!(x > 0.0f)) return 0.0f;
    float r = __uint_as_float(__float_as_uint(x) / 3u + 0x2A555555u);
#pragma unroll
    for (int k = 0; k < 4; ++k) r = (2.0f * r + x / (r * r)) / 3.0f;
    return r;
}

// Depth beyond an inflow edge of discharge q per unit width: the root of
// -q/hG + 2 sqrt(g hG) = riemann (the outgoing characteristic), by Newton in s = sqrt(hG).
__device__ __forceinline__ float inflow_depth(const Phys &p, float q, float riemann) {
    const float root_g = sqrtf(p.g);
    float s = gmax(cbrt_newton(q / (2.0f * root_g)), riemann / (2.0f * root_g));
    for (int k = 0; k < kOpenNewtonSteps; ++k) {
        const float f = 2.0f * root_g * s - q / (s * s) - riemann;
        const float df = 2.0f * root_g + 2.0f * q / (s * s * s);
        s = gmax(s - f / df, 0.5f * s);
    }
    return s * s;
}

// The state beyond an open edge of condition `kind` from the cell inside it.
// value: sqrt(S)/n for NORMAL, the depth over this cell's bed for STAGE, the
// discharge per unit width for INFLOW.
__device__ __forceinline__ void ghost_state(const Phys &p, uint32_t kind, float value, float hL, float huL, float hvL,
                                            float nx, float ny, float &hG, float &huG, float &hvG) {
    const float uL = safe_vel(p, hL, huL);
    const float vL = safe_vel(p, hL, hvL);
    const float unL = uL * nx + vL * ny;
    float ut = -uL * ny + vL * nx;
    const float cL = sqrtf(p.g * gmax(hL, 0.0f));
    float un = -unL;
    hG = hL;
    if (kind == kOpenFree) {
        un = fabsf(unL);
    } else if (kind == kOpenNormal) {
        const float r = cbrt_newton(gmax(hL, 0.0f));
        un = value * (r * r);
    } else if (kind == kOpenStage) {
        if (hL < p.dry_tol || unL < cL) {
            hG = value;
            un = unL + 2.0f * (cL - sqrtf(p.g * value));
        } else {
            un = unL;
        }
    } else if (kind == kOpenInflow && value > 0.0f) {
        hG = inflow_depth(p, value, unL + 2.0f * cL);
        un = -value / hG;
        ut = 0.0f;
    }
    huG = hG * (un * nx - ut * ny);
    hvG = hG * (un * ny + ut * nx);
}

// An inflow keeps its edge live while dry, or its volume would be lost.
__device__ __forceinline__ bool open_forced(uint32_t kind, float value) { return kind == kOpenInflow && value > 0.0f; }

// Mass flux through a boundary edge: outflow conditions never draw water in,
// inflow carries exactly its discharge, a wall passes none.
__device__ __forceinline__ float boundary_mass_flux(uint32_t kind, float value, float Fh) {
    if (kind == kOpenFree || kind == kOpenNormal) return gmax(Fh, 0.0f);
    if (kind == kOpenStage) return Fh;
    if (kind == kOpenInflow) return -value;
    return 0.0f;
}

// Semi-implicit momentum decay factor of a thin film (a rate, independent of the tick).
__device__ __forceinline__ float film_drag(const Phys &p, float h, float dt) {
    const float e = kFilmDepths * p.dry_tol;
    if (h >= e) return 1.0f;
    const float rate = (e * e - h * h) / (2.0f * h * h) * sqrtf(p.g / e);
    return 1.0f / (1.0f + dt * rate);
}

// Knuth's two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    const float t = a + b;
    const float bb = t - a;
    e = (a - (t - bb)) + (b - bb);
    s = t;
}

// (hi + lo) + inc as a renormalised pair, clamped at zero.
__device__ __forceinline__ void add_compensated(float hi, float lo, float inc, float &h_new, float &lo_new) {
    float s, e;
    two_sum(hi, inc, s, e);
    e += lo;
    two_sum(s, e, h_new, lo_new);
    if (h_new < 0.0f || (h_new == 0.0f && lo_new < 0.0f)) {
        h_new = 0.0f;
        lo_new = 0.0f;
    }
}

}  // namespace swe
