/*
 * FP32 oracle of the reference's GPU-resident shallow-water kernels.
 * TEST INFRASTRUCTURE ONLY: the checker, never the product. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline arm load it.
 *
 * A literal, sequential C restatement of the GLSL compute kernels of the
 * reference's resident backend, on the reference's own data layout (edges
 * sorted by the block of their left cell, a 6-word per-edge flux buffer, the
 * remapped signed CSR, per-block flag words {wet, active, forced}):
 *
 *   safe_vel, hllc_speeds, hllc, face_states, wave_bound
 *       inundation/vulkan/shaders/flux.py:63-182
 *   film_drag                      flux.py:46-51
 *   two_sum, add_compensated       flux.py:301-319
 *   flux_resident_gather           resident.py:187-291 (wall ghost :125-146, words :165-184)
 *   update_resident_gather[_comp]  resident.py:401-513 (sum :312-344, depth :359-398)
 *   source_resident                resident.py:665-730
 *   block_mark, block_dilate       resident.py:738-802
 *   cfl_edge_gather, cfl_gather    resident.py:528-607
 *   step_control                   resident.py:813-882
 *   open_ghost, inflow_depth, boundary_mass_flux, outflow-only redo
 *                                  flux.py:187-294, resident.py:127-145
 *   tally_resident                 resident.py:617-660, one pair per open
 *                                  edge as the reference's base solver keeps
 *                                  them (inundation/vulkan/solver.py:432-440)
 *
 * Every expression is evaluated in a stated order, the same as the CUDA
 * kernels': it is compiled with -ffp-contract=off, so the only fused
 * multiply-adds are the explicit fmaf() calls, at the kernels' sites (GLSL
 * contracts a*b+c freely outside `precise` blocks, so a fused site is a value
 * the reference admits; C's fmaf and CUDA's __fmaf_rn both round once).
 * GLSL min/max/clamp are spelled out with their specified comparisons
 * (min(x,y) = y<x ? y : x, max(x,y) = x<y ? y : x). GLSL's pow has no fixed
 * rounding, so the friction's h^(-4/3) is evaluated by the kernels'
 * division-free Newton sequence (inv_pow43 below), and sqrt(g h) as
 * sqrt(g) sqrt(h): values the reference admits, bit-identical to the
 * product's.
 *
 * One deliberate choice: the GLSL source kernel reads a neighbour's depth
 * while that neighbour's own source may be adding to it (a race in the
 * reference). Here all sources are added first and the post-source bounds
 * are taken after, which is one of the outcomes the reference allows.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define EF_WORDS 6u
#define EF_CFL 5u
#define BLK_WORDS 3u
#define BLK_WET 0u
#define BLK_ACTIVE 1u
#define BLK_FORCED 2u
#define FILM_DEPTHS 4.0f
#define TICKS_PER_SECOND 1048576.0f
#define DT_SENTINEL 1e30f

typedef struct {
    uint64_t now_ticks;
    uint64_t stop_ticks;
    uint64_t steps;
    uint32_t dt_ticks;
    uint32_t dt_max_ticks;
    uint32_t dry_dt_ticks;
    float last_raw;
    float cfl_safety;
    uint32_t pad;
} ctrl_t;

/* Everything one resident solver holds, in the reference's layout. */
typedef struct {
    uint32_t N, E, n_blocks;
    float g, dry_tol, cfl;
    const int32_t *ecL, *ecR;
    const float *enx, *eny, *elen, *edz; /* edz: (dzL, dzR) pairs */
    const float *area, *n_mann;
    const uint32_t *cptr, *cidx;
    const uint32_t *erange; /* (first, last) left-cell block per 256-edge workgroup */
    const uint32_t *bptr, *bidx; /* block two-ring */
    float *h, *hu, *hv, *h1, *hu1, *hv1, *h_lo, *h1_lo;
    float *ef;
    uint32_t *touched;
    uint32_t *blk;
    uint32_t *dt_buf; /* [0] this step's dt bits, [1] next step's CFL bound bits */
    float *clamp_mass;
    ctrl_t *ctrl;
    /* Inflow hydrographs of the sources (src_hydro NULL: constant rates). */
    const uint32_t *src_hydro;
    const float *src_hscale;
    const uint32_t *knot_ptr;
    const float *knot_t;
    const float *knot_q;
    /* Open edges: right cell -2 - k is open edge k, with condition words
       open_cond[2k] (kind) and open_cond[2k + 1] (value bits); open_vol holds
       4 words per open edge (out hi, lo, in hi, lo). NULL without open edges. */
    const uint32_t *open_cond;
    float *open_vol;
} oracle_t;

static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline float gmin(float x, float y) { return (y < x) ? y : x; }
static inline float gmax(float x, float y) { return (x < y) ? y : x; }
static inline float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }

/* Divisions: GLSL divides to within 2.5 ulp, so a product by a correctly
   rounded reciprocal (or by the float 1/3) is a quotient the reference
   admits. Quotients that share a denominator use one reciprocal, in the
   same expressions as the CUDA kernels. */
static const float ONE_THIRD = 1.0f / 3.0f;

/* x^(-4/3) for x > 0 without a division: y = x^(-1/3) by Newton's iteration
   for 1/y^3 = x, y <- y + (y/3)(1 - x y^3), from the exponent-thirds estimate
   bits(y) = (4/3)*127*2^23 - bits(x)/3, four steps; then (y^2)^2. Multiplies
   and fused multiply-adds only. */
static float inv_pow43(float x) {
    float y = bitsf(0x54AAAAAAu - fbits(x) / 3u);
    for (int k = 0; k < 4; ++k) {
        float t = x * (y * y);
        y = fmaf(y * ONE_THIRD, fmaf(-t, y, 1.0f), y);
    }
    float y2 = y * y;
    return y2 * y2;
}

static float safe_vel(const oracle_t *o, float h_, float hq) {
    float e_ = FILM_DEPTHS * o->dry_tol;
    return (h_ > o->dry_tol) ? 2.0f * h_ * hq / (h_ * h_ + gmax(h_ * h_, e_ * e_)) : 0.0f;
}

/* safe_vel of two momenta of one depth, with one reciprocal of their denominator. */
static void safe_vel2(const oracle_t *o, float h_, float hq1, float hq2, float *v1, float *v2) {
    if (h_ > o->dry_tol) {
        float e_ = FILM_DEPTHS * o->dry_tol;
        float inv = 1.0f / (h_ * h_ + gmax(h_ * h_, e_ * e_));
        *v1 = 2.0f * h_ * hq1 * inv;
        *v2 = 2.0f * h_ * hq2 * inv;
    } else {
        *v1 = 0.0f;
        *v2 = 0.0f;
    }
}

static void hllc_speeds(const oracle_t *o, float hL, float unL, float hR, float unR, float *SLo, float *SRo) {
    float g = o->g;
    float sqL = sqrtf(gmax(hL, 0.0f));
    float sqR = sqrtf(gmax(hR, 0.0f));
    float root_g = sqrtf(g);
    float cL = root_g * sqL;
    float cR = root_g * sqR;
    float den = sqL + sqR;
    float u_roe = (den > 1e-12f) ? fmaf(sqL, unL, sqR * unR) / den : 0.0f;
    float c_roe = sqrtf(g * 0.5f * (hL + hR));
    float SL = gmin(unL - cL, u_roe - c_roe);
    float SR = gmax(unR + cR, u_roe + c_roe);
    float wetL = gclamp(hL / o->dry_tol - 1.0f, 0.0f, 1.0f);
    float wetR = gclamp(hR / o->dry_tol - 1.0f, 0.0f, 1.0f);
    float dryLeft = (1.0f - wetL) * wetR;
    float dryRight = (1.0f - wetR) * wetL;
    float roe = 1.0f - dryLeft - dryRight;
    *SLo = fmaf(roe, SL, fmaf(dryLeft, fmaf(-2.0f, cR, unR), dryRight * (unL - cL)));
    *SRo = fmaf(roe, SR, fmaf(dryLeft, unR + cR, dryRight * fmaf(2.0f, cL, unL)));
}

static void hllc(const oracle_t *o, float hL, float hqnL, float hqtL, float hR, float hqnR, float hqtR,
                 float *Fh, float *Fhn, float *Fht, float *Smax) {
    float g = o->g;
    float unL, utL, unR, utR;
    safe_vel2(o, hL, hqnL, hqtL, &unL, &utL);
    safe_vel2(o, hR, hqnR, hqtR, &unR, &utR);
    float SL, SR;
    hllc_speeds(o, hL, unL, hR, unR, &SL, &SR);
    *Smax = gmax(fabsf(SL), fabsf(SR));
    float aR = hR * (unR - SR), aL = hL * (unL - SL);
    float num_sm = fmaf(SL, aR, -(SR * aL));
    float den_sm = aR - aL;
    float SM = (fabsf(den_sm) > 1e-12f) ? num_sm / den_sm : 0.0f;
    float FL_h = hL * unL;
    float FL_hn = fmaf(FL_h, unL, 0.5f * g * hL * hL);
    float FL_ht = FL_h * utL;
    float FR_h = hR * unR;
    float FR_hn = fmaf(FR_h, unR, 0.5f * g * hR * hR);
    float FR_ht = FR_h * utR;
    float dSL = SL - SM, dSR = SR - SM;
    float kL = hL * (SL - unL) / ((fabsf(dSL) > 1e-14f) ? dSL : 1e-14f);
    float kR = hR * (SR - unR) / ((fabsf(dSR) > 1e-14f) ? dSR : 1e-14f);
    float FsL_h = fmaf(SL, kL - hL, FL_h);
    float FsL_hn = fmaf(SL, fmaf(kL, SM, -FL_h), FL_hn);
    float FsL_ht = fmaf(SL, (kL - hL) * utL, FL_ht);
    float FsR_h = fmaf(SR, kR - hR, FR_h);
    float FsR_hn = fmaf(SR, fmaf(kR, SM, -FR_h), FR_hn);
    float FsR_ht = fmaf(SR, (kR - hR) * utR, FR_ht);
    if (SL >= 0.0f) { *Fh = FL_h; *Fhn = FL_hn; *Fht = FL_ht; }
    else if (SM >= 0.0f) { *Fh = FsL_h; *Fhn = FsL_hn; *Fht = FsL_ht; }
    else if (SR >= 0.0f) { *Fh = FsR_h; *Fhn = FsR_hn; *Fht = FsR_ht; }
    else { *Fh = FR_h; *Fhn = FR_hn; *Fht = FR_ht; }
}

static void face_states(const oracle_t *o, float hL, float huL, float hvL, float dzL, float hR, float huR,
                        float hvR, float dzR, float nx_, float ny_, float *hLs, float *hqnL, float *hqtL,
                        float *hRs, float *hqnR, float *hqtR) {
    *hLs = gmax(0.0f, hL - dzL);
    *hRs = gmax(0.0f, hR - dzR);
    float uL, vL, uR, vR;
    safe_vel2(o, hL, huL, hvL, &uL, &vL);
    safe_vel2(o, hR, huR, hvR, &uR, &vR);
    float huLs = *hLs * uL, hvLs = *hLs * vL, huRs = *hRs * uR, hvRs = *hRs * vR;
    *hqnL = fmaf(huLs, nx_, hvLs * ny_);
    *hqtL = fmaf(hvLs, nx_, -(huLs * ny_));
    *hqnR = fmaf(huRs, nx_, hvRs * ny_);
    *hqtR = fmaf(hvRs, nx_, -(huRs * ny_));
}

static float wave_bound(const oracle_t *o, float hL, float huL, float hvL, float dzL, float hR, float huR,
                        float hvR, float dzR, float nx_, float ny_) {
    float hLs, hqnL, hqtL, hRs, hqnR, hqtR, SL, SR;
    face_states(o, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx_, ny_, &hLs, &hqnL, &hqtL, &hRs, &hqnR, &hqtR);
    hllc_speeds(o, hLs, safe_vel(o, hLs, hqnL), hRs, safe_vel(o, hRs, hqnR), &SL, &SR);
    return gmax(fabsf(SL), fabsf(SR));
}

static float film_drag(const oracle_t *o, float h_, float dt_) {
    float e_ = FILM_DEPTHS * o->dry_tol;
    if (h_ >= e_) return 1.0f;
    float rate = (e_ * e_ - h_ * h_) / (2.0f * h_ * h_) * sqrtf(o->g / e_);
    return 1.0f / (1.0f + dt_ * rate);
}

static void two_sum(float a, float b, float *s, float *e) {
    float t = a + b;
    float bb = t - a;
    float err = (a - (t - bb)) + (b - bb);
    *s = t;
    *e = err;
}

static void add_compensated(float hi, float loi, float inc, float *h_new, float *lo_new) {
    float s, e;
    two_sum(hi, inc, &s, &e);
    e += loi;
    two_sum(s, e, h_new, lo_new);
    if (*h_new < 0.0f || (*h_new == 0.0f && *lo_new < 0.0f)) { *h_new = 0.0f; *lo_new = 0.0f; }
}

/* ---- open boundaries (flux.py:187-294) ---------------------------------------------------------- */
#define OPEN_WALL 0u
#define OPEN_FREE 1u
#define OPEN_NORMAL 2u
#define OPEN_STAGE 3u
#define OPEN_INFLOW 4u
#define OPEN_NEWTON_STEPS 4

/* x^(1/3) for x >= 0 by Newton's iteration r <- (2r + x/r^2)/3 from the
   exponent-thirds estimate, four steps: GLSL's pow(x, 1/3) has no fixed
   rounding, and this is a value it admits. */
static float cbrt_newton(float x) {
    if (!(x > 0.0f)) return 0.0f;
    float r = bitsf(fbits(x) / 3u + 0x2A555555u);
    for (int k = 0; k < 4; ++k) r = (2.0f * r + x / (r * r)) / 3.0f;
    return r;
}

static uint32_t open_kind(const oracle_t *o, int cR) { return o->open_cond[2u * (uint32_t)(-2 - cR)]; }
static float open_value(const oracle_t *o, int cR) { return bitsf(o->open_cond[2u * (uint32_t)(-2 - cR) + 1u]); }

static int open_forced(const oracle_t *o, int cR) {
    return cR < -1 && open_kind(o, cR) == OPEN_INFLOW && open_value(o, cR) > 0.0f;
}

/* hG solving -q/hG + 2 sqrt(g hG) = riemann, Newton in s = sqrt(hG). */
static float inflow_depth(const oracle_t *o, float q, float riemann) {
    float root_g = sqrtf(o->g);
    float s = gmax(cbrt_newton(q / (2.0f * root_g)), riemann / (2.0f * root_g));
    for (int k = 0; k < OPEN_NEWTON_STEPS; ++k) {
        float f = 2.0f * root_g * s - q / (s * s) - riemann;
        float df = 2.0f * root_g + 2.0f * q / (s * s * s);
        s = gmax(s - f / df, 0.5f * s);
    }
    return s * s;
}

static void ghost_state(const oracle_t *o, uint32_t kind, float value, float hL, float huL, float hvL, float nx_,
                        float ny_, float *hG, float *huG, float *hvG) {
    float uL = safe_vel(o, hL, huL);
    float vL = safe_vel(o, hL, hvL);
    float unL = uL * nx_ + vL * ny_;
    float ut = -uL * ny_ + vL * nx_;
    float cL = sqrtf(o->g * gmax(hL, 0.0f));
    float un = -unL;
    *hG = hL;
    if (kind == OPEN_FREE) {
        un = fabsf(unL);
    } else if (kind == OPEN_NORMAL) {
        float r = cbrt_newton(gmax(hL, 0.0f));
        un = value * (r * r);
    } else if (kind == OPEN_STAGE) {
        if (hL < o->dry_tol || unL < cL) {
            *hG = value;
            un = unL + 2.0f * (cL - sqrtf(o->g * value));
        } else {
            un = unL;
        }
    } else if (kind == OPEN_INFLOW && value > 0.0f) {
        *hG = inflow_depth(o, value, unL + 2.0f * cL);
        un = -value / *hG;
        ut = 0.0f;
    }
    *huG = *hG * (un * nx_ - ut * ny_);
    *hvG = *hG * (un * ny_ + ut * nx_);
}

static float boundary_mass_flux(uint32_t kind, float value, float Fh) {
    if (kind == OPEN_FREE || kind == OPEN_NORMAL) return gmax(Fh, 0.0f);
    if (kind == OPEN_STAGE) return Fh;
    if (kind == OPEN_INFLOW) return -value;
    return 0.0f;
}

/* The ghost probe of the reference's tests: per case (h, hu, hv, nx, ny, flux)
   and condition words, the ghost (h, hu, hv) and the boundary mass flux. */
void oracle_open_ghost(float g, float dry_tol, const float *cases, const uint32_t *cond, float *results, uint32_t n) {
    oracle_t o;
    memset(&o, 0, sizeof o);
    o.g = g;
    o.dry_tol = dry_tol;
    for (uint32_t k = 0; k < n; ++k) {
        const float *c = cases + 6u * k;
        float *r = results + 4u * k;
        float value = bitsf(cond[2u * k + 1u]);
        ghost_state(&o, cond[2u * k], value, c[0], c[1], c[2], c[3], c[4], &r[0], &r[1], &r[2]);
        r[3] = boundary_mass_flux(cond[2u * k], value, c[5]);
    }
}

static inline int block_active(const oracle_t *o, uint32_t b) { return o->blk[BLK_WORDS * b + BLK_ACTIVE] != 0u; }

static void load_state(const oracle_t *o, int stage, int c, float *h_, float *hu_, float *hv_) {
    if (stage && block_active(o, (uint32_t)c >> 8)) { *h_ = o->h1[c]; *hu_ = o->hu1[c]; *hv_ = o->hv1[c]; }
    else { *h_ = o->h[c]; *hu_ = o->hu[c]; *hv_ = o->hv[c]; }
}

void oracle_flux_stage(oracle_t *o, int stage) {
    if (o->dt_buf[0] == 0u) return;
    uint32_t n_wg = (o->E + 255u) / 256u;
    for (uint32_t wg = 0; wg < n_wg; ++wg) {
        int live = 0;
        for (uint32_t b = o->erange[2u * wg]; b <= o->erange[2u * wg + 1u]; ++b)
            if (block_active(o, b)) { live = 1; break; }
        if (!live) continue;
        uint32_t e_end = (wg + 1u) * 256u < o->E ? (wg + 1u) * 256u : o->E;
        for (uint32_t eid = wg * 256u; eid < e_end; ++eid) {
            int cL = o->ecL[eid], cR = o->ecR[eid];
            float nx_ = o->enx[eid], ny_ = o->eny[eid], len = o->elen[eid];
            float hL, huL, hvL, hR, huR, hvR;
            load_state(o, stage, cL, &hL, &huL, &hvL);
            if (cR == -1) {
                hR = hL;
                float twice = -2.0f * fmaf(huL, nx_, hvL * ny_);
                huR = fmaf(twice, nx_, huL);
                hvR = fmaf(twice, ny_, hvL);
            } else if (cR < 0) {
                ghost_state(o, open_kind(o, cR), open_value(o, cR), hL, huL, hvL, nx_, ny_, &hR, &huR, &hvR);
            } else {
                load_state(o, stage, cR, &hR, &huR, &hvR);
            }
            if (hL < o->dry_tol && hR < o->dry_tol && !open_forced(o, cR)) {
                /* an open edge clears its words instead, as the gather reads them */
                if (cR < -1) memset(o->ef + EF_WORDS * eid, 0, EF_WORDS * sizeof(float));
                continue;
            }
            float dzL = o->edz[2u * eid], dzR = o->edz[2u * eid + 1u];
            float hLs, hqnL, hqtL, hRs, hqnR, hqtR, Fh, Fhn, Fht, Smax;
            face_states(o, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx_, ny_, &hLs, &hqnL, &hqtL, &hRs, &hqnR, &hqtR);
            hllc(o, hLs, hqnL, hqtL, hRs, hqnR, hqtR, &Fh, &Fhn, &Fht, &Smax);
            if (cR < -1 && (open_kind(o, cR) == OPEN_FREE || open_kind(o, cR) == OPEN_NORMAL) && Fh < 0.0f) {
                /* an outflow-only edge drawing water in is a wall for this stage, momentum included */
                ghost_state(o, OPEN_WALL, 0.0f, hL, huL, hvL, nx_, ny_, &hR, &huR, &hvR);
                face_states(o, hL, huL, hvL, dzL, hR, huR, hvR, dzR, nx_, ny_, &hLs, &hqnL, &hqtL, &hRs, &hqnR, &hqtR);
                hllc(o, hLs, hqnL, hqtL, hRs, hqnR, hqtR, &Fh, &Fhn, &Fht, &Smax);
                Fh = 0.0f;
            } else if (cR < -1) {
                Fh = boundary_mass_flux(open_kind(o, cR), open_value(o, cR), Fh);
            } else if (cR < 0) {
                Fh = 0.0f; /* a wall passes no mass */
            }
            float Fhu = fmaf(Fhn, nx_, -(Fht * ny_));
            float Fhv = fmaf(Fhn, ny_, Fht * nx_);
            float SL_g = 0.5f * o->g * fmaf(hL, hL, -(hLs * hLs));
            float SR_g = 0.5f * o->g * fmaf(hR, hR, -(hRs * hRs));
            o->touched[cL] = 1u;
            if (cR >= 0) o->touched[cR] = 1u;
            float *w = o->ef + EF_WORDS * eid;
            w[0] = Fh * len;
            w[1] = fmaf(SL_g, nx_, Fhu) * len;
            w[2] = fmaf(SL_g, ny_, Fhv) * len;
            w[3] = fmaf(SR_g, nx_, Fhu) * len;
            w[4] = fmaf(SR_g, ny_, Fhv) * len;
            if (stage) w[EF_CFL] = Smax * len;
        }
    }
}

/* Volume through every open edge after one flux stage: dt/2 of its mass word
   into its out or in pair, skipping edges whose block is inactive (their
   words are stale). */
void oracle_tally(oracle_t *o) {
    if (o->dt_buf[0] == 0u || !o->open_vol) return;
    float half_dt = 0.5f * bitsf(o->dt_buf[0]);
    for (uint32_t e = 0; e < o->E; ++e) {
        int cR = o->ecR[e];
        if (cR >= -1) continue;
        if (!block_active(o, (uint32_t)o->ecL[e] >> 8)) continue;
        float v = half_dt * o->ef[EF_WORDS * e];
        float *t = o->open_vol + 4u * (uint32_t)(-2 - cR) + ((v < 0.0f) ? 2u : 0u);
        float s, err, hi, lo;
        two_sum(t[0], fabsf(v), &s, &err);
        err += t[1];
        two_sum(s, err, &hi, &lo);
        t[0] = hi;
        t[1] = lo;
    }
}

void oracle_update_stage(oracle_t *o, int stage, int compensated, int track_clamp) {
    if (o->dt_buf[0] == 0u) return;
    for (uint32_t i = 0; i < o->N; ++i) {
        uint32_t b = i >> 8;
        if (!block_active(o, b)) continue;
        if (!stage && (i & 255u) == 0u) o->blk[BLK_WORDS * b + BLK_WET] = 0u;
        float A = o->area[i];
        float dt = bitsf(o->dt_buf[0]);
        float dti = dt / A;
        float hi, hui, hvi;
        if (!stage) { hi = o->h[i]; hui = o->hu[i]; hvi = o->hv[i]; }
        else { hi = o->h1[i]; hui = o->hu1[i]; hvi = o->hv1[i]; }
        float sdh = 0.0f, sdhu = 0.0f, sdhv = 0.0f, lam = 0.0f;
        uint32_t kend = o->cptr[i];
        if (o->touched[i] != 0u) { o->touched[i] = 0u; kend = o->cptr[i + 1u]; }
        int own_dry = hi < o->dry_tol;
        for (uint32_t k = o->cptr[i]; k < kend; ++k) {
            uint32_t s = o->cidx[k], e = s >> 1;
            int right = (s & 1u) != 0u;
            if (own_dry) {
                int nb = right ? o->ecL[e] : o->ecR[e];
                if (nb == -1) continue;
                if (nb >= 0) {
                    int pred = stage && block_active(o, (uint32_t)nb >> 8);
                    if ((pred ? o->h1[nb] : o->h[nb]) < o->dry_tol) continue;
                }
            }
            const float *w = o->ef + EF_WORDS * e;
            if (right) { sdh -= w[0]; sdhu -= w[3]; sdhv -= w[4]; }
            else { sdh += w[0]; sdhu += w[1]; sdhv += w[2]; }
            if (stage) lam += w[EF_CFL];
        }
        float h_new, lo_new, h_raw;
        if (compensated) {
            float loi = !stage ? o->h_lo[i] : o->h1_lo[i];
            add_compensated(hi, loi, -dti * sdh, &h_new, &lo_new);
            float s_raw, e_raw;
            two_sum(hi, -dti * sdh, &s_raw, &e_raw);
            h_raw = s_raw + (e_raw + loi);
        } else {
            h_raw = hi - dti * sdh;
            h_new = gmax(h_raw, 0.0f);
            lo_new = 0.0f;
        }
        float hu_new = fmaf(-dti, sdhu, hui);
        float hv_new = fmaf(-dti, sdhv, hvi);
        if (track_clamp) o->clamp_mass[i] += 0.5f * A * (h_new - h_raw);
        if (h_new < o->dry_tol) { hu_new = 0.0f; hv_new = 0.0f; }
        if (h_new >= o->dry_tol) {
            float drag = film_drag(o, h_new, dt);
            hu_new *= drag;
            hv_new *= drag;
        }
        if (h_new >= o->dry_tol) {
            float n = o->n_mann[i];
            float inv_h = 1.0f / h_new;
            float u_ = hu_new * inv_h, v_ = hv_new * inv_h;
            float spd = sqrtf(fmaf(u_, u_, v_ * v_));
            float Sf = o->g * n * n * spd * inv_pow43(h_new);
            float inv_den = 1.0f / fmaf(dt, Sf, 1.0f);
            hu_new = hu_new * inv_den;
            hv_new = hv_new * inv_den;
        }
        float hf = 0.0f;
        if (compensated) {
            if (!stage) { o->h1[i] = h_new; o->h1_lo[i] = lo_new; }
            else {
                float s, e, lof;
                two_sum(o->h[i], h_new, &s, &e);
                e += o->h_lo[i] + lo_new;
                two_sum(0.5f * s, 0.5f * e, &hf, &lof);
                o->h[i] = hf;
                o->h_lo[i] = lof;
            }
        } else {
            if (!stage) o->h1[i] = h_new;
            else { hf = 0.5f * (o->h[i] + h_new); o->h[i] = hf; }
        }
        if (!stage) { o->hu1[i] = hu_new; o->hv1[i] = hv_new; }
        else {
            float huf = 0.5f * (o->hu[i] + hu_new);
            float hvf = 0.5f * (o->hv[i] + hv_new);
            if (hf < o->dry_tol) { huf = 0.0f; hvf = 0.0f; }
            o->hu[i] = huf;
            o->hv[i] = hvf;
            if (hf >= o->dry_tol) o->blk[BLK_WORDS * b + BLK_WET] = 1u;
            if (lam > 1e-30f && A > 1e-10f) {
                uint32_t v = fbits(o->cfl * A / lam);
                if (v < o->dt_buf[1]) o->dt_buf[1] = v;
            }
        }
    }
}

/* Sources as (cell, dh/dt) pairs: all increments first, then the bounds. */
/* A source's hydrograph value at clock t (seconds): piecewise linear between
   the knots, the end values outside them. Not in the reference, whose inflows
   are constant per phase; the product evaluates the same expression at the
   start of every step, t = now_ticks / 2^20 rounded to float. */
static float hydrograph_at(const oracle_t *o, uint32_t j, float t) {
    uint32_t k0 = o->knot_ptr[j], k1 = o->knot_ptr[j + 1u];
    if (k1 <= k0) return 0.0f;
    if (!(t > o->knot_t[k0])) return o->knot_q[k0];
    if (!(t < o->knot_t[k1 - 1u])) return o->knot_q[k1 - 1u];
    uint32_t k = k0;
    while (k + 2u < k1 && !(t < o->knot_t[k + 1u])) ++k;
    float t0 = o->knot_t[k], t1 = o->knot_t[k + 1u];
    float q0 = o->knot_q[k], q1 = o->knot_q[k + 1u];
    return q0 + (q1 - q0) * ((t - t0) / (t1 - t0));
}

void oracle_sources(oracle_t *o, const uint32_t *cells, const float *rate, uint32_t count, int compensated) {
    if (o->dt_buf[0] == 0u) return;
    float dt = bitsf(o->dt_buf[0]);
    float t = (float)o->ctrl->now_ticks * (1.0f / 1048576.0f);
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t i = cells[k];
        float r = rate[k];
        if (o->src_hydro && o->src_hydro[k] != 0xFFFFFFFFu) r = r + o->src_hscale[k] * hydrograph_at(o, o->src_hydro[k], t);
        float inc = dt * r;
        float h_new;
        if (compensated) {
            float lo_new;
            add_compensated(o->h[i], o->h_lo[i], inc, &h_new, &lo_new);
            o->h_lo[i] = lo_new;
        } else {
            h_new = gmax(o->h[i] + inc, 0.0f);
        }
        o->h[i] = h_new;
        if (h_new >= o->dry_tol) o->blk[BLK_WORDS * (i >> 8) + BLK_WET] = 1u;
    }
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t i = cells[k];
        float h_new = o->h[i];
        if (!(h_new >= o->dry_tol)) continue;
        float u = sqrtf(o->hu[i] * o->hu[i] + o->hv[i] * o->hv[i]) / h_new;
        float c = sqrtf(o->g * h_new);
        float lam = 0.0f;
        for (uint32_t q = o->cptr[i]; q < o->cptr[i + 1u]; ++q) {
            uint32_t s = o->cidx[q], e = s >> 1;
            int nb = (s & 1u) ? o->ecL[e] : o->ecR[e];
            int dry_side = nb >= 0 && o->h[nb] < o->dry_tol;
            lam += (u + (dry_side ? 2.0f : 1.0f) * c) * o->elen[e];
        }
        if (lam > 1e-30f && o->area[i] > 1e-10f) {
            uint32_t v = fbits(o->cfl * o->area[i] / lam);
            if (v < o->dt_buf[1]) o->dt_buf[1] = v;
        }
    }
}

void oracle_block_mark(oracle_t *o, int all_active) {
    for (uint32_t b = 0; b < o->n_blocks; ++b) {
        if (all_active) { o->blk[BLK_WORDS * b + BLK_WET] = 0u; o->blk[BLK_WORDS * b + BLK_ACTIVE] = 1u; continue; }
        uint32_t first = b << 8, last = first + 256u < o->N ? first + 256u : o->N, live = 0u;
        for (uint32_t i = first; i < last; ++i)
            if (o->h[i] >= o->dry_tol || o->hu[i] != 0.0f || o->hv[i] != 0.0f) { live = 1u; break; }
        o->blk[BLK_WORDS * b + BLK_WET] = live;
    }
}

void oracle_block_dilate(oracle_t *o, int force) {
    if (!force && o->dt_buf[0] == 0u) return;
    for (uint32_t b = 0; b < o->n_blocks; ++b) {
        uint32_t v = o->blk[BLK_WORDS * b + BLK_WET] | o->blk[BLK_WORDS * b + BLK_FORCED];
        for (uint32_t k = o->bptr[b]; v == 0u && k < o->bptr[b + 1u]; ++k)
            v = o->blk[BLK_WORDS * o->bidx[k] + BLK_WET] | o->blk[BLK_WORDS * o->bidx[k] + BLK_FORCED];
        o->blk[BLK_WORDS * b + BLK_ACTIVE] = v;
    }
}

void oracle_cfl_prologue(oracle_t *o) {
    o->dt_buf[0] = fbits(DT_SENTINEL);
    for (uint32_t eid = 0; eid < o->E; ++eid) {
        int cL = o->ecL[eid], cR = o->ecR[eid];
        float nx_ = o->enx[eid], ny_ = o->eny[eid];
        float hL = o->h[cL], huL = o->hu[cL], hvL = o->hv[cL], hR, huR, hvR;
        if (cR == -1) {
            hR = hL;
            huR = huL - 2.0f * (huL * nx_ + hvL * ny_) * nx_;
            hvR = hvL - 2.0f * (huL * nx_ + hvL * ny_) * ny_;
        } else if (cR < 0) {
            ghost_state(o, open_kind(o, cR), open_value(o, cR), hL, huL, hvL, nx_, ny_, &hR, &huR, &hvR);
        } else { hR = o->h[cR]; huR = o->hu[cR]; hvR = o->hv[cR]; }
        float contrib = 0.0f;
        if (hL >= o->dry_tol || hR >= o->dry_tol)
            contrib = wave_bound(o, hL, huL, hvL, o->edz[2u * eid], hR, huR, hvR, o->edz[2u * eid + 1u], nx_, ny_) * o->elen[eid];
        o->ef[EF_WORDS * eid + EF_CFL] = contrib;
    }
    for (uint32_t i = 0; i < o->N; ++i) {
        float lam = 0.0f;
        for (uint32_t k = o->cptr[i]; k < o->cptr[i + 1u]; ++k) lam += o->ef[EF_WORDS * (o->cidx[k] >> 1) + EF_CFL];
        if (lam > 1e-30f && o->area[i] > 1e-10f) {
            uint32_t v = fbits(o->cfl * o->area[i] / lam);
            if (v < o->dt_buf[0]) o->dt_buf[0] = v;
        }
    }
}

/* mode 0 = START, 1 = STEP, 2 = RETARGET. */
void oracle_step_control(ctrl_t *c, uint32_t *dt_buf, int mode) {
    float raw;
    if (mode == 0) { raw = bitsf(dt_buf[0]); c->last_raw = raw; }
    else if (mode == 1) {
        uint32_t done = c->dt_ticks;
        c->now_ticks += (uint64_t)done;
        if (done > 0u) { c->steps += 1u; raw = bitsf(dt_buf[1]); c->last_raw = raw; }
        else raw = c->last_raw;
    } else raw = c->last_raw;
    uint64_t remaining = c->stop_ticks > c->now_ticks ? c->stop_ticks - c->now_ticks : 0u;
    uint32_t ticks;
    if (remaining == 0u || raw < 1e-10f || raw != raw) ticks = 0u;
    else if (raw >= 1e10f) ticks = c->dry_dt_ticks;
    else {
        float cap = (float)c->dt_max_ticks / TICKS_PER_SECOND;
        ticks = (uint32_t)(gmin(raw * c->cfl_safety, cap) * TICKS_PER_SECOND);
    }
    if (c->dt_max_ticks < ticks) ticks = c->dt_max_ticks;
    if ((uint64_t)ticks > remaining) ticks = (uint32_t)remaining;
    c->dt_ticks = ticks;
    dt_buf[0] = fbits((float)ticks / TICKS_PER_SECOND);
    dt_buf[1] = fbits(DT_SENTINEL);
}

/* One whole resident step as the reference records it (gpu_resident_batch.py:489-513). */
void oracle_step(oracle_t *o, const uint32_t *src_cells, const float *src_rate, uint32_t n_src, int compensated,
                 int track_clamp, int active_set) {
    for (int stage = 0; stage < 2; ++stage) {
        oracle_flux_stage(o, stage);
        oracle_tally(o);
        oracle_update_stage(o, stage, compensated, track_clamp);
    }
    if (n_src) oracle_sources(o, src_cells, src_rate, n_src, compensated);
    if (active_set) oracle_block_dilate(o, 0);
    oracle_step_control(o->ctrl, o->dt_buf, 1);
}

float oracle_inv_pow43(float x) { return inv_pow43(x); }

void oracle_hllc(float g, float dry_tol, const float *in6, float *out4) {
    oracle_t o;
    memset(&o, 0, sizeof o);
    o.g = g;
    o.dry_tol = dry_tol;
    hllc(&o, in6[0], in6[1], in6[2], in6[3], in6[4], in6[5], &out4[0], &out4[1], &out4[2], &out4[3]);
}

void oracle_hllc_speeds(float g, float dry_tol, const float *in4, float *out2) {
    oracle_t o;
    memset(&o, 0, sizeof o);
    o.g = g;
    o.dry_tol = dry_tol;
    hllc_speeds(&o, in4[0], in4[1], in4[2], in4[3], &out2[0], &out2[1]);
}

void oracle_two_sum(float a, float b, float *se) { two_sum(a, b, &se[0], &se[1]); }

size_t oracle_sizeof(void) { return sizeof(oracle_t); }
size_t oracle_ctrl_sizeof(void) { return sizeof(ctrl_t); }
