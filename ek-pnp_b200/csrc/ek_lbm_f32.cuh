// ek_lbm_f32.cuh -- node update of the shifted-storage forms (FP32 and FP16
// populations, FP32 arithmetic).  Included by the single-channel kernels
// (ek_lbm_f32.cu) and the batched persistent kernel (ek_batch.cu).
//
// Storage: d_i = f_i - w_i*R with R = R_s(y) a per-row reference density of
// species s (fluid, c+, c-) at the row where the value is stored.  R_s(y) =
// 36 K 2^-q for integers K, so the change of frame when a population is pulled
// from row y' to row y, d += w_i (R_s(y') - R_s(y)) = (16|4|1) (K' - K) 2^-q, is
// exact in FP32; the profiles follow the fields' row means (set at
// initialisation, re-based on request).  Every quantity of the collision is
// rewritten in deviations so that FP32 keeps the small departures:
//   dens = R + sum_i d_i,  j = sum_i c_i d_i  (sum_i w_i c_i = 0)
//   deq_i = w_i*(d_dens + dens*A_i),  A_i = cu_i*(1 + cu_i/2) - u^2/(2 cs2)
//   TRT:  s = (d_i + d_ibar)/2, a = (d_i - d_ibar)/2,
//         out_i = d_i - w+ (s - seq) - w- (a - aeq), out_ibar = d_ibar - w+(..) + w-(..)
//   Guo source (LBM.cu:556-756) split as F+_i = w_i(-u.F/cs2 + cu_i cF_i),
//         F-_i = w_i cF_i,  cF_i = (c_i.F)/(cfl cs2),  src_i = sp F+_i + sm F-_i
// The physics, wall treatment and step order are those of the FP64 form
// (ek_lbm_f64.cu, which cites the reference lines); only the number format
// and the algebraic form of the collision differ.
//
// Arithmetic: FP32 throughout the collision.  Two places where plain FP32
// would keep a systematic error, and what this form does there:
//  * In the double layer the y-force is 1e3-1e4 times the x-force and the
//    diagonal populations carry both.  Sums such as g_x + g_y, or the
//    momentum (t5 + t8) - (t6 + t7), round the x-part at the scale of the
//    y-part, with the same rounding every step (a bias, not noise: u_x off by
//    3e-5 of its max and the plug velocity by 20% after 10,000 steps of the
//    4096 x 1024 channel).  So the diagonals collide in x/y-separated moments:
//    X = (t5 - t6) + (t8 - t7) (the two differences of values streamed from
//    one row are exact by Sterbenz), Y, the diagonal mass S and the xy-moment
//    Q relax separately and the x-force enters X alone; only the final
//    populations round at the scale of the y-part, once, as a store would.
//  * The ion anti-bounce-back wall (gpu_bc_charge, LBM.cu:908-1024) makes each
//    wall node an undamped period-2 oscillator: its density alternates
//    between rho_0 and 2 c_w - rho_0 (1 and 108 from the noisy start at
//    zeta = -4), so deviations from any fixed reference are large and their
//    rounding never decays.  The wall nodes' ion populations are therefore
//    kept against a per-x frame that alternates with the ping-pong buffer,
//    F_a ~ rho_0 and F_b ~ 2 c_w - F_a (both on the species' dyadic grid):
//    in these frames the anti-bounce-back is an exact reflection of the
//    deviations plus w_i (2 c_w - F_a - F_b), a sub-grid constant.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ek_internal.h"

namespace ek {

// FP32 constants of one channel.
struct ChanF {
    int nx, ny, nxp, flags;
    size_t plane;                    // population and field plane size (elements)
    float wp, wm, wcp, wcm, wtp, wtm, sp, sm;
    float kcu;                       // 1/(cs2*cfl): cu_i = (c_i.u)*kcu
    float hinvcs2;                   // 0.5/cs2
    float inv_cfl, half_dt, dt;
    float gF;                        // 1/(cfl*cs2)
    float inv_cs2;
    float rho0, c0;
    float mob_p, mob_n;
    float ms, md;                    // moving top wall terms
    float f_chargef, ext_xf, exff;   // force F = f_charge (c+ - c-) (E + ext_x) + exf, FP32
    float cfl_hdt;                   // cfl dt/2: population momentum of the half force
    float srcF;                      // sm cfl dt: population momentum of the Guo source per unit F
    float half_inv_dxf, half_inv_dyf;  // E = (psi[-] - psi[+]) * (1/(2 dx))
    float rhs_qf;                    // -f_charge / eps: right-hand side per unit c+ - c-
    // FP64 set-up constants (initialisation; the zero mode of E_y)
    double f_charge, eps, ext_x, exf, dx, dy;
    double half_inv_dx, half_inv_dy;
    const double *zlo, *zhi, *cplo, *cphi, *cnlo, *cnhi;
    // field planes of the step (PoissonPlan::rhsf, psif, psim)
    float *rhsf;
    const float *psif;
    const double *psim;
    const float *lift;               // wall lifting's x-fluctuation (Chan::lift)
    const float *kref;               // per-row references / 36 (see Chan::kref)
    // Ion frames of the wall nodes (/36), per population buffer b (the
    // frame of the values stored in pops[b]), species s (0 c+, 1 c-), wall w
    // (0 lower, 1 upper): kwall[((b*2 + s)*2 + w)*nx + x]; and half the frame
    // defect (2 c_w - F_0 - F_1)/2 per (s, w, x): wdelta[(s*2 + w)*nx + x].
    const float *kwall;
    const float *wdelta;
    int keep_l2;                     // right-hand side stores ask L2 to keep the plane
};

__device__ __forceinline__ float kwall_at(const ChanF &k, int buf, int s, int w, int x) {
    return __ldg(k.kwall + ((size_t)((buf * 2 + s) * 2 + w)) * k.nx + x);
}
__device__ __forceinline__ float wdelta_at(const ChanF &k, int s, int w, int x) {
    return __ldg(k.wdelta + ((size_t)(s * 2 + w)) * k.nx + x);
}

template <typename S> __device__ __forceinline__ float ld_pop(const S *p);
template <> __device__ __forceinline__ float ld_pop<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_pop<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <typename S> __device__ __forceinline__ void st_pop(S *p, float v);
template <> __device__ __forceinline__ void st_pop<float>(float *p, float v) { *p = v; }
template <> __device__ __forceinline__ void st_pop<__half>(__half *p, float v) { *p = __float2half_rn(v); }

constexpr float W0F = 4.0f / 9.0f, WSF = 1.0f / 9.0f, WDF = 1.0f / 36.0f;

// Index arithmetic of the node update in type I: size_t in general,
// uint32_t where every offset into the 27 population planes and the 9 field
// planes fits 32 bits (27 plane < 2^32), which spares the 64-bit address
// arithmetic of every access.
// Whether the 32-bit index form covers a channel of `plane` elements a plane.
__host__ __device__ constexpr bool index32_fits(size_t plane) { return plane < ((size_t)1 << 32) / 27; }

template <typename S, typename I = size_t>
__device__ __forceinline__ void own9s(const S *__restrict__ b, I pl, I o, float p[9]) {
#pragma unroll
    for (int d = 0; d < 9; ++d) p[d] = ld_pop<S>(b + ((I)d * pl + o));
}

template <typename S, typename I = size_t>
__device__ __forceinline__ void pull9s(const S *__restrict__ b, I pl, int nxp, int x, int y, int xm,
                                       int xp, int ym, int yp, float p[9]) {
    const I r0 = (I)y * (I)nxp, rm = (I)ym * (I)nxp, rp = (I)yp * (I)nxp;
    p[0] = ld_pop<S>(b + (r0 + (I)x));
    p[1] = ld_pop<S>(b + (1 * pl + r0 + (I)xm));
    p[2] = ld_pop<S>(b + (2 * pl + rm + (I)x));
    p[3] = ld_pop<S>(b + (3 * pl + r0 + (I)xp));
    p[4] = ld_pop<S>(b + (4 * pl + rp + (I)x));
    p[5] = ld_pop<S>(b + (5 * pl + rm + (I)xm));
    p[6] = ld_pop<S>(b + (6 * pl + rm + (I)xp));
    p[7] = ld_pop<S>(b + (7 * pl + rp + (I)xp));
    p[8] = ld_pop<S>(b + (8 * pl + rp + (I)xm));
}

// Change of frame of pulled populations to the puller's row reference:
// directions 2, 5, 6 came from row y-1 (dm = kref[y-1] - kref[y]), 4, 7, 8
// from row y+1 (dp = kref[y+1] - kref[y]); 36 w = 4 (straight), 1 (diagonal).
__device__ __forceinline__ void reframe_dn(float p[9], float dm) {
    p[2] += 4.0f * dm;
    p[5] += dm;
    p[6] += dm;
}
__device__ __forceinline__ void reframe_up(float p[9], float dp) {
    p[4] += 4.0f * dp;
    p[7] += dp;
    p[8] += dp;
}
__device__ __forceinline__ void reframe(float p[9], float dm, float dp) {
    reframe_dn(p, dm);
    reframe_up(p, dp);
}
// Pulls from a wall row, whose ion values sit in per-x frames kw(x'):
// lower wall (puller y = 1): 2 from x, 5 from x-1, 6 from x+1;
// upper wall (puller y = ny-2): 4 from x, 7 from x+1, 8 from x-1.
__device__ __forceinline__ void reframe_dn_wall(float p[9], float kx, float kxm, float kxp, float k0) {
    p[2] += 4.0f * (kx - k0);
    p[5] += kxm - k0;
    p[6] += kxp - k0;
}
__device__ __forceinline__ void reframe_up_wall(float p[9], float kx, float kxm, float kxp, float k0) {
    p[4] += 4.0f * (kx - k0);
    p[7] += kxp - k0;
    p[8] += kxm - k0;
}

// Ion anti-bounce-back in deviations: d_ibar = -q_i + 2 w_i (c_wall - R).
__device__ __forceinline__ void ion_wall_dev(const float q[9], float dcw, float p[9]) {
    const float m0 = 2.0f * W0F * dcw, ms = 2.0f * WSF * dcw, md = 2.0f * WDF * dcw;
    p[0] = -q[0] + m0;
    p[3] = -q[1] + ms;
    p[4] = -q[2] + ms;
    p[1] = -q[3] + ms;
    p[2] = -q[4] + ms;
    p[7] = -q[5] + md;
    p[8] = -q[6] + md;
    p[5] = -q[7] + md;
    p[6] = -q[8] + md;
}

// Moments with opposite directions paired first.  In the double layer the
// y-opposite populations carry large, nearly opposite parts (the force-
// balanced y-flux); adding those partners first cancels them exactly
// (Sterbenz), so the small remaining sums round at their own scale.
__device__ __forceinline__ float sum9f(const float t[9]) {
    return (t[0] + (t[1] + t[3])) + ((t[2] + t[4]) + ((t[5] + t[7]) + (t[6] + t[8])));
}
// x-momentum: t5 - t6 and t8 - t7 pair values streamed from one row (same
// y-part), so each difference is exact when the y-part dominates.
__device__ __forceinline__ float momx(const float t[9]) {
    return (t[1] - t[3]) + ((t[5] - t[6]) + (t[8] - t[7]));
}
__device__ __forceinline__ float momy(const float t[9]) {
    return (t[2] - t[4]) + ((t[5] + t[6]) - (t[7] + t[8]));
}

// v/36 by multiplication with the rounded 1/36: the momentum-carrying parts
// of the equilibria and of the force are built from these units times the
// exact integers 36 w = 4 (straight) or 1 (diagonal), so their momentum is
// dens*u (or F) up to the rounding of the unit; with the weights rounded to
// FP32 it would be off by a relative 7.4e-9 that the fluid, whose momentum is
// conserved, would gain step after step.
__device__ __forceinline__ float div36(float v) { return v * (1.0f / 36.0f); }

// TRT of one species in deviations, in place, FP32.  ux, uy: the species'
// advection velocity; usq_rest: u^2 of the rest equilibrium (the c- quirk of
// LBM.cu:493 passes the fluid's); FORCE adds the Guo source of (fx, fy) to the
// post-collision values (add_guo's split, LBM.cu:554-756).
// The diagonal pairs (5,7), (6,8) collide in the moments
//   S = d5 + d6 + d7 + d8  (mass)        Q = d5 - d6 + d7 - d8  (xy)
//   X = d5 - d6 - d7 + d8  (x-momentum)  Y = d5 + d6 - d7 - d8  (y-momentum)
// which the pair form's TRT maps linearly: S, Q relax with w+ to
//   S_eq = (base + dens (cx^2 + cy^2)/2)/9,  Q_eq = dens cx cy/9,
// X, Y with w- to their antisymmetric equilibria.
// Conserved quantities are split exactly rather than rebuilt from rounded
// weights: an equilibrium off by a fixed factor 1 + e (the rounding of 1/36,
// or of rho * (m / rho)) is what the relaxation restores every step, so the
// quantity would grow like (1 + e)^t (3e-5 of u_x after 10,000 steps).
//  * mass: the rest equilibrium is the remainder d_dens - sum of the others
//    (plus, for the c- quirk, its extra term), so the equilibria carry d_dens;
//  * fluid momentum (FLUID, P = the population momentum with the half force,
//    cfl rho u): the straight pair takes round(P/3) and the diagonal moment
//    the exact rest P - 2 round(P/3) (Sterbenz), summing to P exactly; the
//    force source sm cfl dt F is split the same way.
// Ions (not FLUID) relax their flux to 4 dens c/36 per pair unit: the ion
// flux is not conserved, so no factor accumulates.
template <bool FORCE, bool FLUID>
__device__ __forceinline__ void trt_f32(float d[9], float ddens, float dens, float ux, float uy, float usq_rest,
                                        float wp, float wm, const ChanF &k, float fx, float fy, float px, float py) {
    const float vsq = ux * ux + uy * uy;
    const float usq = k.hinvcs2 * vsq;
    const float base = ddens - dens * usq;
    const float cx = ux * k.kcu, cy = uy * k.kcu;
    // symmetric equilibria: straight pairs, diagonal mass and xy moments, rest remainder
    const float seq13 = WSF * (base + dens * (0.5f * cx * cx));
    const float seq24 = WSF * (base + dens * (0.5f * cy * cy));
    const float seq_s = (base + dens * (0.5f * (cx * cx + cy * cy))) * (1.0f / 9.0f);
    const float seq_q = dens * (cx * cy) * (1.0f / 9.0f);
    const float e0 = (ddens - ((2.0f * seq13 + 2.0f * seq24) + seq_s)) + W0F * dens * (k.hinvcs2 * (vsq - usq_rest));
    // antisymmetric equilibria (half-pair units: a13 = (d1 - d3)/2, X = d5 - d6 - d7 + d8)
    float aq13, aqx, aq24, aqy;
    if (FLUID) {
        aq13 = px * (1.0f / 3.0f);
        aqx = px - 2.0f * aq13;
        aq24 = py * (1.0f / 3.0f);
        aqy = py - 2.0f * aq24;
    } else {
        aq13 = aqx = 4.0f * div36(dens * cx);
        aq24 = aqy = 4.0f * div36(dens * cy);
    }
    float d0 = d[0] - wp * (d[0] - e0);
    float s13 = 0.5f * (d[1] + d[3]), a13 = 0.5f * (d[1] - d[3]);
    float s24 = 0.5f * (d[2] + d[4]), a24 = 0.5f * (d[2] - d[4]);
    s13 = s13 - wp * (s13 - seq13);
    a13 = a13 - wm * (a13 - aq13);
    s24 = s24 - wp * (s24 - seq24);
    a24 = a24 - wm * (a24 - aq24);
    const float A = d[5] - d[6], B = d[8] - d[7];  // x-differences of values from one row
    const float C = d[5] + d[6], D = d[7] + d[8];
    float X = A + B, Q = A - B, Y = C - D, S = C + D;
    S = S - wp * (S - seq_s);
    Q = Q - wp * (Q - seq_q);
    X = X - wm * (X - aqx);
    Y = Y - wm * (Y - aqy);
    if (FORCE) {
        const float uF = k.inv_cs2 * (ux * fx + uy * fy);
        const float cfx = fx * k.gF, cfy = fy * k.gF;
        const float sp = k.sp * k.dt;
        // symmetric (mass-free) part: the rest takes the remainder
        const float g13 = sp * (WSF * (cx * cfx - uF)), g24 = sp * (WSF * (cy * cfy - uF));
        const float gs = sp * ((cx * cfx + cy * cfy - uF) * (1.0f / 9.0f));
        const float gq = sp * ((cx * cfy + cy * cfx) * (1.0f / 9.0f));
        d0 -= (2.0f * g13 + 2.0f * g24) + gs;
        s13 += g13;
        s24 += g24;
        S += gs;
        Q += gq;
        // momentum: sm cfl dt F, a third to each straight half-pair unit
        const float fsx = k.srcF * fx, fsy = k.srcF * fy;
        const float q13 = fsx * (1.0f / 3.0f), q24 = fsy * (1.0f / 3.0f);
        a13 += q13;
        a24 += q24;
        X += fsx - 2.0f * q13;
        Y += fsy - 2.0f * q24;
    }
    const float P = S + Y, M = S - Y, U = Q + X, V = Q - X;
    d[0] = d0;
    d[1] = s13 + a13;
    d[3] = s13 - a13;
    d[2] = s24 + a24;
    d[4] = s24 - a24;
    d[5] = 0.25f * (P + U);
    d[6] = 0.25f * (P - U);
    d[7] = 0.25f * (M + V);
    d[8] = 0.25f * (M - V);
}

// Central-difference E of the shifted forms (the stencil of gpu_efield and
// gpu_bc, poisson.cu:145-174: wall rows take the adjacent row's Ey), with
// the 1/(2 dx), 1/(2 dy) factors precomputed: a multiply in place of an
// FP64 division per component.
__device__ __forceinline__ void efield_shifted(const ChanF &k, const double *__restrict__ psi, int x, int y, int xm,
                                               int xp, double *ex, double *ey) {
    const size_t r = (size_t)y * k.nxp;
    *ex = (__ldg(psi + r + xm) - __ldg(psi + r + xp)) * k.half_inv_dx;
    const int yc = y == 0 ? 1 : (y == k.ny - 1 ? k.ny - 2 : y);
    *ey = (__ldg(psi + (size_t)(yc - 1) * k.nxp + x) - __ldg(psi + (size_t)(yc + 1) * k.nxp + x)) * k.half_inv_dy;
}

// E of the step from psi = psim (row means, FP64) + psif (FP32): Ex from the
// FP32 fluctuations alone, Ey from the FP64 difference of the two row means
// (the zero mode, rounded once) plus that of the fluctuations.  Stencil of
// gpu_efield / gpu_bc (poisson.cu:145-174).
template <typename I = size_t>
__device__ __forceinline__ void efield_f32(const ChanF &k, int x, int y, int xm, int xp, float *ex, float *ey) {
    const I r = (I)y * (I)k.nxp;
    *ex = (__ldg(k.psif + (r + (I)xm)) - __ldg(k.psif + (r + (I)xp))) * k.half_inv_dxf;
    const int yc = y == 0 ? 1 : (y == k.ny - 1 ? k.ny - 2 : y);
    const float eym = (float)((__ldg(k.psim + yc - 1) - __ldg(k.psim + yc + 1)) * k.half_inv_dy);
    *ey = eym + (__ldg(k.psif + ((I)(yc - 1) * (I)k.nxp + (I)x)) - __ldg(k.psif + ((I)(yc + 1) * (I)k.nxp + (I)x))) *
                    k.half_inv_dyf;
}

// One node of one step.  src/dst: 27 population planes (species-major);
// fields: the channel's 9 FP64 field planes.
// Raw populations of one node, as stored: FIRST -> the node's own
// (pre-collision) values; otherwise the fluid pulled from the neighbours and
// the ions pulled (interior rows) or the node's own values (wall rows).
template <typename S, bool FIRST, typename I = size_t>
__device__ __forceinline__ void gather_global(const ChanF &k, const S *__restrict__ src, int x, int y, float f[9],
                                              float h[9], float t[9]) {
    const I pl = (I)k.plane;
    const int nxp = k.nxp;
    const I o = (I)y * (I)nxp + (I)x;
    const bool wall = y == 0 || y == k.ny - 1;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
    const S *sf = src, *sh = src + 9 * pl, *st = src + 18 * pl;
    if (FIRST) {
        own9s<S, I>(sf, pl, o, f);
        own9s<S, I>(sh, pl, o, h);
        own9s<S, I>(st, pl, o, t);
    } else {
        pull9s<S, I>(sf, pl, nxp, x, y, xm, xp, ym, yp, f);
        if (wall) {
            own9s<S, I>(sh, pl, o, h);
            own9s<S, I>(st, pl, o, t);
        } else {
            pull9s<S, I>(sh, pl, nxp, x, y, xm, xp, ym, yp, h);
            pull9s<S, I>(st, pl, nxp, x, y, xm, xp, ym, yp, t);
        }
    }
}

// Collision, walls and stores of one node from its raw populations (see
// gather_global); src is read only for the lower wall's row-1 pull.  sbuf:
// index (0/1) of the population buffer that src is, which names the wall
// nodes' ion frames of the values read (sbuf) and written (sbuf ^ 1).
// `moments` is a run-time flag on purpose: as a template parameter it gave
// two instantiations that the compiler fused into multiply-adds differently,
// so a step that wrote the moments could round differently from one that
// did not.  One body with predicated stores keeps every step's arithmetic
// independent of how the steps are split into calls.
template <typename S, bool FIRST, bool EXPLICIT_E, typename I = size_t>
__device__ __forceinline__ void collide_shifted(const ChanF &k, float f[9], float h[9], float t[9],
                                                const S *__restrict__ src, S *__restrict__ dst,
                                                double *__restrict__ fields, int x, int y, bool moments, int sbuf) {
    const I pl = (I)k.plane;
    const int nxp = k.nxp;
    const I o = (I)y * (I)nxp + (I)x;
    const bool lo = y == 0, hi = y == k.ny - 1, wall = lo || hi;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
    const S *sf = src;
    const int ny = k.ny;
    // frames (/36) of this node's values: the fluid and interior ions use the
    // row references, the wall nodes' ions the per-x frame of the output buffer
    const float kf0 = __ldg(k.kref + y);
    float kh0, kt0;
    if (wall) {
        const int w = lo ? 0 : 1;
        kh0 = kwall_at(k, sbuf ^ 1, 0, w, x);
        kt0 = kwall_at(k, sbuf ^ 1, 1, w, x);
    } else {
        kh0 = __ldg(k.kref + ny + y);
        kt0 = __ldg(k.kref + 2 * ny + y);
    }
    const float Rf = 36.0f * kf0, Rh = 36.0f * kh0, Rt = 36.0f * kt0;  // exact: 36 K 2^-q < 2^22 2^-q
    if (!FIRST) reframe(f, __ldg(k.kref + ym) - kf0, __ldg(k.kref + yp) - kf0);
    if (wall) {
        // anti-bounce-back (gpu_bc_charge) from the stored frame into the
        // other: an exact reflection plus w_i times the frame defect; the
        // first step too, whose stored values init_node_shifted reflected
        const int w = lo ? 0 : 1;
        float q[9];
#pragma unroll
        for (int d = 0; d < 9; ++d) q[d] = h[d];
        ion_wall_dev(q, wdelta_at(k, 0, w, x), h);
#pragma unroll
        for (int d = 0; d < 9; ++d) q[d] = t[d];
        ion_wall_dev(q, wdelta_at(k, 1, w, x), t);
    } else if (!FIRST) {
        if (y == 1) {
            reframe_dn_wall(h, kwall_at(k, sbuf, 0, 0, x), kwall_at(k, sbuf, 0, 0, xm), kwall_at(k, sbuf, 0, 0, xp), kh0);
            reframe_dn_wall(t, kwall_at(k, sbuf, 1, 0, x), kwall_at(k, sbuf, 1, 0, xm), kwall_at(k, sbuf, 1, 0, xp), kt0);
        } else {
            reframe_dn(h, __ldg(k.kref + ny + ym) - kh0);
            reframe_dn(t, __ldg(k.kref + 2 * ny + ym) - kt0);
        }
        if (y == ny - 2) {
            reframe_up_wall(h, kwall_at(k, sbuf, 0, 1, x), kwall_at(k, sbuf, 0, 1, xm), kwall_at(k, sbuf, 0, 1, xp), kh0);
            reframe_up_wall(t, kwall_at(k, sbuf, 1, 1, x), kwall_at(k, sbuf, 1, 1, xm), kwall_at(k, sbuf, 1, 1, xp), kt0);
        } else {
            reframe_up(h, __ldg(k.kref + ny + yp) - kh0);
            reframe_up(t, __ldg(k.kref + 2 * ny + yp) - kt0);
        }
    }
    const float drho = sum9f(f), dcp = sum9f(h), dcn = sum9f(t);
    const float rho = Rf + drho;
    float ex, ey;
    if (EXPLICIT_E) {
        ex = (float)fields[F_EX * pl + o];
        ey = (float)fields[F_EY * pl + o];
    } else {
        efield_f32<I>(k, x, y, xm, xp, &ex, &ey);
    }
    float fx = 0.0f, fy = 0.0f;
    const float dq = dcp - dcn;
    const float qnet = (Rh - Rt) + dq;  // c+ - c-
    if (k.flags & EK_FLAG_FORCE) {
        const float q = k.f_chargef * qnet;
        fx = q * (ex + k.ext_xf) + k.exff;
        fy = q * ey;
    }
    const float rrho = 1.0f / rho;
    float ux = (momx(f) * k.inv_cfl + fx * k.half_dt) * rrho;
    float uy = (momy(f) * k.inv_cfl + fy * k.half_dt) * rrho;
    if (lo) {
        float m[9];
        const I o1 = (I)nxp + (I)x;
        const float kf1 = __ldg(k.kref + 1);
        if (FIRST) {
            own9s<S, I>(sf, pl, o1, m);
        } else {
            pull9s<S, I>(sf, pl, nxp, x, 1, xm, xp, 0, 2, m);
            reframe(m, __ldg(k.kref + 0) - kf1, __ldg(k.kref + 2) - kf1);
        }
        const float rrho1 = 1.0f / (36.0f * kf1 + sum9f(m));
        ux = -(momx(m) * k.inv_cfl + fx * k.half_dt) * rrho1;
        uy = -(momy(m) * k.inv_cfl + fy * k.half_dt) * rrho1;
    }
    if (moments) {
        fields[(I)F_RHO * pl + o] = (double)Rf + (double)drho;
        fields[(I)F_UX * pl + o] = ux;
        fields[(I)F_UY * pl + o] = uy;
        fields[(I)F_CP * pl + o] = (double)Rh + (double)dcp;
        fields[(I)F_CN * pl + o] = (double)Rt + (double)dcn;
    }
    // right-hand side without its FP64 row constant (rhs_q (R+ - R-) and the
    // lifting's x-mean, added by the row pass), with the lifting's x-fluctuation
    if (!wall) {
        float v = k.rhs_qf * dq;
        if (y == 1) v -= __ldg(k.lift + x);
        if (y == ny - 2) v -= __ldg(k.lift + k.nx + x);
        st_field_f(k.rhsf + o, v, k.keep_l2);
    }
    // ions: FP32 TRT, moment form (trt_f32)
    {
        {
            const float vx = ux + k.mob_p * ex, vy = uy + k.mob_p * ey;
            trt_f32<false, false>(h, dcp, Rh + dcp, vx, vy, vx * vx + vy * vy, k.wcp, k.wcm, k, 0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int d = 0; d < 9; ++d) st_pop<S>(dst + ((I)(9 + d) * pl + o), h[d]);
        }
        {
            const float vx = ux + k.mob_n * ex, vy = uy + k.mob_n * ey;
            trt_f32<false, false>(t, dcn, Rt + dcn, vx, vy,
                                  (k.flags & EK_FLAG_REST_QUIRK) ? ux * ux + uy * uy : vx * vx + vy * vy, k.wtp, k.wtm,
                                  k, 0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int d = 0; d < 9; ++d) st_pop<S>(dst + ((I)(18 + d) * pl + o), t[d]);
        }
    }
    S *df = dst;
    if (lo) {
        st_pop<S>(df + o, f[0]);
#pragma unroll
        for (int d = 1; d < 9; ++d) st_pop<S>(df + ((I)oppd(d) * pl + o), f[d]);
        return;
    }
    if (hi) {
        st_pop<S>(df + o, f[0]);
        st_pop<S>(df + (3 * pl + o), f[1] - k.ms);
        st_pop<S>(df + (4 * pl + o), f[2]);
        st_pop<S>(df + (1 * pl + o), f[3] + k.ms);
        st_pop<S>(df + (2 * pl + o), f[4]);
        st_pop<S>(df + (7 * pl + o), f[5] - k.md);
        st_pop<S>(df + (8 * pl + o), f[6] + k.md);
        st_pop<S>(df + (5 * pl + o), f[7] + k.md);
        st_pop<S>(df + (6 * pl + o), f[8] - k.md);
        return;
    }
    // fluid: FP32 TRT with the Guo source, moment form (trt_f32); the
    // population momentum with the half force, cfl rho u
    const float px = momx(f) + k.cfl_hdt * fx, py = momy(f) + k.cfl_hdt * fy;
    if (k.flags & EK_FLAG_FORCE)
        trt_f32<true, true>(f, drho, rho, ux, uy, ux * ux + uy * uy, k.wp, k.wm, k, fx, fy, px, py);
    else
        trt_f32<false, true>(f, drho, rho, ux, uy, ux * ux + uy * uy, k.wp, k.wm, k, 0.0f, 0.0f, px, py);
#pragma unroll
    for (int d = 0; d < 9; ++d) st_pop<S>(df + ((I)d * pl + o), f[d]);
}

template <typename S, bool FIRST, bool EXPLICIT_E, typename I = size_t>
__device__ __forceinline__ void node_shifted(const ChanF &k, const S *__restrict__ src, S *__restrict__ dst,
                                             double *__restrict__ fields, int x, int y, bool moments, int sbuf) {
    float f[9], h[9], t[9];
    gather_global<S, FIRST, I>(k, src, x, y, f, h, t);
    collide_shifted<S, FIRST, EXPLICIT_E, I>(k, f, h, t, src, dst, fields, x, y, moments, sbuf);
}

// Equilibrium deviations from the fields (pre-collision layout), written to
// population buffer `buf`.  The wall nodes' ions are stored reflected
// (anti-bounce-back from their frame in buf ^ 1 into the one of buf), since
// every step, the first included, reflects them on load.
template <typename S>
__device__ __forceinline__ void init_node_shifted(const ChanF &k, S *__restrict__ pops, const double *__restrict__ fields,
                                                  bool explicit_e, int x, int y, int buf) {
    const size_t pl = k.plane, o = (size_t)y * k.nxp + x;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    double exd, eyd;
    if (explicit_e) {
        exd = fields[F_EX * pl + o];
        eyd = fields[F_EY * pl + o];
    } else {
        efield_shifted(k, fields + F_PSI * pl, x, y, xm, xp, &exd, &eyd);
    }
    const float Ex = (float)exd, Ey = (float)eyd;
    const float ux = (float)fields[F_UX * pl + o], uy = (float)fields[F_UY * pl + o];
    const double densd[3] = {fields[F_RHO * pl + o], fields[F_CP * pl + o], fields[F_CN * pl + o]};
    const float dens[3] = {(float)densd[0], (float)densd[1], (float)densd[2]};
    const float mob[3] = {0.0f, k.mob_p, k.mob_n};
    const bool wall = y == 0 || y == k.ny - 1;
    const int w = y == 0 ? 0 : 1;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const float vx = ux + mob[s] * Ex, vy = uy + mob[s] * Ey;
        const float usq = k.hinvcs2 * (vx * vx + vy * vy);
        const bool wion = wall && s > 0;
        const float kframe = wion ? kwall_at(k, buf ^ 1, s - 1, w, x) : __ldg(k.kref + s * k.ny + y);
        const float dd = (float)(densd[s] - 36.0 * (double)kframe);
        const float base = dd - dens[s] * usq;
        const float cx = vx * k.kcu, cy = vy * k.kcu;
        const float ax = div36(dens[s] * cx), ay = div36(dens[s] * cy);
        float e[9];
        e[0] = W0F * base;
        const float cu[4] = {cx, cy, cx + cy, cy - cx};
        const float an[4] = {4.0f * ax, 4.0f * ay, ax + ay, ay - ax};
        const int ia[4] = {1, 2, 5, 6};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float w = q < 2 ? WSF : WDF;
            const float sym = w * (base + dens[s] * 0.5f * cu[q] * cu[q]);
            const float anti = an[q];
            e[ia[q]] = sym + anti;
            e[oppd(ia[q])] = sym - anti;
        }
        if (wion) {
            float r[9];
            ion_wall_dev(e, wdelta_at(k, s - 1, w, x), r);
#pragma unroll
            for (int d = 0; d < 9; ++d) e[d] = r[d];
        }
#pragma unroll
        for (int d = 0; d < 9; ++d) st_pop<S>(pops + (s * 9 + d) * pl + o, e[d]);
    }
}

// Wall frames of the ions at initialisation, one thread per (species s, wall
// w, x): F_a = the wall node's density on the species' grid (the frame of the
// state after the first step, buffer buf ^ 1), F_b = 2 c_w - F_a on the same
// grid (buffer buf, where the reflected initial values go), and half the
// defect (2 c_w - F_a - F_b)/2.  FP64 here: set-up, not the step.
__device__ __forceinline__ void wall_frames_dev(const ChanF &k, const double *__restrict__ fields, int qp, int qn, int buf,
                                                float *__restrict__ kwall, float *__restrict__ wdelta, int i) {
    const int x = i % k.nx, sw = i / k.nx, s = sw >> 1, w = sw & 1;
    const int y = w ? k.ny - 1 : 0;
    const double dens = fields[(s ? F_CN : F_CP) * k.plane + (size_t)y * k.nxp + x];
    const double cw = s ? (w ? k.cnhi[x] : k.cnlo[x]) : (w ? k.cphi[x] : k.cplo[x]);
    const double g = ldexp(1.0, s ? qn : qp);
    const double fa = ldexp(rint(dens / 36.0 * g), -(s ? qn : qp));      // /36
    const double fb = ldexp(rint((2.0 * cw / 36.0 - fa) * g), -(s ? qn : qp));
    kwall[((size_t)(((buf ^ 1) * 2 + s) * 2 + w)) * k.nx + x] = (float)fa;
    kwall[((size_t)((buf * 2 + s) * 2 + w)) * k.nx + x] = (float)fb;
    wdelta[(size_t)(s * 2 + w) * k.nx + x] = (float)(cw - 18.0 * (fa + fb));
}

// Half the frame defect after the wall concentrations change (per-x walls set
// after initialisation): the frames stay, the defect follows c_w.
__device__ __forceinline__ void wall_delta_dev(const ChanF &k, const float *__restrict__ kwall, float *__restrict__ wdelta,
                                               int i) {
    const int x = i % k.nx, sw = i / k.nx, s = sw >> 1, w = sw & 1;
    const double cw = s ? (w ? k.cnhi[x] : k.cnlo[x]) : (w ? k.cphi[x] : k.cplo[x]);
    const double f0 = kwall[((size_t)((0 * 2 + s) * 2 + w)) * k.nx + x];
    const double f1 = kwall[((size_t)((1 * 2 + s) * 2 + w)) * k.nx + x];
    wdelta[(size_t)(s * 2 + w) * k.nx + x] = (float)(cw - 18.0 * (f0 + f1));
}

// Row y's means of rho, c+, c- rounded to the reference grids K 2^-q (stored
// /36), FP64 sums; a block of 256 threads per row, kout[s*ny + y].
__device__ __forceinline__ void row_refs_dev(int nx, int nxp, int ny, size_t plane, const double *__restrict__ fields,
                                             int qf, int qp, int qn, float *__restrict__ kout, int y) {
    double acc[3] = {0.0, 0.0, 0.0};
    const size_t r = (size_t)y * nxp;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        acc[0] += fields[F_RHO * plane + r + x];
        acc[1] += fields[F_CP * plane + r + x];
        acc[2] += fields[F_CN * plane + r + x];
    }
    __shared__ double red[8][3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        double v = acc[s];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][s] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
        const int q = threadIdx.x == 0 ? qf : (threadIdx.x == 1 ? qp : qn);
        const double mean = v / (double)nx;
        const double K = rint(mean / 36.0 * ldexp(1.0, q));
        kout[threadIdx.x * ny + y] = (float)ldexp(K, -q);
    }
}

// Re-basing of one stored value of plane (species s, direction d) at row y:
// d += 36 w_d (kold - knew), exact in FP32.
template <typename S>
__device__ __forceinline__ void rebase_dev(S *p, int plane_idx, int ny, int y, const float *__restrict__ kold,
                                           const float *__restrict__ knew) {
    const int s = plane_idx / 9, d = plane_idx - 9 * s;
    if (s > 0 && (y == 0 || y == ny - 1)) return;  // wall ions keep their per-x frames
    const float wint = d == 0 ? 16.0f : (d < 5 ? 4.0f : 1.0f);
    const float corr = wint * (kold[s * ny + y] - knew[s * ny + y]);
    st_pop<S>(p, ld_pop<S>(p) + corr);
}

ChanF make_chanf(const Chan &c);

}  // namespace ek
