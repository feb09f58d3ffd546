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
    // FP64 constants of the fluid relaxation + Guo source (see node_shifted)
    double wpd, wmd, spd, smd, kcud, hinvcs2d, gFd, inv_cs2d, dtd;
    double f_charge, eps, ext_x, exf, dx, dy;
    double wcpd, wcmd, wtpd, wtmd, mob_pd, mob_nd;  // FP64 ion relaxation constants
    double half_inv_dx, half_inv_dy;   // E = (psi[-] - psi[+]) * (1/(2 dx)), one multiply each
    double rhs_q;                      // -f_charge / eps: Poisson right-hand side per unit c+ - c-
    double inv_dy2;                    // 1/dy^2 of the wall lifting term
    const double *zlo, *zhi, *cplo, *cphi, *cnlo, *cnhi;
    const float *kref;               // per-row references / 36 (see Chan::kref)
    int keep_l2;                     // right-hand side stores ask L2 to keep the plane
};

template <typename S> __device__ __forceinline__ float ld_pop(const S *p);
template <> __device__ __forceinline__ float ld_pop<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_pop<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <typename S> __device__ __forceinline__ void st_pop(S *p, float v);
template <> __device__ __forceinline__ void st_pop<float>(float *p, float v) { *p = v; }
template <> __device__ __forceinline__ void st_pop<__half>(__half *p, float v) { *p = __float2half_rn(v); }

constexpr float W0F = 4.0f / 9.0f, WSF = 1.0f / 9.0f, WDF = 1.0f / 36.0f;

template <typename S>
__device__ __forceinline__ void own9s(const S *__restrict__ b, size_t pl, size_t o, float p[9]) {
#pragma unroll
    for (int d = 0; d < 9; ++d) p[d] = ld_pop<S>(b + d * pl + o);
}

template <typename S>
__device__ __forceinline__ void pull9s(const S *__restrict__ b, size_t pl, int nxp, int x, int y, int xm,
                                       int xp, int ym, int yp, float p[9]) {
    const size_t r0 = (size_t)y * nxp, rm = (size_t)ym * nxp, rp = (size_t)yp * nxp;
    p[0] = ld_pop<S>(b + r0 + x);
    p[1] = ld_pop<S>(b + 1 * pl + r0 + xm);
    p[2] = ld_pop<S>(b + 2 * pl + rm + x);
    p[3] = ld_pop<S>(b + 3 * pl + r0 + xp);
    p[4] = ld_pop<S>(b + 4 * pl + rp + x);
    p[5] = ld_pop<S>(b + 5 * pl + rm + xm);
    p[6] = ld_pop<S>(b + 6 * pl + rm + xp);
    p[7] = ld_pop<S>(b + 7 * pl + rp + xp);
    p[8] = ld_pop<S>(b + 8 * pl + rp + xm);
}

// Change of frame of pulled populations to the puller's row reference:
// directions 2, 5, 6 came from row y-1 (dm = kref[y-1] - kref[y]), 4, 7, 8
// from row y+1 (dp = kref[y+1] - kref[y]); 36 w = 4 (straight), 1 (diagonal).
__device__ __forceinline__ void reframe(float p[9], float dm, float dp) {
    p[2] += 4.0f * dm;
    p[5] += dm;
    p[6] += dm;
    p[4] += 4.0f * dp;
    p[7] += dp;
    p[8] += dp;
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
__device__ __forceinline__ float momx(const float t[9]) {
    return (t[1] - t[3]) + ((t[5] + t[8]) - (t[6] + t[7]));
}
__device__ __forceinline__ float momy(const float t[9]) {
    return (t[2] - t[4]) + ((t[5] + t[6]) - (t[7] + t[8]));
}

// Constants of the collision in compute type T.
template <typename T> struct CollK {
    T wp, wm, sp, sm, kcu, hinvcs2, gF, inv_cs2, dt;
};
// v/36.  FP64: multiplication by the rounded 1/36 (relative bias 1e-17).
// FP32 (ion species only): likewise; the resulting 7e-9 bias of the ion
// equilibrium flux does not accumulate, because the ion flux is not a
// conserved quantity (the fluid momentum, which is, runs in FP64).
__device__ __forceinline__ float div36(float v) { return v * (1.0f / 36.0f); }
__device__ __forceinline__ double div36(double v) { return v * (1.0 / 36.0); }

// TRT of one pair in deviations.  w: lattice weight, cu: (c_i.u)*kcu,
// base: d_dens - dens*usq (symmetric equilibrium without the cu^2 term),
// aeq: antisymmetric equilibrium w*dens*cu (built by the caller, see trt_dev).
template <typename T>
__device__ __forceinline__ void trt_pair_dev(T &da, T &db, T w, T dens, T cu, T base, T aeq, T wp, T wm) {
    const T seq = w * (base + dens * (T(0.5) * cu * cu));
    const T s = T(0.5) * (da + db), a = T(0.5) * (da - db);
    const T ps = wp * (s - seq), pa = wm * (a - aeq);
    da = da - ps - pa;
    db = db - ps + pa;
}

// Full TRT of one species in deviations, in place.  ux, uy: the species'
// advection velocity; usq_rest: u^2 used by the rest equilibrium.
// The antisymmetric equilibria carry the momentum (w- relaxes it to them
// every step): they are built from the units dens*cu/36 times the exact
// integers 36 w = 4 or 1, so that their momentum is dens*u up to the rounding
// of the unit; with weights w rounded to FP32 it would be dens*u*(1+7.4e-9),
// which the fluid, whose momentum is conserved, would gain step after step.
template <typename T>
__device__ __forceinline__ void trt_dev(T d[9], T ddens, T dens, T ux, T uy, T usq_rest, T wp, T wm,
                                        const CollK<T> &k) {
    const T w0 = T(4.0 / 9.0), ws = T(1.0 / 9.0), wd = T(1.0 / 36.0);
    const T usq = k.hinvcs2 * (ux * ux + uy * uy);
    const T base = ddens - dens * usq;
    const T e0 = w0 * (ddens - dens * (k.hinvcs2 * usq_rest));
    d[0] = d[0] - wp * (d[0] - e0);
    const T cx = ux * k.kcu, cy = uy * k.kcu;
    const T ax = div36(dens * cx), ay = div36(dens * cy);
    trt_pair_dev<T>(d[1], d[3], ws, dens, cx, base, T(4) * ax, wp, wm);
    trt_pair_dev<T>(d[2], d[4], ws, dens, cy, base, T(4) * ay, wp, wm);
    trt_pair_dev<T>(d[5], d[7], wd, dens, cx + cy, base, ax + ay, wp, wm);
    trt_pair_dev<T>(d[6], d[8], wd, dens, cy - cx, base, ay - ax, wp, wm);
}

// Guo source added to post-collision fluid deviations.
template <typename T>
__device__ __forceinline__ void add_guo(T d[9], T ux, T uy, T fx, T fy, const CollK<T> &k) {
    const T w0 = T(4.0 / 9.0), ws = T(1.0 / 9.0), wd = T(1.0 / 36.0);
    const T uF = k.inv_cs2 * (ux * fx + uy * fy);
    const T cux = ux * k.kcu, cuy = uy * k.kcu;
    const T cfx = fx * k.gF, cfy = fy * k.gF;
    const T sp = k.sp * k.dt, sm = k.sm * k.dt;
    d[0] += sp * (w0 * -uF);
    // pair (a, abar) with c_a.u -> cu, c_a.F -> cf; the momentum-carrying
    // part w*cf is built from cf/36 times 36 w = 4 or 1 (see trt_dev)
    const T gx = div36(cfx), gy = div36(cfy);
    auto pair = [&](T &da, T &db, T w, T cu, T cf, T fm) {
        const T fp = w * (cu * cf - uF);
        da += sp * fp + sm * fm;
        db += sp * fp - sm * fm;
    };
    pair(d[1], d[3], ws, cux, cfx, T(4) * gx);
    pair(d[2], d[4], ws, cuy, cfy, T(4) * gy);
    pair(d[5], d[7], wd, cux + cuy, cfx + cfy, gx + gy);
    pair(d[6], d[8], wd, cuy - cux, cfy - cfx, gy - gx);
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

// One node of one step.  src/dst: 27 population planes (species-major);
// fields: the channel's 9 FP64 field planes.
// Raw populations of one node, as stored: FIRST -> the node's own
// (pre-collision) values; otherwise the fluid pulled from the neighbours and
// the ions pulled (interior rows) or the node's own values (wall rows).
template <typename S, bool FIRST>
__device__ __forceinline__ void gather_global(const ChanF &k, const S *__restrict__ src, int x, int y, float f[9],
                                              float h[9], float t[9]) {
    const size_t pl = k.plane;
    const int nxp = k.nxp;
    const size_t o = (size_t)y * nxp + x;
    const bool wall = y == 0 || y == k.ny - 1;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
    const S *sf = src, *sh = src + 9 * pl, *st = src + 18 * pl;
    if (FIRST) {
        own9s<S>(sf, pl, o, f);
        own9s<S>(sh, pl, o, h);
        own9s<S>(st, pl, o, t);
    } else {
        pull9s<S>(sf, pl, nxp, x, y, xm, xp, ym, yp, f);
        if (wall) {
            own9s<S>(sh, pl, o, h);
            own9s<S>(st, pl, o, t);
        } else {
            pull9s<S>(sh, pl, nxp, x, y, xm, xp, ym, yp, h);
            pull9s<S>(st, pl, nxp, x, y, xm, xp, ym, yp, t);
        }
    }
}

// Collision, walls and stores of one node from its raw populations (see
// gather_global); src is read only for the lower wall's row-1 pull.
// `moments` is a run-time flag on purpose: as a template parameter it gave
// two instantiations that the compiler fused into multiply-adds differently,
// so a step that wrote the moments could round differently from one that
// did not.  One body with predicated stores keeps every step's arithmetic
// independent of how the steps are split into calls.
template <typename S, bool FIRST, bool EXPLICIT_E>
__device__ __forceinline__ void collide_shifted(const ChanF &k, float f[9], float h[9], float t[9],
                                                const S *__restrict__ src, S *__restrict__ dst,
                                                double *__restrict__ fields, int x, int y, bool moments) {
    const size_t pl = k.plane;
    const int nxp = k.nxp;
    const size_t o = (size_t)y * nxp + x;
    const bool lo = y == 0, hi = y == k.ny - 1;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
    const S *sf = src;
    const int ny = k.ny;
    // row references (/36) of the three species at rows y, y-1, y+1
    const float kf0 = __ldg(k.kref + y), kh0 = __ldg(k.kref + ny + y), kt0 = __ldg(k.kref + 2 * ny + y);
    const double Rf = 36.0 * kf0, Rh = 36.0 * kh0, Rt = 36.0 * kt0;
    if (!FIRST) {
        reframe(f, __ldg(k.kref + ym) - kf0, __ldg(k.kref + yp) - kf0);
        if (lo || hi) {
            float q[9];
#pragma unroll
            for (int d = 0; d < 9; ++d) q[d] = h[d];
            ion_wall_dev(q, (float)((lo ? k.cplo[x] : k.cphi[x]) - Rh), h);
#pragma unroll
            for (int d = 0; d < 9; ++d) q[d] = t[d];
            ion_wall_dev(q, (float)((lo ? k.cnlo[x] : k.cnhi[x]) - Rt), t);
        } else {
            reframe(h, __ldg(k.kref + ny + ym) - kh0, __ldg(k.kref + ny + yp) - kh0);
            reframe(t, __ldg(k.kref + 2 * ny + ym) - kt0, __ldg(k.kref + 2 * ny + yp) - kt0);
        }
    }
    const float drho = sum9f(f), dcp = sum9f(h), dcn = sum9f(t);
    const float rho = (float)(Rf + (double)drho);
    double exd, eyd;
    if (EXPLICIT_E) {
        exd = fields[F_EX * pl + o];
        eyd = fields[F_EY * pl + o];
    } else {
        efield_shifted(k, fields + F_PSI * pl, x, y, xm, xp, &exd, &eyd);
    }
    float fx = 0.0f, fy = 0.0f;
    const double qnet = (Rh - Rt) + ((double)dcp - (double)dcn);  // c+ - c-
    if (k.flags & EK_FLAG_FORCE) {
        const double q = k.f_charge * qnet;
        fx = (float)(q * (exd + k.ext_x) + k.exf);
        fy = (float)(q * eyd);
    }
    const float rrho = 1.0f / rho;
    float ux = (momx(f) * k.inv_cfl + fx * k.half_dt) * rrho;
    float uy = (momy(f) * k.inv_cfl + fy * k.half_dt) * rrho;
    if (lo) {
        float m[9];
        const size_t o1 = (size_t)nxp + x;
        const float kf1 = __ldg(k.kref + 1);
        if (FIRST) {
            own9s<S>(sf, pl, o1, m);
        } else {
            pull9s<S>(sf, pl, nxp, x, 1, xm, xp, 0, 2, m);
            reframe(m, __ldg(k.kref + 0) - kf1, __ldg(k.kref + 2) - kf1);
        }
        const float rrho1 = 1.0f / (float)(36.0 * kf1 + (double)sum9f(m));
        ux = -(momx(m) * k.inv_cfl + fx * k.half_dt) * rrho1;
        uy = -(momy(m) * k.inv_cfl + fy * k.half_dt) * rrho1;
    }
    if (moments) {
        fields[F_RHO * pl + o] = Rf + (double)drho;
        fields[F_UX * pl + o] = ux;
        fields[F_UY * pl + o] = uy;
        fields[F_CP * pl + o] = Rh + (double)dcp;
        fields[F_CN * pl + o] = Rt + (double)dcn;
    }
    if (!lo && !hi) {
        double v = k.rhs_q * qnet;
        if (y == 1) v = v - k.zlo[x] * k.inv_dy2;
        if (y == k.ny - 2) v = v - k.zhi[x] * k.inv_dy2;
        st_field(fields + F_RHS * pl + o, v, k.keep_l2);
    }
    const float uxf = ux, uyf = uy;
    // Ion relaxation in FP64 on the FP32 deviations, rounded once on the
    // store: in FP32 the ions' c+ / c- error against the FP64 path after
    // 10,000 steps of the 4096x1024 channel from its noisy start was 3.4e-5
    // / 5.3e-5 of max-abs (plug velocity 1.5e-3 of itself); in FP64 1.9e-5 /
    // 1.3e-5 (plug 1.4e-5), for 4 % more kernel time.
    {
        const CollK<double> kd{k.wpd, k.wmd, k.spd, k.smd, k.kcud, k.hinvcs2d, k.gFd, k.inv_cs2d, k.dtd};
        const double uxd = uxf, uyd = uyf;
        double q[9];
        {
            const double vx = uxd + k.mob_pd * exd, vy = uyd + k.mob_pd * eyd;
#pragma unroll
            for (int d = 0; d < 9; ++d) q[d] = (double)h[d];
            trt_dev<double>(q, (double)dcp, Rh + (double)dcp, vx, vy, vx * vx + vy * vy, k.wcpd, k.wcmd, kd);
            S *dh = dst + 9 * pl;
#pragma unroll
            for (int d = 0; d < 9; ++d) st_pop<S>(dh + d * pl + o, (float)q[d]);
        }
        {
            const double vx = uxd + k.mob_nd * exd, vy = uyd + k.mob_nd * eyd;
#pragma unroll
            for (int d = 0; d < 9; ++d) q[d] = (double)t[d];
            trt_dev<double>(q, (double)dcn, Rt + (double)dcn, vx, vy,
                            (k.flags & EK_FLAG_REST_QUIRK) ? uxd * uxd + uyd * uyd : vx * vx + vy * vy, k.wtpd, k.wtmd,
                            kd);
            S *dt_ = dst + 18 * pl;
#pragma unroll
            for (int d = 0; d < 9; ++d) st_pop<S>(dt_ + d * pl + o, (float)q[d]);
        }
    }
    S *df = dst;
    if (lo) {
        st_pop<S>(df + o, f[0]);
#pragma unroll
        for (int d = 1; d < 9; ++d) st_pop<S>(df + oppd(d) * pl + o, f[d]);
        return;
    }
    if (hi) {
        st_pop<S>(df + o, f[0]);
        st_pop<S>(df + 3 * pl + o, f[1] - k.ms);
        st_pop<S>(df + 4 * pl + o, f[2]);
        st_pop<S>(df + 1 * pl + o, f[3] + k.ms);
        st_pop<S>(df + 2 * pl + o, f[4]);
        st_pop<S>(df + 7 * pl + o, f[5] - k.md);
        st_pop<S>(df + 8 * pl + o, f[6] + k.md);
        st_pop<S>(df + 5 * pl + o, f[7] + k.md);
        st_pop<S>(df + 6 * pl + o, f[8] - k.md);
        return;
    }
    // Fluid relaxation and Guo source in FP64 on the FP32 moments, rounded
    // once on the store.  In the double layer the y-force is ~1e3-1e4 x the
    // x-force and the diagonal populations carry both: FP32 sums such as
    // g_x + g_y of the diagonal source terms would cost the x-force a relative
    // 1e-4 of its diagonal share every step (measured: u_x error 6e-5 against
    // 2e-6 with this form).
    const CollK<double> kd{k.wpd, k.wmd, k.spd, k.smd, k.kcud, k.hinvcs2d, k.gFd, k.inv_cs2d, k.dtd};
    double fd[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) fd[q] = (double)f[q];
    const double uxd = ux, uyd = uy;
    trt_dev<double>(fd, (double)drho, (double)rho, uxd, uyd, uxd * uxd + uyd * uyd, k.wpd, k.wmd, kd);
    if (k.flags & EK_FLAG_FORCE) add_guo<double>(fd, uxd, uyd, (double)fx, (double)fy, kd);
#pragma unroll
    for (int d = 0; d < 9; ++d) st_pop<S>(df + d * pl + o, (float)fd[d]);
}

template <typename S, bool FIRST, bool EXPLICIT_E>
__device__ __forceinline__ void node_shifted(const ChanF &k, const S *__restrict__ src, S *__restrict__ dst,
                                             double *__restrict__ fields, int x, int y, bool moments) {
    float f[9], h[9], t[9];
    gather_global<S, FIRST>(k, src, x, y, f, h, t);
    collide_shifted<S, FIRST, EXPLICIT_E>(k, f, h, t, src, dst, fields, x, y, moments);
}

// Equilibrium deviations from the fields (pre-collision layout).
template <typename S>
__device__ __forceinline__ void init_node_shifted(const ChanF &k, S *__restrict__ pops, const double *__restrict__ fields,
                                                  bool explicit_e, int x, int y) {
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
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const float vx = ux + mob[s] * Ex, vy = uy + mob[s] * Ey;
        const float usq = k.hinvcs2 * (vx * vx + vy * vy);
        const float dd = (float)(densd[s] - 36.0 * (double)__ldg(k.kref + s * k.ny + y));
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
#pragma unroll
        for (int d = 0; d < 9; ++d) st_pop<S>(pops + (s * 9 + d) * pl + o, e[d]);
    }
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
    const float wint = d == 0 ? 16.0f : (d < 5 ? 4.0f : 1.0f);
    const float corr = wint * (kold[s * ny + y] - knew[s * ny + y]);
    st_pop<S>(p, ld_pop<S>(p) + corr);
}

ChanF make_chanf(const Chan &c);

}  // namespace ek
