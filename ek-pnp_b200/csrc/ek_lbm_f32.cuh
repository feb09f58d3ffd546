// ek_lbm_f32.cuh -- node update of the shifted-storage forms (FP32 and FP16
// populations, FP32 arithmetic).  Included by the single-channel kernels
// (ek_lbm_f32.cu) and the batched persistent kernel (ek_batch.cu).
//
// Storage: d_i = f_i - w_i*R with R = rho0 for the fluid and c0 for both ion
// species.  Every quantity of the collision is rewritten in deviations so
// that FP32 keeps the small departures from the reference state:
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
    double f_charge, eps, ext_x, exf, dx, dy;
    const double *zlo, *zhi, *cplo, *cphi, *cnlo, *cnhi;
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

// Ion anti-bounce-back in deviations: d_ibar = -q_i + 2 w_i (c_wall - c0).
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

__device__ __forceinline__ float sum9f(const float t[9]) {
    return ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7])) + t[8];
}

// TRT of one pair in deviations.  w: lattice weight, cu: (c_i.u)*kcu,
// base: d_dens - dens*usq (symmetric equilibrium without the cu^2 term).
__device__ __forceinline__ void trt_pair_dev(float &da, float &db, float w, float dens, float cu, float base,
                                             float wp, float wm) {
    const float seq = w * (base + dens * (0.5f * cu * cu));
    const float aeq = w * dens * cu;
    const float s = 0.5f * (da + db), a = 0.5f * (da - db);
    const float ps = wp * (s - seq), pa = wm * (a - aeq);
    da = da - ps - pa;
    db = db - ps + pa;
}

// Full TRT of one species in deviations, in place.  ux, uy: the species'
// advection velocity; usq_rest: u^2 used by the rest equilibrium.
__device__ __forceinline__ void trt_dev(float d[9], float ddens, float dens, float ux, float uy, float usq_rest,
                                        float wp, float wm, const ChanF &k) {
    const float usq = k.hinvcs2 * (ux * ux + uy * uy);
    const float base = ddens - dens * usq;
    const float e0 = W0F * (ddens - dens * (k.hinvcs2 * usq_rest));
    d[0] = d[0] - wp * (d[0] - e0);
    const float cx = ux * k.kcu, cy = uy * k.kcu;
    trt_pair_dev(d[1], d[3], WSF, dens, cx, base, wp, wm);
    trt_pair_dev(d[2], d[4], WSF, dens, cy, base, wp, wm);
    trt_pair_dev(d[5], d[7], WDF, dens, cx + cy, base, wp, wm);
    trt_pair_dev(d[6], d[8], WDF, dens, cy - cx, base, wp, wm);
}

// Guo source added to post-collision fluid deviations.
__device__ __forceinline__ void add_guo(float d[9], float ux, float uy, float fx, float fy, const ChanF &k) {
    const float uF = k.inv_cs2 * (ux * fx + uy * fy);
    const float cux = ux * k.kcu, cuy = uy * k.kcu;
    const float cfx = fx * k.gF, cfy = fy * k.gF;
    const float sp = k.sp * k.dt, sm = k.sm * k.dt;
    d[0] += sp * (W0F * -uF);
    // pair (a, abar) with c_a.u -> cu, c_a.F -> cf
    auto pair = [&](float &da, float &db, float w, float cu, float cf) {
        const float fp = w * (cu * cf - uF), fm = w * cf;
        da += sp * fp + sm * fm;
        db += sp * fp - sm * fm;
    };
    pair(d[1], d[3], WSF, cux, cfx);
    pair(d[2], d[4], WSF, cuy, cfy);
    pair(d[5], d[7], WDF, cux + cuy, cfx + cfy);
    pair(d[6], d[8], WDF, cuy - cux, cfy - cfx);
}

__device__ __forceinline__ void efield_at_d(const double *__restrict__ psi, int nxp, int ny, double dx, double dy,
                                            int x, int y, int xm, int xp, double *ex, double *ey) {
    const size_t r = (size_t)y * nxp;
    *ex = 0.5 * (__ldg(psi + r + xm) - __ldg(psi + r + xp)) / dx;
    const int yc = y == 0 ? 1 : (y == ny - 1 ? ny - 2 : y);
    *ey = 0.5 * (__ldg(psi + (size_t)(yc - 1) * nxp + x) - __ldg(psi + (size_t)(yc + 1) * nxp + x)) / dy;
}

// One node of one step.  src/dst: 27 population planes (species-major);
// fields: the channel's 9 FP64 field planes.
template <typename S, bool FIRST, bool EXPLICIT_E, bool MOMENTS>
__device__ __forceinline__ void node_shifted(const ChanF &k, const S *__restrict__ src, S *__restrict__ dst,
                                             double *__restrict__ fields, int x, int y) {
    const size_t pl = k.plane;
    const int nxp = k.nxp;
    const size_t o = (size_t)y * nxp + x;
    const bool lo = y == 0, hi = y == k.ny - 1;
    const int xm = x == 0 ? k.nx - 1 : x - 1, xp = x + 1 == k.nx ? 0 : x + 1;
    const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
    const S *sf = src, *sh = src + 9 * pl, *st = src + 18 * pl;

    float f[9], h[9], t[9];
    if (FIRST) {
        own9s<S>(sf, pl, o, f);
        own9s<S>(sh, pl, o, h);
        own9s<S>(st, pl, o, t);
    } else {
        pull9s<S>(sf, pl, nxp, x, y, xm, xp, ym, yp, f);
        if (lo || hi) {
            float q[9];
            own9s<S>(sh, pl, o, q);
            ion_wall_dev(q, (float)((lo ? k.cplo[x] : k.cphi[x]) - (double)k.c0), h);
            own9s<S>(st, pl, o, q);
            ion_wall_dev(q, (float)((lo ? k.cnlo[x] : k.cnhi[x]) - (double)k.c0), t);
        } else {
            pull9s<S>(sh, pl, nxp, x, y, xm, xp, ym, yp, h);
            pull9s<S>(st, pl, nxp, x, y, xm, xp, ym, yp, t);
        }
    }
    const float drho = sum9f(f), dcp = sum9f(h), dcn = sum9f(t);
    const float rho = k.rho0 + drho, cp = k.c0 + dcp, cn = k.c0 + dcn;
    double exd, eyd;
    if (EXPLICIT_E) {
        exd = fields[F_EX * pl + o];
        eyd = fields[F_EY * pl + o];
    } else {
        efield_at_d(fields + F_PSI * pl, nxp, k.ny, k.dx, k.dy, x, y, xm, xp, &exd, &eyd);
    }
    const float Ex = (float)exd, Ey = (float)eyd;
    float fx = 0.0f, fy = 0.0f;
    if (k.flags & EK_FLAG_FORCE) {
        const double q = k.f_charge * ((double)dcp - (double)dcn);
        fx = (float)(q * (exd + k.ext_x) + k.exf);
        fy = (float)(q * eyd);
    }
    const float jx = (f[1] + f[5] + f[8]) - (f[3] + f[6] + f[7]);
    const float jy = (f[2] + f[5] + f[6]) - (f[4] + f[7] + f[8]);
    float ux = (jx * k.inv_cfl + fx * k.half_dt) / rho;
    float uy = (jy * k.inv_cfl + fy * k.half_dt) / rho;
    if (lo) {
        float m[9];
        const size_t o1 = (size_t)nxp + x;
        if (FIRST) own9s<S>(sf, pl, o1, m);
        else pull9s<S>(sf, pl, nxp, x, 1, xm, xp, 0, 2, m);
        const float rho1 = k.rho0 + sum9f(m);
        const float jx1 = (m[1] + m[5] + m[8]) - (m[3] + m[6] + m[7]);
        const float jy1 = (m[2] + m[5] + m[6]) - (m[4] + m[7] + m[8]);
        ux = -(jx1 * k.inv_cfl + fx * k.half_dt) / rho1;
        uy = -(jy1 * k.inv_cfl + fy * k.half_dt) / rho1;
    }
    if (MOMENTS) {
        fields[F_RHO * pl + o] = (double)k.rho0 + (double)drho;
        fields[F_UX * pl + o] = ux;
        fields[F_UY * pl + o] = uy;
        fields[F_CP * pl + o] = (double)k.c0 + (double)dcp;
        fields[F_CN * pl + o] = (double)k.c0 + (double)dcn;
    }
    if (!lo && !hi) {
        double v = -k.f_charge * ((double)dcp - (double)dcn) / k.eps;
        if (y == 1) v = v - k.zlo[x] / k.dy / k.dy;
        if (y == k.ny - 2) v = v - k.zhi[x] / k.dy / k.dy;
        fields[F_RHS * pl + o] = v;
    }
    const float usq_f = ux * ux + uy * uy;
    {
        const float vx = ux + k.mob_p * Ex, vy = uy + k.mob_p * Ey;
        trt_dev(h, dcp, cp, vx, vy, vx * vx + vy * vy, k.wcp, k.wcm, k);
        S *dh = dst + 9 * pl;
#pragma unroll
        for (int d = 0; d < 9; ++d) st_pop<S>(dh + d * pl + o, h[d]);
    }
    {
        const float vx = ux + k.mob_n * Ex, vy = uy + k.mob_n * Ey;
        trt_dev(t, dcn, cn, vx, vy, (k.flags & EK_FLAG_REST_QUIRK) ? usq_f : vx * vx + vy * vy, k.wtp, k.wtm, k);
        S *dt_ = dst + 18 * pl;
#pragma unroll
        for (int d = 0; d < 9; ++d) st_pop<S>(dt_ + d * pl + o, t[d]);
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
    trt_dev(f, drho, rho, ux, uy, usq_f, k.wp, k.wm, k);
    if (k.flags & EK_FLAG_FORCE) add_guo(f, ux, uy, fx, fy, k);
#pragma unroll
    for (int d = 0; d < 9; ++d) st_pop<S>(df + d * pl + o, f[d]);
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
        efield_at_d(fields + F_PSI * pl, k.nxp, k.ny, k.dx, k.dy, x, y, xm, xp, &exd, &eyd);
    }
    const float ux = (float)fields[F_UX * pl + o], uy = (float)fields[F_UY * pl + o];
    const float Ex = (float)exd, Ey = (float)eyd;
    const float dens[3] = {(float)fields[F_RHO * pl + o], (float)fields[F_CP * pl + o], (float)fields[F_CN * pl + o]};
    const float ref[3] = {k.rho0, k.c0, k.c0};
    const float mob[3] = {0.0f, k.mob_p, k.mob_n};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const float vx = ux + mob[s] * Ex, vy = uy + mob[s] * Ey;
        const float usq = k.hinvcs2 * (vx * vx + vy * vy);
        const float dd = (float)((double)dens[s] - (double)ref[s]);
        const float base = dd - dens[s] * usq;
        const float cx = vx * k.kcu, cy = vy * k.kcu;
        float e[9];
        e[0] = W0F * base;
        const float cu[4] = {cx, cy, cx + cy, cy - cx};
        const int ia[4] = {1, 2, 5, 6};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float w = q < 2 ? WSF : WDF;
            const float sym = w * (base + dens[s] * 0.5f * cu[q] * cu[q]);
            const float anti = w * dens[s] * cu[q];
            e[ia[q]] = sym + anti;
            e[oppd(ia[q])] = sym - anti;
        }
#pragma unroll
        for (int d = 0; d < 9; ++d) st_pop<S>(pops + (s * 9 + d) * pl + o, e[d]);
    }
}

ChanF make_chanf(const Chan &c);

}  // namespace ek
