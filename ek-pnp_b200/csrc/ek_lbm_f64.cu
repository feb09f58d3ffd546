// ek_lbm_f64.cu -- FP64 fused pull-scheme step in the reference's arithmetic
// order.  One thread per node; one launch does what the reference does in four
// (gpu_collide_save, gpu_boundary, gpu_stream, gpu_bc_charge, LBM.cu:307-1024)
// and also writes the Poisson right-hand side (odd_extension's interior
// values, poisson.cu:220-263).
//
// Arithmetic: every expression that sets a population, a moment or a force
// keeps the operation order of the reference kernel it restates (cited at each
// place), so that a build with the same compiler contracts and rounds it the
// same way.  That is what lets the FP64 form match the reference build to
// 1e-12 after tens of thousands of steps; the code around those expressions
// (pull gather, wall handling, buffers) is this project's own.
//
// Wall semantics restated for the pull scheme:
//   fluid  walls store their pre-collision populations reversed (full-way
//          bounce-back, LBM.cu:816-846) as their "post-collision" output, and
//          keep the rest population unchanged (the reference restores it from
//          f0bc each step, LBM.cu:347-349, 818, 838).  Wall rows pull with the
//          periodic y-wrap of gpu_stream (LBM.cu:869-872).
//   ions   walls store their raw post-collision populations (what gpu_stream
//          pushes to the neighbours) and apply the Dirichlet anti-bounce-back
//          of gpu_bc_charge (LBM.cu:935-1020) to their own stored values when
//          they load them on the next step.
//   lower wall velocity: minus the velocity of row 1 from row 1's
//          PRE-collision populations (LBM.cu:402-443; the reference may read
//          row 1's rest populations after they were overwritten in place).
#include <cuda_runtime.h>

#include "ek_internal.h"

namespace ek {
namespace {

constexpr int TPB = 128;

__device__ __forceinline__ double sum9(const double t[9]) {
    return t[0] + t[1] + t[2] + t[3] + t[4] + t[5] + t[6] + t[7] + t[8];
}

// Load the nine populations stored at (x, y) of one species.  I: the index
// type, uint32_t where the 27 population planes fit 2^32 elements (32-bit
// offsets from the buffer's base pointer spare the 64-bit address arithmetic).
template <typename I>
__device__ __forceinline__ void own9(const double *__restrict__ b, I pl, I o, double p[9]) {
#pragma unroll
    for (int d = 0; d < 9; ++d) p[d] = __ldg(b + ((I)d * pl + o));
}

// Pull: direction d arrives from (x - cx_d, y - cy_d).  xm/xp and ym/yp are
// the periodic neighbours (gpu_stream wraps x and y, LBM.cu:869-872).
template <typename I>
__device__ __forceinline__ void pull9(const double *__restrict__ b, I pl, int nxp, int x,
                                      int y, int xm, int xp, int ym, int yp, double p[9]) {
    const I r0 = (I)y * (I)nxp, rm = (I)ym * (I)nxp, rp = (I)yp * (I)nxp;
    p[0] = __ldg(b + (r0 + (I)x));
    p[1] = __ldg(b + (1 * pl + r0 + (I)xm));
    p[2] = __ldg(b + (2 * pl + rm + (I)x));
    p[3] = __ldg(b + (3 * pl + r0 + (I)xp));
    p[4] = __ldg(b + (4 * pl + rp + (I)x));
    p[5] = __ldg(b + (5 * pl + rm + (I)xm));
    p[6] = __ldg(b + (6 * pl + rm + (I)xp));
    p[7] = __ldg(b + (7 * pl + rp + (I)xp));
    p[8] = __ldg(b + (8 * pl + rp + (I)xm));
}

// Dirichlet anti-bounce-back of one ion species at a wall node, applied to the
// node's own post-collision populations q (gpu_bc_charge, LBM.cu:916-943).
__device__ __forceinline__ void ion_wall(const double q[9], double cw, double p[9]) {
    const double m0 = 2.0 * cw * W0, ms = 2.0 * cw * WS, md = 2.0 * cw * WD;
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

// w*dens*(omusq + cu*(1 + cu/2)) -- LBM.cu:491-552
__device__ __forceinline__ double feq_term(double wd, double om, double cu) {
    return wd * (om + cu * (1.0 + 0.5 * cu));
}

__device__ __forceinline__ void equilibria(double dens, double tux, double tuy, double om,
                                           double om_rest, double e[9]) {
    const double w0d = W0 * dens, wsd = WS * dens, wdd = WD * dens;
    e[0] = w0d * (om_rest);
    e[1] = feq_term(wsd, om, tux);
    e[2] = feq_term(wsd, om, tuy);
    e[3] = feq_term(wsd, om, -tux);
    e[4] = feq_term(wsd, om, -tuy);
    e[5] = feq_term(wdd, om, tux + tuy);
    e[6] = feq_term(wdd, om, tuy - tux);
    e[7] = feq_term(wdd, om, -(tux + tuy));
    e[8] = feq_term(wdd, om, tux - tuy);
}

// Guo forcing populations (LBM.cu:556-572); e_i = c_i/CFL.
__device__ __forceinline__ void guo_pops(double ux, double uy, double fx, double fy, double cs2,
                                         double cfl, double s[9]) {
    const double coe0 = W0 / cs2, coes = WS / cs2, coed = WD / cs2;
    const double ci = 1.0 / cfl;
    s[0] = coe0 * (-ux * fx - uy * fy);
    s[1] = coes * (((ci - ux) + (ci * ux) * ci / cs2) * fx - uy * fy);
    s[2] = coes * (-ux * fx + ((ci - uy) + (ci * uy) * ci / cs2) * fy);
    s[3] = coes * (((-ci - ux) + (ci * ux) * ci / cs2) * fx - uy * fy);
    s[4] = coes * (-ux * fx + ((-ci - uy) + (ci * uy) * ci / cs2) * fy);
    const double ci2 = ci * ci / cs2;
    s[5] = coed * (((ci - ux) + (ux + uy) * ci2) * fx + ((ci - uy) + (ux + uy) * ci2) * fy);
    s[6] = coed * (((-ci - ux) + (ux - uy) * ci2) * fx + ((ci - uy) + (-ux + uy) * ci2) * fy);
    s[7] = coed * (((-ci - ux) + (ux + uy) * ci2) * fx + ((-ci - uy) + (ux + uy) * ci2) * fy);
    s[8] = coed * (((ci - ux) + (ux - uy) * ci2) * fx + ((-ci - uy) + (-ux + uy) * ci2) * fy);
}

// TRT relaxation of one opposite pair (a, b = opp(a)) -- LBM.cu:574-803.
__device__ __forceinline__ void trt_pair(double ta, double tb, double ea, double eb, double wp,
                                         double wm, double *oa, double *ob) {
    const double p = 0.5 * (ta + tb), m = 0.5 * (ta - tb);
    const double ep = 0.5 * (ea + eb), em = 0.5 * (ea - eb);
    *oa = ta - (wp * (p - ep) + wm * (m - em));
    *ob = tb - (wp * (p - ep) + wm * (-m - -em));
}

__device__ __forceinline__ void relax(const double t[9], const double e[9], double wp, double wm,
                                      double o[9]) {
    o[0] = t[0] - (wp * (t[0] - e[0]) + wm * (0.0 - 0.0));
    trt_pair(t[1], t[3], e[1], e[3], wp, wm, &o[1], &o[3]);
    trt_pair(t[2], t[4], e[2], e[4], wp, wm, &o[2], &o[4]);
    trt_pair(t[5], t[7], e[5], e[7], wp, wm, &o[5], &o[7]);
    trt_pair(t[6], t[8], e[6], e[8], wp, wm, &o[6], &o[8]);
}

// Field E at a node from psi: central differences with periodic x, and the
// wall rows take the adjacent row's Ey (gpu_efield + gpu_bc, poisson.cu:145-174).
__device__ __forceinline__ void efield_at(const double *__restrict__ psi, const Chan &c, int x,
                                          int y, int xm, int xp, double *ex, double *ey) {
    const size_t r = (size_t)y * c.nxp;
    *ex = 0.5 * (__ldg(psi + r + xm) - __ldg(psi + r + xp)) / c.dx;
    const int yc = y == 0 ? 1 : (y == c.ny - 1 ? c.ny - 2 : y);
    *ey = 0.5 * (__ldg(psi + (size_t)(yc - 1) * c.nxp + x) - __ldg(psi + (size_t)(yc + 1) * c.nxp + x)) / c.dy;
}

// The raw populations of node (x, y) as stored: FIRST -> its own values;
// otherwise the fluid pulled from the neighbours and the ions pulled
// (interior rows) or the node's own values (wall rows, reflected by node_f64).
template <bool FIRST, typename I>
__device__ __forceinline__ void gather_f64(const Chan &c, const double *__restrict__ src, int x, int y, double ft[9],
                                           double ht[9], double tt[9]) {
    const I pl = (I)c.plane;
    const int nxp = c.nxp;
    const I o = (I)y * (I)nxp + (I)x;
    const int xm = x == 0 ? c.nx - 1 : x - 1, xp = x + 1 == c.nx ? 0 : x + 1;
    const int ym = y == 0 ? c.ny - 1 : y - 1, yp = y + 1 == c.ny ? 0 : y + 1;
    const double *sf = src, *sh = src + 9 * pl, *st = src + 18 * pl;
    if (FIRST) {
        own9(sf, pl, o, ft);
        own9(sh, pl, o, ht);
        own9(st, pl, o, tt);
    } else {
        pull9(sf, pl, nxp, x, y, xm, xp, ym, yp, ft);
        if (y == 0 || y == c.ny - 1) {
            own9(sh, pl, o, ht);
            own9(st, pl, o, tt);
        } else {
            pull9(sh, pl, nxp, x, y, xm, xp, ym, yp, ht);
            pull9(st, pl, nxp, x, y, xm, xp, ym, yp, tt);
        }
    }
}

// The update of node (x, y) from its raw populations (gather_f64): ion
// anti-bounce-back at the walls, moments, E, force, right-hand side,
// equilibria, Guo source, TRT and the stores.  src is read only for the lower
// wall's row-1 pull.
template <bool FIRST, bool EXPLICIT_E, bool MOMENTS, typename I>
__device__ __forceinline__ void node_f64(const Chan &c, double ft[9], double ht_raw[9], double tt_raw[9],
                                         const double *__restrict__ src, double *__restrict__ dst,
                                         double *__restrict__ fields, int x, int y) {
    const I pl = (I)c.plane;
    const int nxp = c.nxp;
    const I o = (I)y * (I)nxp + (I)x;
    const bool lo = y == 0, hi = y == c.ny - 1;
    const int xm = x == 0 ? c.nx - 1 : x - 1, xp = x + 1 == c.nx ? 0 : x + 1;
    const double *sf = src;

    double ht[9], tt[9];
    if (!FIRST && (lo || hi)) {
        ion_wall(ht_raw, lo ? c.cplo[x] : c.cphi[x], ht);
        ion_wall(tt_raw, lo ? c.cnlo[x] : c.cnhi[x], tt);
    } else {
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            ht[d] = ht_raw[d];
            tt[d] = tt_raw[d];
        }
    }

    // moments, LBM.cu:382-392
    const double rho = sum9(ft);
    const double rhoinv = 1.0 / rho;
    const double charge = sum9(ht);
    const double temp = sum9(tt);
    double Ex, Ey;
    if (EXPLICIT_E) {
        Ex = __ldg(fields + F_EX * pl + o);
        Ey = __ldg(fields + F_EY * pl + o);
    } else {
        efield_at(fields + F_PSI * pl, c, x, y, xm, xp, &Ex, &Ey);
    }
    double forcex = 0.0, forcey = 0.0;
    if (c.flags & EK_FLAG_FORCE) {  // the expression commented out at LBM.cu:388-389
        forcex = c.f_charge * (charge - temp) * (Ex + c.ext_x) + c.exf;
        forcey = c.f_charge * (charge - temp) * Ey;
    }
    double ux = rhoinv * ((ft[1] + ft[5] + ft[8] - (ft[3] + ft[6] + ft[7])) / c.cfl + forcex * c.dt * 0.5);
    double uy = rhoinv * ((ft[2] + ft[5] + ft[6] - (ft[4] + ft[7] + ft[8])) / c.cfl + forcey * c.dt * 0.5);
    if (lo) {
        // lower wall: minus the velocity of row 1 (LBM.cu:402-443)
        double fm[9];
        const I o1 = (I)nxp + (I)x;
        if (FIRST) own9(sf, pl, o1, fm);
        else pull9(sf, pl, nxp, x, 1, xm, xp, 0, 2, fm);
        const double rhoinvm = 1.0 / sum9(fm);
        ux = -rhoinvm * ((fm[1] + fm[5] + fm[8] - (fm[3] + fm[6] + fm[7])) / c.cfl + forcex * c.dt * 0.5);
        uy = -rhoinvm * ((fm[2] + fm[5] + fm[6] - (fm[4] + fm[7] + fm[8])) / c.cfl + forcey * c.dt * 0.5);
    }
    if (MOMENTS) {
        fields[F_RHO * pl + o] = rho;
        fields[F_UX * pl + o] = ux;
        fields[F_UY * pl + o] = uy;
        fields[F_CP * pl + o] = charge;
        fields[F_CN * pl + o] = temp;
    }
    if (!lo && !hi) {
        // Poisson right-hand side with the Dirichlet lifting (poisson.cu:228-241)
        double v = -c.f_charge * (charge - temp) / c.eps;
        if (y == 1) v = v - c.zlo[x] / c.dy / c.dy;
        if (y == c.ny - 2) v = v - c.zhi[x] / c.dy / c.dy;
        fields[F_RHS * pl + o] = v;
    }

    // ion equilibria in the drift velocities u + K E (LBM.cu:479-552)
    const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy) / c.cs2;
    const double omusq_c = 1.0 - 0.5 * ((ux + c.mob_p * Ex) * (ux + c.mob_p * Ex) + (uy + c.mob_p * Ey) * (uy + c.mob_p * Ey)) / c.cs2;
    const double omusq_cn = 1.0 - 0.5 * ((ux + c.mob_n * Ex) * (ux + c.mob_n * Ex) + (uy + c.mob_n * Ey) * (uy + c.mob_n * Ey)) / c.cs2;
    {
        double e[9], out[9];
        equilibria(charge, (ux + c.mob_p * Ex) / c.cs2 / c.cfl, (uy + c.mob_p * Ey) / c.cs2 / c.cfl,
                   omusq_c, omusq_c, e);
        relax(ht, e, c.r.wcp, c.r.wcm, out);
        double *dh = dst + 9 * pl;
#pragma unroll
        for (int d = 0; d < 9; ++d) dh[d * pl + o] = out[d];
        equilibria(temp, (ux + c.mob_n * Ex) / c.cs2 / c.cfl, (uy + c.mob_n * Ey) / c.cs2 / c.cfl,
                   omusq_cn, (c.flags & EK_FLAG_REST_QUIRK) ? omusq : omusq_cn, e);
        relax(tt, e, c.r.wtp, c.r.wtm, out);
        double *dt_ = dst + 18 * pl;
#pragma unroll
        for (int d = 0; d < 9; ++d) dt_[d * pl + o] = out[d];
    }

    double *df = dst;
    if (lo) {
        df[o] = ft[0];
#pragma unroll
        for (int d = 1; d < 9; ++d) df[oppd(d) * pl + o] = ft[d];
        return;
    }
    if (hi) {
        const double ms = c.r.ms, md = c.r.md;
        df[o] = ft[0];
        df[3 * pl + o] = ft[1] - ms;
        df[4 * pl + o] = ft[2];
        df[1 * pl + o] = ft[3] + ms;
        df[2 * pl + o] = ft[4];
        df[7 * pl + o] = ft[5] - md;
        df[8 * pl + o] = ft[6] + md;
        df[5 * pl + o] = ft[7] + md;
        df[6 * pl + o] = ft[8] - md;
        return;
    }
    // fluid: equilibrium, Guo source, TRT (LBM.cu:468-803)
    double e[9], fpop[9];
    equilibria(rho, ux / c.cs2 / c.cfl, uy / c.cs2 / c.cfl, omusq, omusq, e);
    guo_pops(ux, uy, forcex, forcey, c.cs2, c.cfl, fpop);
    const double sp = c.r.sp, sm = c.r.sm, dt = c.dt;
    double src9[9];
    src9[0] = sp * fpop[0];
    {
        const int a[4] = {1, 2, 5, 6};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = a[k], j = oppd(i);
            const double fp = 0.5 * (fpop[i] + fpop[j]), fmn = 0.5 * (fpop[i] - fpop[j]);
            src9[i] = sp * fp + sm * fmn;
            src9[j] = sp * fp + sm * -fmn;
        }
    }
    double out[9];
    relax(ft, e, c.r.wp, c.r.wm, out);
#pragma unroll
    for (int d = 0; d < 9; ++d) df[d * pl + o] = out[d] + dt * src9[d];
}

template <bool FIRST, bool EXPLICIT_E, bool MOMENTS, typename I>
__global__ void __launch_bounds__(TPB)
step_f64(const Chan c, const double *__restrict__ src, double *__restrict__ dst,
         double *__restrict__ fields) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    double ft[9], ht[9], tt[9];
    gather_f64<FIRST, I>(c, src, x, y, ft, ht, tt);
    node_f64<FIRST, EXPLICIT_E, MOMENTS, I>(c, ft, ht, tt, src, dst, fields, x, y);
}

__global__ void rates_kernel(ek_params p, Rates *out) {
    // LBM.cu:336-341
    const double omega_plus = 1.0 / (p.nu / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double omega_minus = 1.0 / (p.magic_f / (p.nu / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    const double omega_c_minus = 1.0 / (p.diff_p / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double omega_c_plus = 1.0 / (p.magic_p / (p.diff_p / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    const double omega_T_minus = 1.0 / (p.diff_n / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double omega_T_plus = 1.0 / (p.magic_n / (p.diff_n / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    Rates r;
    r.wp = omega_plus * p.dt;
    r.wm = omega_minus * p.dt;
    r.wcp = omega_c_plus * p.dt;
    r.wcm = omega_c_minus * p.dt;
    r.wtp = omega_T_plus * p.dt;
    r.wtm = omega_T_minus * p.dt;
    r.sp = 1.0 - 0.5 * p.dt * omega_plus;   // LBM.cu:745-746
    r.sm = 1.0 - 0.5 * p.dt * omega_minus;
    r.ms = 2.0 * p.rho0 * p.uw / p.cs2 * WS / p.cfl;  // LBM.cu:812-813
    r.md = 2.0 * p.rho0 * p.uw / p.cs2 * WD / p.cfl;
    *out = r;
}

// Equilibrium populations from the fields, written in place (pre-collision
// layout): gpu_init_equilibrium, LBM.cu:195-305.
__global__ void __launch_bounds__(TPB)
init_f64(const Chan c, double *__restrict__ pops, const double *__restrict__ fields, bool explicit_e) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const size_t pl = c.plane, o = (size_t)y * c.nxp + x;
    const int xm = x == 0 ? c.nx - 1 : x - 1, xp = x + 1 == c.nx ? 0 : x + 1;
    const double rho = fields[F_RHO * pl + o], ux = fields[F_UX * pl + o], uy = fields[F_UY * pl + o];
    const double charge = fields[F_CP * pl + o], Temp = fields[F_CN * pl + o];
    double Ex, Ey;
    if (explicit_e) {
        Ex = fields[F_EX * pl + o];
        Ey = fields[F_EY * pl + o];
    } else {
        efield_at(fields + F_PSI * pl, c, x, y, xm, xp, &Ex, &Ey);
    }
    const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy) / c.cs2;
    const double omusq_c = 1.0 - 0.5 * ((ux + c.mob_p * Ex) * (ux + c.mob_p * Ex) + (uy + c.mob_p * Ey) * (uy + c.mob_p * Ey)) / c.cs2;
    const double omusq_cn = 1.0 - 0.5 * ((ux + c.mob_n * Ex) * (ux + c.mob_n * Ex) + (uy + c.mob_n * Ey) * (uy + c.mob_n * Ey)) / c.cs2;
    double e[9];
    equilibria(rho, ux / c.cs2 / c.cfl, uy / c.cs2 / c.cfl, omusq, omusq, e);
#pragma unroll
    for (int d = 0; d < 9; ++d) pops[d * pl + o] = e[d];
    equilibria(charge, (ux + c.mob_p * Ex) / c.cs2 / c.cfl, (uy + c.mob_p * Ey) / c.cs2 / c.cfl,
               omusq_c, omusq_c, e);
#pragma unroll
    for (int d = 0; d < 9; ++d) pops[(9 + d) * pl + o] = e[d];
    equilibria(Temp, (ux + c.mob_n * Ex) / c.cs2 / c.cfl, (uy + c.mob_n * Ey) / c.cs2 / c.cfl,
               omusq_cn, omusq_cn, e);
#pragma unroll
    for (int d = 0; d < 9; ++d) pops[(18 + d) * pl + o] = e[d];
}

__global__ void __launch_bounds__(TPB) efield_f64(const Chan c, double *__restrict__ fields) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const int xm = x == 0 ? c.nx - 1 : x - 1, xp = x + 1 == c.nx ? 0 : x + 1;
    double Ex, Ey;
    efield_at(fields + F_PSI * c.plane, c, x, y, xm, xp, &Ex, &Ey);
    const size_t o = (size_t)y * c.nxp + x;
    fields[F_EX * c.plane + o] = Ex;
    fields[F_EY * c.plane + o] = Ey;
}

// Right-hand side from the stored moments (for a Poisson solve outside a step).
__global__ void __launch_bounds__(TPB) rhs_f64(const Chan c, double *__restrict__ fields) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y + 1;
    if (x >= c.nx || y > c.ny - 2) return;
    const size_t pl = c.plane, o = (size_t)y * c.nxp + x;
    double v = -c.f_charge * (fields[F_CP * pl + o] - fields[F_CN * pl + o]) / c.eps;
    if (y == 1) v = v - c.zlo[x] / c.dy / c.dy;
    if (y == c.ny - 2) v = v - c.zhi[x] / c.dy / c.dy;
    fields[F_RHS * pl + o] = v;
}

dim3 node_grid(const Chan &c, int rows) { return dim3((c.nx + TPB - 1) / TPB, rows, 1); }

}  // namespace

cudaError_t launch_rates(const ek_params &p, Rates *dev_out, cudaStream_t s) {
    rates_kernel<<<1, 1, 0, s>>>(p, dev_out);
    return cudaGetLastError();
}

cudaError_t launch_init_f64(const Chan &c, double *pops, const double *fields, bool explicit_e,
                            cudaStream_t s) {
    init_f64<<<node_grid(c, c.ny), TPB, 0, s>>>(c, pops, fields, explicit_e);
    return cudaGetLastError();
}

cudaError_t launch_step_f64(const Chan &c, const double *src, double *dst, double *fields,
                            bool first, bool explicit_e, bool moments, cudaStream_t s) {
    const dim3 g = node_grid(c, c.ny);
    // 32-bit offsets while the 27 population planes fit 2^32 elements
    const bool i32 = (size_t)27 * c.plane < ((size_t)1 << 32);
#define EK_STEP(F, E, M)                                                                       \
    do {                                                                                       \
        if (i32) step_f64<F, E, M, uint32_t><<<g, TPB, 0, s>>>(c, src, dst, fields);           \
        else step_f64<F, E, M, size_t><<<g, TPB, 0, s>>>(c, src, dst, fields);                 \
    } while (0)
    const int key = (first ? 4 : 0) | (explicit_e ? 2 : 0) | (moments ? 1 : 0);
    switch (key) {
        case 0: EK_STEP(false, false, false); break;
        case 1: EK_STEP(false, false, true); break;
        case 2: EK_STEP(false, true, false); break;
        case 3: EK_STEP(false, true, true); break;
        case 4: EK_STEP(true, false, false); break;
        case 5: EK_STEP(true, false, true); break;
        case 6: EK_STEP(true, true, false); break;
        default: EK_STEP(true, true, true); break;
    }
#undef EK_STEP
    return cudaGetLastError();
}

cudaError_t launch_efield_f64(const Chan &c, double *fields, cudaStream_t s) {
    efield_f64<<<node_grid(c, c.ny), TPB, 0, s>>>(c, fields);
    return cudaGetLastError();
}

cudaError_t launch_rhs_from_moments_f64(const Chan &c, double *fields, cudaStream_t s) {
    rhs_f64<<<node_grid(c, c.ny - 2), TPB, 0, s>>>(c, fields);
    return cudaGetLastError();
}

}  // namespace ek
