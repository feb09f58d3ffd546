// ek_init.cu -- kernels of the Poisson-Boltzmann start.
//
// The reference's start (initialization, LBM.cu:95-145) sets the fields of
// gpu_initialization (LBM.cu:147-160) and then iterates gpu_PBE
// (c+- = chargeinf exp(-+ e psi/kT), LBM.cu:139-145), fast_Poisson and
// gpu_PBE_phi (psi = omega psi + (1-omega) psi_old, LBM.cu:132-137).
// The Newton start (new) solves the same equation column by column to
// convergence (pb_newton).
#include <cuda_runtime.h>

#include "ek_internal.h"

namespace ek {
namespace {

constexpr int ITPB = 128;

// gpu_initialization: rho0, u = 0, psi = voltage (the lower wall value), E = 0.
__global__ void pb_fill(const Chan c, double *__restrict__ fields, double *__restrict__ psi_old) {
    const int x = blockIdx.x * ITPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const size_t pl = c.plane, o = (size_t)y * c.nxp + x;
    fields[F_RHO * pl + o] = c.rho0;
    fields[F_UX * pl + o] = 0.0;
    fields[F_UY * pl + o] = 0.0;
    fields[F_EX * pl + o] = 0.0;
    fields[F_EY * pl + o] = 0.0;
    fields[F_PSI * pl + o] = c.zlo[x];
    psi_old[o] = c.zlo[x];
}

// gpu_PBE: Boltzmann concentrations from the current psi.
__global__ void pb_conc(const Chan c, double e_kt, double *__restrict__ fields) {
    const int x = blockIdx.x * ITPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const size_t pl = c.plane, o = (size_t)y * c.nxp + x;
    const double v = fields[F_PSI * pl + o];
    fields[F_CP * pl + o] = c.c0 * exp(-e_kt * v);
    fields[F_CN * pl + o] = c.c0 * exp(e_kt * v);
}

// gpu_PBE_phi: under-relaxation against the previous iterate.
__global__ void pb_relax(const Chan c, double omega, double *__restrict__ fields, double *__restrict__ psi_old) {
    const int x = blockIdx.x * ITPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const size_t o = (size_t)y * c.nxp + x;
    double *psi = fields + F_PSI * c.plane;
    const double v = omega * psi[o] + (1.0 - omega) * psi_old[o];
    psi[o] = v;
    psi_old[o] = v;
}

dim3 grid_of(const Chan &c) { return dim3((c.nx + ITPB - 1) / ITPB, c.ny, 1); }

// Damped Newton iteration of the discrete 1D Poisson-Boltzmann equation down
// one column (rows 1..ny-2):
//   (psi_{j-1} - 2 psi_j + psi_{j+1})/dy^2 + g (exp(-a psi_j) - exp(a psi_j)) = 0,
// psi_0 = zl, psi_{ny-1} = zh, g = f_charge c0/eps, a = e/kT; one thread per
// column q (a distinct pair of wall potentials, walls[q]), from the linear
// profile.  Each step solves J delta = -G by the Thomas algorithm (off-
// diagonals 1/dy^2) and changes a*psi by at most 1; after |a delta| falls
// below 1e-9 of the wall scale two more full steps reach rounding (Newton
// converges quadratically).  Column q's values sit at psi[j * ncol + q] (and
// the Thomas coefficients cp, dp alike), so a warp's accesses are coalesced.
// ok[q] = 1 when the column converged within 500 steps.
__global__ void pb_newton(int ny, double dy, double g, double a, const double2 *__restrict__ walls, int ncol,
                          double *__restrict__ psi, double *__restrict__ cp, double *__restrict__ dp,
                          int *__restrict__ ok) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ncol) return;
    const double zl = walls[q].x, zh = walls[q].y;
    auto P = [&](int j) -> double & { return psi[(size_t)j * ncol + q]; };
    auto CP = [&](int j) -> double & { return cp[(size_t)j * ncol + q]; };
    auto DP = [&](int j) -> double & { return dp[(size_t)j * ncol + q]; };
    for (int j = 0; j < ny; ++j) P(j) = zl + (zh - zl) * (double)j / (double)(ny - 1);
    const int n = ny - 2;
    const double inv = 1.0 / (dy * dy);
    const double scale = fmax(fmax(fabs(zl), fabs(zh)), 1.0);
    int polish = -1;
    for (int it = 0; it < 500; ++it) {
        // forward sweep: residual, Jacobian diagonal and the Thomas elimination together
        double pm = P(0), pc = P(1);
        double cprev = 0.0, dprev = 0.0;
        for (int j = 0; j < n; ++j) {
            const double pn = P(j + 2);
            const double em = exp(-a * pc), ep = exp(a * pc);
            const double G = (pm - 2.0 * pc + pn) * inv + g * (em - ep);
            const double diag = -2.0 * inv - g * a * (em + ep);
            const double den = j == 0 ? diag : diag - inv * cprev;
            cprev = inv / den;
            dprev = (j == 0 ? -G : -G - inv * dprev) / den;
            CP(j) = cprev;
            DP(j) = dprev;
            pm = pc;
            pc = pn;
        }
        // back substitution and the largest |a delta|
        double next = 0.0, dmax = 0.0;
        for (int j = n - 1; j >= 0; --j) {
            const double d = DP(j) - (j == n - 1 ? 0.0 : CP(j) * next);
            DP(j) = d;
            next = d;
            dmax = fmax(dmax, fabs(a * d));
        }
        const double damp = dmax > 1.0 ? 1.0 / dmax : 1.0;
        for (int j = 0; j < n; ++j) P(j + 1) += damp * DP(j);
        if (polish < 0 && damp == 1.0 && dmax < 1e-9 * scale) polish = 2;
        if (polish >= 0 && polish-- == 0) {
            ok[q] = 1;
            return;
        }
    }
    ok[q] = 0;
}

// The Newton start's fields: psi of the node's column, Boltzmann
// concentrations c0 exp(-+ a psi), rho0, u = 0 (E follows from psi).
__global__ void pb_newton_fill(const Chan c, double a, const double *__restrict__ psi, const int *__restrict__ colmap,
                               int ncol, double *__restrict__ fields) {
    const int x = blockIdx.x * ITPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= c.nx) return;
    const size_t pl = c.plane, o = (size_t)y * c.nxp + x;
    const double v = psi[(size_t)y * ncol + colmap[x]];
    fields[F_RHO * pl + o] = c.rho0;
    fields[F_UX * pl + o] = 0.0;
    fields[F_UY * pl + o] = 0.0;
    fields[F_PSI * pl + o] = v;
    fields[F_CP * pl + o] = c.c0 * exp(-a * v);
    fields[F_CN * pl + o] = c.c0 * exp(a * v);
}

}  // namespace

cudaError_t launch_pb_newton(const Chan &c, double dy, double g, double a, const double2 *walls, int ncol,
                             double *psi, double *cp, double *dp, int *ok, const int *colmap, double *fields,
                             cudaStream_t s) {
    pb_newton<<<(ncol + 63) / 64, 64, 0, s>>>(c.ny, dy, g, a, walls, ncol, psi, cp, dp, ok);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pb_newton_fill<<<grid_of(c), ITPB, 0, s>>>(c, a, psi, colmap, ncol, fields);
    return cudaGetLastError();
}

cudaError_t launch_pb_fill(const Chan &c, double *fields, double *psi_old, cudaStream_t s) {
    pb_fill<<<grid_of(c), ITPB, 0, s>>>(c, fields, psi_old);
    return cudaGetLastError();
}

cudaError_t launch_pb_conc(const Chan &c, double e_kt, double *fields, cudaStream_t s) {
    pb_conc<<<grid_of(c), ITPB, 0, s>>>(c, e_kt, fields);
    return cudaGetLastError();
}

cudaError_t launch_pb_relax(const Chan &c, double omega, double *fields, double *psi_old, cudaStream_t s) {
    pb_relax<<<grid_of(c), ITPB, 0, s>>>(c, omega, fields, psi_old);
    return cudaGetLastError();
}

}  // namespace ek
