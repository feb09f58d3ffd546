// ek_init.cu -- kernels of the Poisson-Boltzmann start.
//
// The reference's start (initialization, LBM.cu:95-145) sets the fields of
// gpu_initialization (LBM.cu:147-160) and then iterates gpu_PBE
// (c+- = chargeinf exp(-+ e psi/kT), LBM.cu:139-145), fast_Poisson and
// gpu_PBE_phi (psi = omega psi + (1-omega) psi_old, LBM.cu:132-137).
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

}  // namespace

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
