// ek_jacobi.cu -- grid relaxation of the Poisson equation, the counterpart of
// the reference's iterative solver (poisson_phi / gpu_poisson,
// poisson.cu:35-130), which its time loop never calls (main.cu uses the
// spectral fast_Poisson): kept for geometries that leave the periodic
// channel, where no x-transform applies.
//
// The reference relaxes psi in place with the five-point update
//     psi = (psi_L + psi_R + psi_U + psi_D + dx^2 c / eps) / 4
// on the interior rows, the walls held at voltage / voltage2, until the
// largest change of a sweep is below 1e-9 (at most 1e6 sweeps).  Its blocks
// read neighbours that other blocks may already have overwritten, so the
// iterates depend on the schedule.  Here every sweep reads one buffer and
// writes the other (weighted Jacobi, omega = 1 being the plain update), so
// the iterates are deterministic.  The update, with dx != dy allowed:
//     ((psi_L + psi_R) / dx^2 + (psi_U + psi_D) / dy^2 - rhs) / (2/dx^2 + 2/dy^2),
//     rhs = -f_charge (c+ - c-) / eps,
// the walls at the channel's wall potentials zeta(x).  Its fixed point is
// the five-point discretisation, three-point in x as well as in y, so it
// differs from the spectral solve (exact kx^2 along x, fast_Poisson) by the
// x-discretisation error, O((kx dx)^2 / 12) for mode kx.
#include <cuda_runtime.h>

#include <cstring>

#include "ek_ctx.h"

namespace ek {
namespace {

constexpr int JTPB = 128;

// Right-hand side of the interior rows from the moments (no wall lifting:
// the walls are held in psi itself).
__global__ void __launch_bounds__(JTPB) jacobi_rhs(const Chan c, const double *__restrict__ fields,
                                                   double *__restrict__ rhs) {
    const int x = blockIdx.x * JTPB + threadIdx.x, y = blockIdx.y + 1;
    if (x >= c.nx) return;
    const size_t o = (size_t)y * c.nxp + x;
    rhs[o] = -c.f_charge * (fields[F_CP * c.plane + o] - fields[F_CN * c.plane + o]) / c.eps;
}

// Wall rows of a psi buffer: the Dirichlet values (odd_extract's walls,
// poisson.cu:297-304, and gpu_poisson's, poisson.cu:99-106).
__global__ void __launch_bounds__(JTPB) jacobi_walls(const Chan c, double *__restrict__ psi) {
    const int x = blockIdx.x * JTPB + threadIdx.x;
    if (x >= c.nx) return;
    psi[x] = c.zlo[x];
    psi[(size_t)(c.ny - 1) * c.nxp + x] = c.zhi[x];
}

// One sweep over the interior rows, src -> dst.  With maxchg set, the
// largest |dst - src| of the sweep is folded into *maxchg (the bits of a
// non-negative double order like the double, so an integer max works).
__global__ void __launch_bounds__(JTPB) jacobi_sweep(const Chan c, const double *__restrict__ src,
                                                     double *__restrict__ dst, const double *__restrict__ rhs,
                                                     double omega, unsigned long long *__restrict__ maxchg) {
    const int x = blockIdx.x * JTPB + threadIdx.x, y = blockIdx.y + 1;
    double d = 0.0;
    if (x < c.nx) {
        const int xm = x == 0 ? c.nx - 1 : x - 1, xp = x + 1 == c.nx ? 0 : x + 1;
        const size_t r = (size_t)y * c.nxp, o = r + x;
        const double idx2 = 1.0 / (c.dx * c.dx), idy2 = 1.0 / (c.dy * c.dy);
        const double old = src[o];
        const double fit = ((src[r + xm] + src[r + xp]) * idx2 + (src[o - c.nxp] + src[o + c.nxp]) * idy2 - rhs[o]) /
                           (2.0 * idx2 + 2.0 * idy2);
        const double v = old + omega * (fit - old);
        dst[o] = v;
        d = fabs(v - old);
    }
    if (!maxchg) return;
    for (int off = 16; off > 0; off >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, off));
    if ((threadIdx.x & 31) == 0) atomicMax(maxchg, (unsigned long long)__double_as_longlong(d));
}

}  // namespace
}  // namespace ek

using namespace ek;

extern "C" int ek_poisson_jacobi(ek_ctx *c, int32_t max_sweeps, double tol, double omega, int32_t check_every,
                                 int32_t *sweeps, double *change) {
    if (!c || max_sweeps < 1 || !(tol >= 0.0) || !(omega > 0.0 && omega < 2.0) || check_every < 1)
        return ctx_fail(EK_ERR_INVALID, "ek_poisson_jacobi: null context, max_sweeps < 1, tol < 0, omega outside "
                                        "(0, 2) or check_every < 1");
    if (c->p.ny < 3) return ctx_fail(EK_ERR_INVALID, "ek_poisson_jacobi: no interior rows");
    cudaError_t e = cudaSuccess;
    if (!c->jacobi_word) e = cudaMalloc(&c->jacobi_word, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        c->jacobi_word = nullptr;
        return ctx_fail(EK_ERR_NOMEM, "ek_poisson_jacobi: device word");
    }
    const Chan &ch = c->chan;
    double *psi = c->fields + F_PSI * c->plane;
    double *spare = c->fields + F_EX * c->plane;  // E is recomputed from psi at the end
    double *rhs = c->fields + F_RHS * c->plane;
    const dim3 gi((ch.nx + JTPB - 1) / JTPB, ch.ny - 2), gw((ch.nx + JTPB - 1) / JTPB);
    jacobi_rhs<<<gi, JTPB, 0, c->stream>>>(ch, c->fields, rhs);
    jacobi_walls<<<gw, JTPB, 0, c->stream>>>(ch, psi);
    jacobi_walls<<<gw, JTPB, 0, c->stream>>>(ch, spare);
    c->launches += 3;
    if ((e = cudaGetLastError()) != cudaSuccess) return ctx_fail(EK_ERR_CUDA, cudaGetErrorString(e));
    double *a = psi, *b = spare;
    double last = -1.0;
    int32_t k = 0;
    while (k < max_sweeps) {
        ++k;
        const bool measure = k % check_every == 0 || k == max_sweeps;
        if (measure) e = cudaMemsetAsync(c->jacobi_word, 0, sizeof(unsigned long long), c->stream);
        if (e == cudaSuccess) {
            jacobi_sweep<<<gi, JTPB, 0, c->stream>>>(ch, a, b, rhs, omega, measure ? c->jacobi_word : nullptr);
            ++c->launches;
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return ctx_fail(EK_ERR_CUDA, cudaGetErrorString(e));
        double *t = a;
        a = b;
        b = t;
        if (measure) {
            unsigned long long bits = 0;
            e = cudaMemcpyAsync(&bits, c->jacobi_word, sizeof(bits), cudaMemcpyDeviceToHost, c->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) return ctx_fail(EK_ERR_CUDA, cudaGetErrorString(e));
            std::memcpy(&last, &bits, sizeof(last));
            if (last < tol) break;
        }
    }
    if (a != psi) {
        e = cudaMemcpyAsync(psi, a, c->plane * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return ctx_fail(EK_ERR_CUDA, cudaGetErrorString(e));
    }
    int rc = ctx_after_psi(c);  // E from psi; the FP32 planes follow the FP64 psi
    if (rc != EK_OK) return rc;
    if (sweeps) *sweeps = k;
    if (change) *change = last;
    return EK_OK;
}
