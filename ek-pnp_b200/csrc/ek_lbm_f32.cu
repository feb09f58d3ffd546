// ek_lbm_f32.cu -- single-channel kernels of the shifted-storage forms
// (FP32 / FP16 populations).  The node update lives in ek_lbm_f32.cuh.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ek_lbm_f32.cuh"

namespace ek {

ChanF make_chanf(const Chan &c) {
    ChanF k;
    k.nx = c.nx;
    k.ny = c.ny;
    k.nxp = c.nxp;
    k.flags = c.flags;
    k.plane = c.plane;
    k.wp = (float)c.r.wp;
    k.wm = (float)c.r.wm;
    k.wcp = (float)c.r.wcp;
    k.wcm = (float)c.r.wcm;
    k.wtp = (float)c.r.wtp;
    k.wtm = (float)c.r.wtm;
    k.sp = (float)c.r.sp;
    k.sm = (float)c.r.sm;
    k.kcu = (float)(1.0 / (c.cs2 * c.cfl));
    k.hinvcs2 = (float)(0.5 / c.cs2);
    k.inv_cfl = (float)(1.0 / c.cfl);
    k.half_dt = (float)(0.5 * c.dt);
    k.dt = (float)c.dt;
    k.gF = (float)(1.0 / (c.cfl * c.cs2));
    k.inv_cs2 = (float)(1.0 / c.cs2);
    k.rho0 = (float)c.rho0;
    k.c0 = (float)c.c0;
    k.mob_p = (float)c.mob_p;
    k.mob_n = (float)c.mob_n;
    k.ms = (float)c.r.ms;
    k.md = (float)c.r.md;
    k.cfl_hdt = (float)(c.cfl * 0.5 * c.dt);
    k.srcF = (float)(c.r.sm * c.cfl * c.dt);
    k.f_chargef = (float)c.f_charge;
    k.ext_xf = (float)c.ext_x;
    k.exff = (float)c.exf;
    k.half_inv_dxf = (float)(0.5 / c.dx);
    k.half_inv_dyf = (float)(0.5 / c.dy);
    k.rhs_qf = (float)(-c.f_charge / c.eps);
    k.f_charge = c.f_charge;
    k.eps = c.eps;
    k.ext_x = c.ext_x;
    k.exf = c.exf;
    k.dx = c.dx;
    k.dy = c.dy;
    k.half_inv_dx = 0.5 / c.dx;
    k.half_inv_dy = 0.5 / c.dy;
    k.zlo = c.zlo;
    k.zhi = c.zhi;
    k.cplo = c.cplo;
    k.cphi = c.cphi;
    k.cnlo = c.cnlo;
    k.cnhi = c.cnhi;
    k.kref = c.kref;
    k.rhsf = c.rhsf;
    k.psif = c.psif;
    k.psim = c.psim;
    k.lift = c.lift;
    k.kwall = c.kwall;
    k.wdelta = c.wdelta;
    k.keep_l2 = c.keep_l2;
    return k;
}

namespace {

constexpr int TPB = 128;
// Blocks per SM the register allocation must allow.  Unconstrained the node
// update takes 108 registers (4 blocks of 4 warps per SM); at 7 blocks (72
// registers, no spills) the kernel hides more of the HBM latency: 0.169 ms
// against 0.219 ms per launch on 4096x1024 FP32 (B200; 6 blocks 0.183, 8
// blocks with 16-byte spills 0.181).
#ifndef EK_LBM_MIN_BLOCKS
#define EK_LBM_MIN_BLOCKS 7
#endif

// I: the index type of the node update (uint32_t when every offset into the
// population and field planes fits 32 bits, see own9s).
template <typename S, bool FIRST, bool EE, typename I>
__global__ void __launch_bounds__(TPB, EK_LBM_MIN_BLOCKS)
step_shifted(const ChanF k, const S *__restrict__ src, S *__restrict__ dst, double *__restrict__ fields, bool mom,
             int sbuf) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    if (x >= k.nx) return;
    node_shifted<S, FIRST, EE, I>(k, src, dst, fields, x, blockIdx.y, mom, sbuf);
}

template <typename S>
__global__ void __launch_bounds__(TPB)
init_shifted(const ChanF k, S *__restrict__ pops, const double *__restrict__ fields, bool explicit_e, int buf) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    if (x >= k.nx) return;
    init_node_shifted<S>(k, pops, fields, explicit_e, x, blockIdx.y, buf);
}

__global__ void __launch_bounds__(256) wall_frames(const ChanF k, const double *__restrict__ fields, int qp, int qn,
                                                   int buf, float *__restrict__ kwall, float *__restrict__ wdelta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4 * k.nx) wall_frames_dev(k, fields, qp, qn, buf, kwall, wdelta, i);
}

__global__ void __launch_bounds__(256) wall_delta(const ChanF k, const float *__restrict__ kwall,
                                                  float *__restrict__ wdelta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4 * k.nx) wall_delta_dev(k, kwall, wdelta, i);
}

template <typename S, typename I>
cudaError_t step_indexed(const ChanF &k, const void *src, void *dst, double *fields, bool first, bool ee,
                         bool mom, int sbuf, cudaStream_t s) {
    const dim3 g((k.nx + TPB - 1) / TPB, k.ny);
    const S *a = (const S *)src;
    S *b = (S *)dst;
    if (first) {
        if (ee) step_shifted<S, true, true, I><<<g, TPB, 0, s>>>(k, a, b, fields, mom, sbuf);
        else step_shifted<S, true, false, I><<<g, TPB, 0, s>>>(k, a, b, fields, mom, sbuf);
    } else {
        if (ee) step_shifted<S, false, true, I><<<g, TPB, 0, s>>>(k, a, b, fields, mom, sbuf);
        else step_shifted<S, false, false, I><<<g, TPB, 0, s>>>(k, a, b, fields, mom, sbuf);
    }
    return cudaGetLastError();
}

template <typename S>
cudaError_t step_typed(const ChanF &k, const void *src, void *dst, double *fields, bool first, bool ee,
                       bool mom, int sbuf, cudaStream_t s) {
    if (index32_fits(k.plane)) return step_indexed<S, uint32_t>(k, src, dst, fields, first, ee, mom, sbuf, s);
    return step_indexed<S, size_t>(k, src, dst, fields, first, ee, mom, sbuf, s);
}

__global__ void __launch_bounds__(256) row_refs(const Chan c, const double *__restrict__ fields, int qf, int qp,
                                                int qn, float *__restrict__ kout) {
    row_refs_dev(c.nx, c.nxp, c.ny, c.plane, fields, qf, qp, qn, kout, blockIdx.x);
}

template <typename S>
__global__ void __launch_bounds__(TPB) rebase_pops(const Chan c, S *__restrict__ pops, const float *__restrict__ kold,
                                                   const float *__restrict__ knew) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y, plane = blockIdx.z;
    if (x >= c.nx) return;
    rebase_dev<S>(pops + (size_t)plane * c.plane + (size_t)y * c.nxp + x, plane, c.ny, y, kold, knew);
}

// psim[y] = the row's FP64 mean of psi, psif = psi - psim in FP32; a block
// of 256 threads per row.
__global__ void __launch_bounds__(256) split_psi(const PoissonPlan pp, const Chan c, const double *__restrict__ psi) {
    const int y = blockIdx.x;
    const double *r = psi + (size_t)y * c.nxp;
    double acc = 0.0;
    for (int x = threadIdx.x; x < c.nx; x += 256) acc += r[x];
    __shared__ double red[8];
    __shared__ double mean;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[w];
        mean = v / (double)c.nx;
        pp.psim[y] = mean;
    }
    __syncthreads();
    float *f = pp.psif + (size_t)y * c.nxp;
    for (int x = threadIdx.x; x < c.nx; x += 256) f[x] = (float)(r[x] - mean);
}

// The FP64 right-hand side of the interior rows from rhsf: the row constant
// rhs_q (R+ - R-) and the wall lifting added back (the FP64 passes' input).
__global__ void __launch_bounds__(TPB) compose_rhs(const PoissonPlan pp, const Chan c, double *__restrict__ rhs) {
    const int x = blockIdx.x * TPB + threadIdx.x, y = blockIdx.y + 1;
    if (x >= c.nx) return;
    const size_t o = (size_t)y * c.nxp + x;
    rhs[o] = (double)pp.rhsf[o] + rhs_row_constant(pp, c, y);
}

// rhsf of the interior rows from the c+, c- moments (a solve outside the step).
__global__ void __launch_bounds__(TPB) rhsf_from_moments(const PoissonPlan pp, const Chan c,
                                                         const double *__restrict__ fields) {
    const int x = blockIdx.x * TPB + threadIdx.x, y = blockIdx.y + 1;
    if (x >= c.nx) return;
    const size_t o = (size_t)y * c.nxp + x;
    const double rq = -c.f_charge / c.eps;
    const double q = fields[F_CP * c.plane + o] - fields[F_CN * c.plane + o];
    double v = rq * (q - (36.0 * (double)c.kref[c.ny + y] - 36.0 * (double)c.kref[2 * c.ny + y]));
    if (y == 1) v -= c.lift[x];
    if (y == c.ny - 2) v -= c.lift[c.nx + x];
    pp.rhsf[o] = (float)v;
}

}  // namespace

cudaError_t launch_split_psi(const PoissonPlan &pp, const Chan &c, const double *psi, cudaStream_t s) {
    split_psi<<<c.ny, 256, 0, s>>>(pp, c, psi);
    return cudaGetLastError();
}

cudaError_t launch_compose_rhs(const PoissonPlan &pp, const Chan &c, double *rhs, cudaStream_t s) {
    compose_rhs<<<dim3((c.nx + TPB - 1) / TPB, c.ny - 2), TPB, 0, s>>>(pp, c, rhs);
    return cudaGetLastError();
}

cudaError_t launch_rhsf_from_moments(const PoissonPlan &pp, const Chan &c, const double *fields, cudaStream_t s) {
    rhsf_from_moments<<<dim3((c.nx + TPB - 1) / TPB, c.ny - 2), TPB, 0, s>>>(pp, c, fields);
    return cudaGetLastError();
}

cudaError_t launch_row_refs(const Chan &c, const double *fields, int qf, int qp, int qn, float *kout,
                            cudaStream_t s) {
    row_refs<<<c.ny, 256, 0, s>>>(c, fields, qf, qp, qn, kout);
    return cudaGetLastError();
}

cudaError_t launch_rebase(const Chan &c, int storage, void *pops, const float *kold, const float *knew,
                          cudaStream_t s) {
    const dim3 g((c.nx + TPB - 1) / TPB, c.ny, 27);
    if (storage == EK_STORE_F16) rebase_pops<__half><<<g, TPB, 0, s>>>(c, (__half *)pops, kold, knew);
    else rebase_pops<float><<<g, TPB, 0, s>>>(c, (float *)pops, kold, knew);
    return cudaGetLastError();
}

cudaError_t launch_step_shifted(const Chan &c, int storage, const void *src, void *dst, double *fields,
                                bool first, bool explicit_e, bool moments, int sbuf, cudaStream_t s) {
    const ChanF k = make_chanf(c);
    if (storage == EK_STORE_F16) return step_typed<__half>(k, src, dst, fields, first, explicit_e, moments, sbuf, s);
    return step_typed<float>(k, src, dst, fields, first, explicit_e, moments, sbuf, s);
}

cudaError_t launch_init_shifted(const Chan &c, int storage, void *pops, const double *fields, bool explicit_e,
                                int buf, cudaStream_t s) {
    const ChanF k = make_chanf(c);
    const dim3 g((k.nx + TPB - 1) / TPB, k.ny);
    if (storage == EK_STORE_F16) init_shifted<__half><<<g, TPB, 0, s>>>(k, (__half *)pops, fields, explicit_e, buf);
    else init_shifted<float><<<g, TPB, 0, s>>>(k, (float *)pops, fields, explicit_e, buf);
    return cudaGetLastError();
}

cudaError_t launch_wall_frames(const Chan &c, const double *fields, int qp, int qn, int buf, float *kwall,
                               float *wdelta, cudaStream_t s) {
    const ChanF k = make_chanf(c);
    wall_frames<<<(4 * c.nx + 255) / 256, 256, 0, s>>>(k, fields, qp, qn, buf, kwall, wdelta);
    return cudaGetLastError();
}

cudaError_t launch_wall_delta(const Chan &c, const float *kwall, float *wdelta, cudaStream_t s) {
    const ChanF k = make_chanf(c);
    wall_delta<<<(4 * c.nx + 255) / 256, 256, 0, s>>>(k, kwall, wdelta);
    return cudaGetLastError();
}

}  // namespace ek
