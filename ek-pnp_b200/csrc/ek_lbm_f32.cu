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
    k.wpd = c.r.wp;
    k.wmd = c.r.wm;
    k.spd = c.r.sp;
    k.smd = c.r.sm;
    k.kcud = 1.0 / (c.cs2 * c.cfl);
    k.hinvcs2d = 0.5 / c.cs2;
    k.gFd = 1.0 / (c.cfl * c.cs2);
    k.inv_cs2d = 1.0 / c.cs2;
    k.dtd = c.dt;
    k.f_charge = c.f_charge;
    k.eps = c.eps;
    k.ext_x = c.ext_x;
    k.exf = c.exf;
    k.dx = c.dx;
    k.dy = c.dy;
    k.wcpd = c.r.wcp;
    k.wcmd = c.r.wcm;
    k.wtpd = c.r.wtp;
    k.wtmd = c.r.wtm;
    k.mob_pd = c.mob_p;
    k.mob_nd = c.mob_n;
    k.half_inv_dx = 0.5 / c.dx;
    k.half_inv_dy = 0.5 / c.dy;
    k.rhs_q = -c.f_charge / c.eps;
    k.inv_dy2 = 1.0 / (c.dy * c.dy);
    k.zlo = c.zlo;
    k.zhi = c.zhi;
    k.cplo = c.cplo;
    k.cphi = c.cphi;
    k.cnlo = c.cnlo;
    k.cnhi = c.cnhi;
    k.kref = c.kref;
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

template <typename S, bool FIRST, bool EE>
__global__ void __launch_bounds__(TPB, EK_LBM_MIN_BLOCKS)
step_shifted(const ChanF k, const S *__restrict__ src, S *__restrict__ dst, double *__restrict__ fields, bool mom) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    if (x >= k.nx) return;
    node_shifted<S, FIRST, EE>(k, src, dst, fields, x, blockIdx.y, mom);
}

template <typename S>
__global__ void __launch_bounds__(TPB)
init_shifted(const ChanF k, S *__restrict__ pops, const double *__restrict__ fields, bool explicit_e) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    if (x >= k.nx) return;
    init_node_shifted<S>(k, pops, fields, explicit_e, x, blockIdx.y);
}

template <typename S>
cudaError_t step_typed(const ChanF &k, const void *src, void *dst, double *fields, bool first, bool ee,
                       bool mom, cudaStream_t s) {
    const dim3 g((k.nx + TPB - 1) / TPB, k.ny);
    const S *a = (const S *)src;
    S *b = (S *)dst;
    if (first) {
        if (ee) step_shifted<S, true, true><<<g, TPB, 0, s>>>(k, a, b, fields, mom);
        else step_shifted<S, true, false><<<g, TPB, 0, s>>>(k, a, b, fields, mom);
    } else {
        if (ee) step_shifted<S, false, true><<<g, TPB, 0, s>>>(k, a, b, fields, mom);
        else step_shifted<S, false, false><<<g, TPB, 0, s>>>(k, a, b, fields, mom);
    }
    return cudaGetLastError();
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

}  // namespace

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
                                bool first, bool explicit_e, bool moments, cudaStream_t s) {
    const ChanF k = make_chanf(c);
    if (storage == EK_STORE_F16) return step_typed<__half>(k, src, dst, fields, first, explicit_e, moments, s);
    return step_typed<float>(k, src, dst, fields, first, explicit_e, moments, s);
}

cudaError_t launch_init_shifted(const Chan &c, int storage, void *pops, const double *fields, bool explicit_e,
                                cudaStream_t s) {
    const ChanF k = make_chanf(c);
    const dim3 g((k.nx + TPB - 1) / TPB, k.ny);
    if (storage == EK_STORE_F16) init_shifted<__half><<<g, TPB, 0, s>>>(k, (__half *)pops, fields, explicit_e);
    else init_shifted<float><<<g, TPB, 0, s>>>(k, (float *)pops, fields, explicit_e);
    return cudaGetLastError();
}

}  // namespace ek
