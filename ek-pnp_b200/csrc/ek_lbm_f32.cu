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
    k.f_charge = c.f_charge;
    k.eps = c.eps;
    k.ext_x = c.ext_x;
    k.exf = c.exf;
    k.dx = c.dx;
    k.dy = c.dy;
    k.zlo = c.zlo;
    k.zhi = c.zhi;
    k.cplo = c.cplo;
    k.cphi = c.cphi;
    k.cnlo = c.cnlo;
    k.cnhi = c.cnhi;
    return k;
}

namespace {

constexpr int TPB = 128;

template <typename S, bool FIRST, bool EE, bool MOM>
__global__ void __launch_bounds__(TPB)
step_shifted(const ChanF k, const S *__restrict__ src, S *__restrict__ dst, double *__restrict__ fields) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    if (x >= k.nx) return;
    node_shifted<S, FIRST, EE, MOM>(k, src, dst, fields, x, blockIdx.y);
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
#define EK_SS(F, E, M) step_shifted<S, F, E, M><<<g, TPB, 0, s>>>(k, a, b, fields)
    switch ((first ? 4 : 0) | (ee ? 2 : 0) | (mom ? 1 : 0)) {
        case 0: EK_SS(false, false, false); break;
        case 1: EK_SS(false, false, true); break;
        case 2: EK_SS(false, true, false); break;
        case 3: EK_SS(false, true, true); break;
        case 4: EK_SS(true, false, false); break;
        case 5: EK_SS(true, false, true); break;
        case 6: EK_SS(true, true, false); break;
        default: EK_SS(true, true, true); break;
    }
#undef EK_SS
    return cudaGetLastError();
}

}  // namespace

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
