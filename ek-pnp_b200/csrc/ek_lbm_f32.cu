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
    k.zlo = c.zlo;
    k.zhi = c.zhi;
    k.cplo = c.cplo;
    k.cphi = c.cphi;
    k.cnlo = c.cnlo;
    k.cnhi = c.cnhi;
    k.kref = c.kref;
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

// Row means of rho, c+, c- rounded to the reference grid K 2^-q (stored /36):
// one block per row, FP64 sums.
__global__ void __launch_bounds__(256) row_refs(const Chan c, const double *__restrict__ fields, int qf, int qp,
                                                int qn, float *__restrict__ kout) {
    const int y = blockIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    const size_t r = (size_t)y * c.nxp;
    for (int x = threadIdx.x; x < c.nx; x += blockDim.x) {
        acc[0] += fields[F_RHO * c.plane + r + x];
        acc[1] += fields[F_CP * c.plane + r + x];
        acc[2] += fields[F_CN * c.plane + r + x];
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
        const double mean = v / (double)c.nx;
        const double K = rint(mean / 36.0 * ldexp(1.0, q));
        kout[threadIdx.x * c.ny + y] = (float)ldexp(K, -q);
    }
}

// d += 36 w_d (kold - knew) for every stored value (exact in FP32).
template <typename S>
__global__ void __launch_bounds__(TPB) rebase_pops(const Chan c, S *__restrict__ pops, const float *__restrict__ kold,
                                                   const float *__restrict__ knew) {
    const int x = blockIdx.x * TPB + threadIdx.x;
    const int y = blockIdx.y, plane = blockIdx.z;
    if (x >= c.nx) return;
    const int s = plane / 9, d = plane - 9 * s;
    const float wint = d == 0 ? 16.0f : (d < 5 ? 4.0f : 1.0f);
    const float corr = wint * (kold[s * c.ny + y] - knew[s * c.ny + y]);
    S *p = pops + (size_t)plane * c.plane + (size_t)y * c.nxp + x;
    st_pop<S>(p, ld_pop<S>(p) + corr);
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
