// ek_residual.cu -- steady-state residual reduction in FP64 (new; the
// reference has none).  For q in (ux, c+, c-, psi) it sums (q - q_snap)^2 and
// q^2 over all nodes, and stores q as the next snapshot, in one pass.  The
// reduction is deterministic: fixed grid, warp shuffles, one partial per block
// and a single-block final sum in block order.
#include <cuda_runtime.h>

#include "ek_internal.h"

namespace ek {
namespace {

constexpr int RTPB = 256;
__device__ __forceinline__ int qfield(int q) { return q == 0 ? F_UX : (q == 1 ? F_CP : (q == 2 ? F_CN : F_PSI)); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// Partial sums of block `blk` of `nblocks` over one channel's nodes.
__device__ __forceinline__ void residual_partials_dev(const Chan &c, const double *__restrict__ fields,
                                                      double *__restrict__ snap, double *__restrict__ part, int blk,
                                                      int nblocks) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long long nn = (long long)c.nx * c.ny;
    for (long long i = (long long)blk * RTPB + threadIdx.x; i < nn; i += (long long)nblocks * RTPB) {
        const int y = (int)(i / c.nx), x = (int)(i - (long long)y * c.nx);
        const size_t o = (size_t)y * c.nxp + x;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double v = fields[qfield(q) * c.plane + o];
            const double d = v - snap[q * c.plane + o];
            acc[q] += d * d;
            acc[4 + q] += v * v;
            snap[q * c.plane + o] = v;
        }
    }
    __shared__ double red[RTPB / 32][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double s = warp_sum(acc[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int w = 0; w < RTPB / 32; ++w) s += red[w][threadIdx.x];
        part[(size_t)blk * 8 + threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(RTPB)
residual_partials(const Chan c, const double *__restrict__ fields, double *__restrict__ snap,
                  double *__restrict__ part) {
    residual_partials_dev(c, fields, snap, part, blockIdx.x, gridDim.x);
}

// Many channels: item {channel, block, blocks of the channel, first partial}.
__global__ void __launch_bounds__(RTPB)
batch_residual_partials(const Chan *__restrict__ chans, double *const *__restrict__ fields,
                        double *const *__restrict__ snaps, const int4 *__restrict__ items, double *__restrict__ part) {
    const int4 it = items[blockIdx.x];
    residual_partials_dev(chans[it.x], fields[it.x], snaps[it.x], part + (size_t)it.w * 8, it.y, it.z);
}

// One warp per channel: lanes 0..7 sum their column of the channel's
// partials in block order (the order of residual_final).
__global__ void batch_residual_final(const int2 *__restrict__ ranges, int nch, const double *__restrict__ part,
                                     double *__restrict__ out8) {
    const int ch = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (ch >= nch || lane >= 8) return;
    const int2 r = ranges[ch];  // {first partial, blocks}
    double s = 0.0;
    for (int b = 0; b < r.y; ++b) s += part[(size_t)(r.x + b) * 8 + lane];
    out8[(size_t)ch * 8 + lane] = s;
}

__global__ void residual_final(const double *__restrict__ part, int nblocks, double *__restrict__ out8) {
    // thread k sums column k in block order: deterministic
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * 8 + threadIdx.x];
        out8[threadIdx.x] = s;
    }
}

}  // namespace

int residual_blocks(const Chan &c) {
    const long long nn = (long long)c.nx * c.ny;
    long long b = (nn + RTPB - 1) / RTPB;
    return (int)(b < 148 * 4 ? b : 148 * 4);
}

cudaError_t launch_residual_f64(const Chan &c, const double *fields, double *snap, double *part,
                                int nblocks, double *out8, cudaStream_t s) {
    residual_partials<<<nblocks, RTPB, 0, s>>>(c, fields, snap, part);
    residual_final<<<1, 32, 0, s>>>(part, nblocks, out8);
    return cudaGetLastError();
}

cudaError_t launch_batch_residual(const Chan *chans, double *const *fields, double *const *snaps, const int4 *items,
                                  int nitems, const int2 *ranges, int nch, double *part, double *out8,
                                  cudaStream_t s) {
    batch_residual_partials<<<nitems, RTPB, 0, s>>>(chans, fields, snaps, items, part);
    batch_residual_final<<<(nch + 7) / 8, 256, 0, s>>>(ranges, nch, part, out8);
    return cudaGetLastError();
}

}  // namespace ek
