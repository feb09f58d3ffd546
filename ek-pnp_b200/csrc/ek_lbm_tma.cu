// ek_lbm_tma.cu -- TMA-fed persistent form of the shifted-storage step.
//
// The plain kernel (ek_lbm_f32.cu) pulls its 27 populations with ordinary
// loads, so the bytes in flight are bounded by the registers of the resident
// warps.  Here a producer warp streams the data into shared memory with the
// tensor-memory accelerator while four compute warps work on earlier tiles:
//
//   tile      one row y, TX = 128 consecutive columns x0 .. x0+127
//   stage     27 boxes, one per population plane, each 1 row x (TX + 2 HALO)
//             elements starting at x0 - HALO (HALO = 16 bytes, so every TMA
//             x coordinate is 16-byte aligned).  The row of a box is the row
//             the plane's direction streams from (y - c_y, periodic), or y for
//             values read in place (first step after initialisation, ion
//             populations of wall rows).
//   ring      NSTAGE stages; "full" mbarriers complete on the TMA byte count,
//             "empty" mbarriers collect the 128 consumers' releases.
//
// The consumers gather their populations from shared memory (the halo gives
// the x-1/x+1 neighbours), release the stage, and run the same collision as
// the plain kernel (collide_shifted), so both forms give bit-identical
// results.  The two wrap columns of a channel (x = 0 pulling from nx-1 and
// nx-1 pulling from 0) and the lower wall's row-1 pull read global memory.
// Every mbarrier wait of the pipeline gives up after a bound (by default about
// 2^31 clock cycles, ~1 s; EK_OPT_WAIT_CYCLES), sets the context's error word
// and leaves the loop; the producer then waits, at the default bound, for the
// copies it issued before the block exits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include "ek_lbm_f32.cuh"

namespace ek {
namespace {

constexpr int TX = 128;
constexpr int NCONS = TX;
constexpr int NTHREADS = NCONS + 32;
constexpr int NSTAGE = 4;
constexpr long long WAIT_CYCLES = 1LL << 31;

template <typename S> struct Geom {
    static constexpr int HALO = 16 / (int)sizeof(S);
    static constexpr int BOXW = TX + 2 * HALO;
    static constexpr int BOX_BYTES = BOXW * (int)sizeof(S);
    static constexpr int PLANE_BYTES = (BOX_BYTES + 127) / 128 * 128;
    static constexpr int STAGE_BYTES = 27 * PLANE_BYTES;
    static constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 2 * NSTAGE * 8;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of parity `parity` to complete, at most `limit` cycles.
__device__ __noinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, long long limit) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            atomicOr(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <typename S> __device__ __forceinline__ float ld_smem(const S *p);
template <> __device__ __forceinline__ float ld_smem<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ld_smem<__half>(const __half *p) { return __half2float(*p); }

template <typename S, bool FIRST, bool EE>
__global__ void __launch_bounds__(NTHREADS)
step_tma(const __grid_constant__ CUtensorMap tsrc, const ChanF k, const S *__restrict__ src, S *__restrict__ dst,
         double *__restrict__ fields, int *__restrict__ err, bool mom, long long wait_cycles, int sbuf) {
    using G = Geom<S>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = (uint64_t *)(smem + NSTAGE * G::STAGE_BYTES);
    uint64_t *empty = full + NSTAGE;
    const int tid = threadIdx.x;
    const int tiles_x = (k.nx + TX - 1) / TX;
    const int ntiles = tiles_x * k.ny;
    if (tid == 0) {
        for (int i = 0; i < NSTAGE; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], NCONS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid >= NCONS) {  // producer warp: one lane issues the copies
        if (tid != NCONS) return;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int stage = it % NSTAGE;
            const uint32_t ph = (uint32_t)(it / NSTAGE) & 1u;
            if (it >= NSTAGE && !mbar_wait(&empty[stage], ph ^ 1u, err, wait_cycles)) break;
            const int y = tile / tiles_x, x0 = (tile - y * tiles_x) * TX;
            const bool wall = y == 0 || y == k.ny - 1;
            const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
            unsigned char *base = smem + stage * G::STAGE_BYTES;
            mbar_arrive_expect_tx(&full[stage], 27u * G::BOX_BYTES);
#pragma unroll 1
            for (int plane = 0; plane < 27; ++plane) {
                const int d = plane % 9;
                const bool own = FIRST || (wall && plane >= 9);
                const int row = own ? y : (cyd(d) > 0 ? ym : (cyd(d) < 0 ? yp : y));
                tma_load_3d(base + plane * G::PLANE_BYTES, &tsrc, x0 - G::HALO, row, plane, &full[stage]);
            }
        }
        // copies still in flight must land before the block exits: waited
        // for at the default bound whatever the pipeline's bound is
        for (int j = it > NSTAGE ? it - NSTAGE : 0; j < it; ++j)
            mbar_wait(&full[j % NSTAGE], (uint32_t)(j / NSTAGE) & 1u, err, WAIT_CYCLES);
        return;
    }

    const size_t pl = k.plane;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int stage = it % NSTAGE;
        const uint32_t ph = (uint32_t)(it / NSTAGE) & 1u;
        if (!mbar_wait(&full[stage], ph, err, wait_cycles)) break;
        const int y = tile / tiles_x, x0 = (tile - y * tiles_x) * TX;
        const int x = x0 + tid;
        const bool wall = y == 0 || y == k.ny - 1;
        const unsigned char *base = smem + stage * G::STAGE_BYTES;
        float v[27];
#pragma unroll
        for (int plane = 0; plane < 27; ++plane) {
            const int d = plane % 9;
            const bool own = FIRST || (wall && plane >= 9);
            const int col = G::HALO + tid - (own ? 0 : cxd(d));
            v[plane] = ld_smem<S>((const S *)(base + plane * G::PLANE_BYTES) + col);
        }
        mbar_arrive(&empty[stage]);
        if (x < k.nx) {
            if (!FIRST && (x == 0 || x == k.nx - 1)) {
                // periodic wrap in x: the halo column holds fill values there
                const int ym = y == 0 ? k.ny - 1 : y - 1, yp = y + 1 == k.ny ? 0 : y + 1;
                const int xs = x == 0 ? k.nx - 1 : 0;
                const int want = x == 0 ? 1 : -1;
#pragma unroll
                for (int plane = 0; plane < 27; ++plane) {
                    const int d = plane % 9;
                    if (cxd(d) != want || (wall && plane >= 9)) continue;
                    const int row = cyd(d) > 0 ? ym : (cyd(d) < 0 ? yp : y);
                    v[plane] = ld_pop<S>(src + plane * pl + (size_t)row * k.nxp + xs);
                }
            }
            collide_shifted<S, FIRST, EE>(k, v, v + 9, v + 18, src, dst, fields, x, y, mom, sbuf);
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

template <typename S>
cudaError_t launch_typed(const CUtensorMap &map, const ChanF &k, const void *src, void *dst, double *fields,
                         bool first, bool ee, bool mom, int sbuf, int *err, long long wait_cycles, int grid,
                         cudaStream_t s) {
    const S *a = (const S *)src;
    S *b = (S *)dst;
    const int smem = Geom<S>::SMEM_BYTES;
#define EK_TMA(F, E) \
    step_tma<S, F, E><<<grid, NTHREADS, smem, s>>>(map, k, a, b, fields, err, mom, wait_cycles, sbuf)
    if (first) {
        if (ee) EK_TMA(true, true);
        else EK_TMA(true, false);
    } else {
        if (ee) EK_TMA(false, true);
        else EK_TMA(false, false);
    }
#undef EK_TMA
    return cudaGetLastError();
}

template <typename S> cudaError_t set_attrs() {
    const void *fns[] = {
        (const void *)step_tma<S, false, false>, (const void *)step_tma<S, false, true>,
        (const void *)step_tma<S, true, false>, (const void *)step_tma<S, true, true>};
    for (const void *f : fns) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, Geom<S>::SMEM_BYTES);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

// Tensor map over one population buffer: dims (nxp, ny, 27), box (TX+2 HALO, 1, 1).
cudaError_t make_pop_tensor_map(int storage, const void *pops, int nxp, int ny, void *map_out) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const bool half = storage == EK_STORE_F16;
    const cuuint64_t es = half ? 2 : 4;
    const cuuint64_t dims[3] = {(cuuint64_t)nxp, (cuuint64_t)ny, 27};
    const cuuint64_t strides[2] = {(cuuint64_t)nxp * es, (cuuint64_t)nxp * ny * es};
    const cuuint32_t box[3] = {(cuuint32_t)(half ? Geom<__half>::BOXW : Geom<float>::BOXW), 1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn((CUtensorMap *)map_out, half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                    const_cast<void *>(pops), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_step_tma(const Chan &c, int storage, const void *map, const void *src, void *dst, double *fields,
                            bool first, bool explicit_e, bool moments, int sbuf, int *err, long long wait_cycles,
                            cudaStream_t s) {
    static bool attrs = false;
    if (!attrs) {
        cudaError_t e = set_attrs<float>();
        if (e == cudaSuccess) e = set_attrs<__half>();
        if (e != cudaSuccess) return e;
        attrs = true;
    }
    const ChanF k = make_chanf(c);
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const bool half = storage == EK_STORE_F16;
    cudaError_t e = half ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step_tma<__half, false, false>,
                                                                       NTHREADS, Geom<__half>::SMEM_BYTES)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step_tma<float, false, false>,
                                                                       NTHREADS, Geom<float>::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    const int ntiles = ((c.nx + TX - 1) / TX) * c.ny;
    int grid = sms * (per > 0 ? per : 1);
    if (grid > ntiles) grid = ntiles;
    const CUtensorMap &m = *(const CUtensorMap *)map;
    return half ? launch_typed<__half>(m, k, src, dst, fields, first, explicit_e, moments, sbuf, err, wait_cycles,
                                       grid, s)
                : launch_typed<float>(m, k, src, dst, fields, first, explicit_e, moments, sbuf, err, wait_cycles,
                                      grid, s);
}

}  // namespace ek
