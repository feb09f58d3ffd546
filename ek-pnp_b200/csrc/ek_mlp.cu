// ek_mlp.cu -- the learned warm start (new; the reference has none): a
// 4 -> 256 -> 256 -> 256 -> 512 MLP with SiLU, trained and evaluated on the
// GPU by hand-written kernels.
//
//   GEMMs      C = A B^T on the 5th-generation tensor cores: BF16 operands
//              copied asynchronously into a 4-slot ring of shared-memory
//              stages (K-major, no swizzle), tcgen05.mma issued by one thread
//              into an FP32 accumulator in tensor memory as each K chunk
//              lands, completion through tcgen05.commit on each slot's
//              mbarrier (bounded waits), tcgen05.ld into registers for a fused
//              epilogue (bias, SiLU, SiLU derivative, BF16 and transposed
//              BF16 stores).
//   training   per iteration: batch gather, 4 forward GEMMs, MSE loss and its
//              gradient, 3 backward-data and 4 weight-gradient GEMMs, bias
//              gradients, Adam on FP32 master weights, BF16 weight casts --
//              16 launches, captured once in a CUDA graph and replayed.
// Weights are used in BF16 with FP32 accumulation; the FP32 master copy, the
// Adam moments and the gradients live in one flat buffer laid out per layer
// as W (out x in, row-major, layer-0 inputs padded from 4 to 16) then b.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "ek_ctx.h"
#include "ek_tc.cuh"

using bf16 = __nv_bfloat16;

namespace {

constexpr int TM = 128;  // rows of a CTA tile (the MMA's M)
constexpr int KC = 64;   // K elements staged per round
constexpr int NT_MAX = 128;
constexpr int NL = 4;
constexpr int IN = 4, INP = 16, HID = 256, OUT = 512;
constexpr int DIM_IN[NL] = {INP, HID, HID, HID};
constexpr int DIM_OUT[NL] = {HID, HID, HID, OUT};

enum Epi { EPI_F32 = 0, EPI_FWD_HIDDEN = 1, EPI_FWD_OUT = 2, EPI_BWD_HIDDEN = 3 };

struct GemmArgs {
    const bf16 *a;  // M x K, row stride lda
    const bf16 *b;  // N x K, row stride ldb
    int lda, ldb, m, n, k, nt;
    float *c;       // EPI_F32 / EPI_FWD_OUT: M x N fp32, row stride ldc
    int ldc;
    const float *bias;
    float *z;       // EPI_FWD_HIDDEN: pre-activations out; EPI_BWD_HIDDEN: pre-activations in
    int ldz;
    bf16 *h;        // BF16 result, row stride ldh
    int ldh;
    bf16 *ht;       // BF16 transposed result, row stride ldht
    int ldht;
    int *err;
    long long wait_cycles;  // bound of each wait for the MMAs of a K chunk
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// One 128 x nt tile of C = A B^T per CTA of 128 threads.
//
// K is cut into chunks of KC; chunk c is staged in ring slot c % STAGES
// (A: TM x KC, B: nt x KC, BF16, the canonical K-major layout).  The copies
// are 16-byte asynchronous copies (cp.async.cg, global -> shared) issued by
// all threads, one commit group per chunk: the first STAGES chunks are all
// in flight before the first MMA, and a slot is refilled as soon as the MMAs
// that read it have completed, so loads of later chunks overlap the MMAs of
// earlier ones.  One thread issues each chunk's tcgen05.mma instructions and
// commits them to the slot's mbarrier; every slot has at most one
// uncompleted commit at a time, so a wait by parity is unambiguous.
constexpr int STAGES = 4;
constexpr size_t STAGE_A = (size_t)TM * KC * 2, STAGE_BYTES = STAGE_A + (size_t)NT_MAX * KC * 2;
constexpr size_t GEMM_SMEM = STAGES * STAGE_BYTES;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(ek::tc::smem_u32(smem)), "l"(gmem) : "memory");
}
// Wait until at most n of this thread's commit groups are pending (n < STAGES).
__device__ __forceinline__ void cp_async_wait_pending(int n) {
    switch (n) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    }
}

template <int EPI>
__global__ void __launch_bounds__(128) mlp_gemm(const GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t stage_mem[];
    __shared__ __align__(8) uint64_t bar[STAGES];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * g.nt;
    if (warp == 0) {
        ek::tc::tmem_alloc(&tmem_base, NT_MAX);
        ek::tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int b = 0; b < STAGES; ++b) ek::tc::mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    ek::tc::fence_before_sync();
    __syncthreads();
    ek::tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = ek::tc::idesc_bf16_f32(TM, g.nt);
    const int nk = (g.k + KC - 1) / KC;
    // copies of chunk c into its ring slot
    auto load = [&](int c) {
        uint8_t *sa = stage_mem + (size_t)(c % STAGES) * STAGE_BYTES, *sb = sa + STAGE_A;
        const int k0 = c * KC;
        const int vpr = min(KC, g.k - k0) >> 3;  // 16-byte vectors per row (kk a multiple of 16)
        for (int v = tid; v < TM * vpr; v += 128) {
            const int r = v / vpr, cc = v - r * vpr;
            cp_async16(sa + ((r >> 3) * (KC / 8) + cc) * 128 + (r & 7) * 16, g.a + (size_t)(m0 + r) * g.lda + k0 + cc * 8);
        }
        for (int v = tid; v < g.nt * vpr; v += 128) {
            const int r = v / vpr, cc = v - r * vpr;
            cp_async16(sb + ((r >> 3) * (KC / 8) + cc) * 128 + (r & 7) * 16, g.b + (size_t)(n0 + r) * g.ldb + k0 + cc * 8);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    uint32_t phase = 0;  // bit b: parity of slot b's next completion
    uint32_t open = 0;   // bit b: slot b has a commit not yet waited for
    const int pre = min(nk, STAGES);
    for (int c = 0; c < pre; ++c) load(c);
    bool failed = false;
    for (int i = 0; i < nk && !failed; ++i) {
        const int st = i % STAGES;
        cp_async_wait_pending(min(nk - 1 - i, STAGES - 1));  // chunk i's copies (this thread's) have landed
        ek::tc::fence_async_smem();                            // visible to the tensor cores
        __syncthreads();                                       // every thread's copies of chunk i
        if (tid == 0) {
            ek::tc::fence_after_sync();
            const uint32_t a0 = ek::tc::smem_u32(stage_mem + (size_t)st * STAGE_BYTES), b0 = a0 + (uint32_t)STAGE_A;
            const int kk = min(KC, g.k - i * KC);
            for (int kq = 0; kq < kk / 16; ++kq) {
                // 16 K-elements = two core matrices along K
                const uint64_t ad = ek::tc::smem_desc(a0 + kq * 256, 128, (KC / 8) * 128);
                const uint64_t bd = ek::tc::smem_desc(b0 + kq * 256, 128, (KC / 8) * 128);
                ek::tc::mma_bf16(tmem, ad, bd, idesc, (i > 0 || kq > 0) ? 1u : 0u);
            }
            ek::tc::mma_commit(&bar[st]);
        }
        open |= 1u << st;
        if (i + STAGES < nk) {
            // the slot is refilled once the MMAs that read it have completed
            const bool ok = ek::tc::mbar_wait_bounded(&bar[st], (phase >> st) & 1u, g.wait_cycles);
            failed = __syncthreads_or(!ok) != 0;
            if (!failed) {
                phase ^= 1u << st;
                open &= ~(1u << st);
                ek::tc::fence_after_sync();
                load(i + STAGES);
            }
        }
    }
    // the accumulator is complete once every open commit has arrived (the
    // last one tracks all MMAs issued before it); after a failed wait, MMAs
    // still in flight get one more wait at the default bound before the
    // tensor memory is freed
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    for (int b = 0; b < STAGES; ++b) {
        if (!((open >> b) & 1u)) continue;
        if (!failed && ek::tc::mbar_wait_bounded(&bar[b], (phase >> b) & 1u, g.wait_cycles)) continue;
        failed = true;
        ek::tc::mbar_wait_bounded(&bar[b], (phase >> b) & 1u, ek::tc::WAIT_CYCLES_DEFAULT);
    }
    failed = __syncthreads_or(failed) != 0;
    ek::tc::fence_after_sync();
    if (failed) {
        if (tid == 0) atomicOr(g.err, 1);
    } else {
        const int row = m0 + warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        for (int j = 0; j < g.nt; j += 8) {
            float v[8];
            ek::tc::tmem_ld8(trow + j, v);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int col = n0 + j + i;
                if (EPI == EPI_F32) {
                    g.c[(size_t)row * g.ldc + col] = v[i];
                } else if (EPI == EPI_FWD_OUT) {
                    g.c[(size_t)row * g.ldc + col] = v[i] + g.bias[col];
                } else if (EPI == EPI_FWD_HIDDEN) {
                    const float z = v[i] + g.bias[col];
                    g.z[(size_t)row * g.ldz + col] = z;
                    const bf16 h = __float2bfloat16_rn(silu(z));
                    g.h[(size_t)row * g.ldh + col] = h;
                    g.ht[(size_t)col * g.ldht + row] = h;
                } else {
                    const float dz = v[i] * silu_grad(g.z[(size_t)row * g.ldz + col]);
                    const bf16 d = __float2bfloat16_rn(dz);
                    g.h[(size_t)row * g.ldh + col] = d;
                    g.ht[(size_t)col * g.ldht + row] = d;
                }
            }
        }
    }
    ek::tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) ek::tc::tmem_dealloc(tmem, NT_MAX);
}

// Batch rows idx[offset .. offset+B) of the data set: X (padded to 16 inputs,
// BF16, and transposed), targets T (FP32).  offset = (*step - *base) * B, or 0.
__global__ void gather_batch(const float *__restrict__ xs, const float *__restrict__ ts, const int *__restrict__ idx,
                             const int64_t *__restrict__ step, const int64_t *__restrict__ base, int B,
                             bf16 *__restrict__ x, bf16 *__restrict__ xt, float *__restrict__ t) {
    const int64_t off = step ? (*step - *base) * B : 0;
    const int b = blockIdx.x;
    const int src = idx[off + b];
    for (int j = threadIdx.x; j < OUT; j += blockDim.x) t[(size_t)b * OUT + j] = ts[(size_t)src * OUT + j];
    if (threadIdx.x < INP) {
        const float v = threadIdx.x < IN ? xs[(size_t)src * IN + threadIdx.x] : 0.0f;
        const bf16 h = __float2bfloat16_rn(v);
        x[(size_t)b * INP + threadIdx.x] = h;
        xt[(size_t)threadIdx.x * B + b] = h;
    }
}

// MSE over B x 512 outputs: dY = 2 (Y - T) / (B 512) (BF16, and transposed);
// the loss of the iteration is added to loss[*step - *base].
__global__ void mse_grad(const float *__restrict__ y, const float *__restrict__ t, int B, bf16 *__restrict__ dy,
                         bf16 *__restrict__ dyt, double *__restrict__ loss, const int64_t *__restrict__ step,
                         const int64_t *__restrict__ base) {
    const int b = blockIdx.x;
    const float scale = 2.0f / ((float)B * (float)OUT);
    double acc = 0.0;
    for (int j = threadIdx.x; j < OUT; j += blockDim.x) {
        const float d = y[(size_t)b * OUT + j] - t[(size_t)b * OUT + j];
        acc += (double)d * (double)d;
        const bf16 g = __float2bfloat16_rn(scale * d);
        dy[(size_t)b * OUT + j] = g;
        dyt[(size_t)j * B + b] = g;
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        const int64_t slot = step ? (*step - *base) : 0;
        atomicAdd(loss + slot, s / ((double)B * OUT));
    }
}

struct BiasSeg {
    const bf16 *dzt[NL];  // (out x B) transposed deltas
    float *db[NL];
    int rows[NL];
};

// db[n] = sum over the batch of dZ[:, n]: one warp per output n.
__global__ void bias_grads(const BiasSeg s, int B) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int l = 0, n = w;
    while (l < NL && n >= s.rows[l]) n -= s.rows[l++];
    if (l >= NL) return;
    const bf16 *r = s.dzt[l] + (size_t)n * B;
    float acc = 0.0f;
    for (int b = lane; b < B; b += 32) acc += __bfloat162float(r[b]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) s.db[l][n] = acc;
}

// Adam on the flat FP32 parameters; step count t = *step + 1.
__global__ void adam_update(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                            const int64_t *__restrict__ step) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t = (double)(*step + 1);
    const float c1 = (float)(1.0 - pow((double)b1, t)), c2 = (float)(1.0 - pow((double)b2, t));
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct CastSeg {
    const float *w[NL];
    bf16 *wb[NL];
    bf16 *wt[NL];
    int out[NL], in[NL];
};

// BF16 copies W (out x in) and W^T (in x out) of every layer; the last thread
// advances the step counter (after Adam, before the next gather).
__global__ void cast_weights(const CastSeg s, int64_t *__restrict__ step, int total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && step) ++*step;
    if (i >= total) return;
    int l = 0, e = i;
    while (l < NL && e >= s.out[l] * s.in[l]) e -= s.out[l] * s.in[l], ++l;
    if (l >= NL) return;
    const int o = e / s.in[l], c = e - o * s.in[l];
    const bf16 h = __float2bfloat16_rn(s.w[l][e]);
    s.wb[l][e] = h;
    s.wt[l][(size_t)c * s.out[l] + o] = h;
}

}  // namespace

struct ek_mlp {
    int B = 256;
    cudaStream_t stream = nullptr;
    int64_t nparam = 0;
    int64_t off_w[NL], off_b[NL];
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // flat FP32
    bf16 *wb[NL] = {}, *wt[NL] = {};
    bf16 *x = nullptr, *xt = nullptr;
    float *t = nullptr, *y = nullptr;
    float *z[3] = {};
    bf16 *h[3] = {}, *ht[3] = {};   // outputs of hidden layers 0..2
    bf16 *dz[3] = {}, *dzt[3] = {};
    bf16 *dy = nullptr, *dyt = nullptr;
    // data set and iteration state
    float *xs = nullptr, *ts = nullptr;
    int64_t nrows = 0;
    int *idx = nullptr;
    int64_t idx_cap = 0;            // iterations the index buffer holds
    double *loss = nullptr;
    int64_t *step = nullptr, *base = nullptr;
    int64_t host_step = 0;
    std::mt19937_64 rng;
    std::vector<int> perm;          // permutation of the current epoch
    int *err = nullptr;
    long long wait_cycles = ek::tc::WAIT_CYCLES_DEFAULT;
    cudaGraphExec_t graph = nullptr;
    float graph_lr = -1.0f;
    int64_t launches = 0;
};

namespace {

int cuda_err(cudaError_t e, const char *what) {
    return ek::ctx_fail(e == cudaErrorMemoryAllocation ? EK_ERR_NOMEM : EK_ERR_CUDA,
                        (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}
#define EK_MCUDA(call, what)                              \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_err(e_, what); \
    } while (0)

// The GEMM's ring of stages is dynamic shared memory above the 48 KB
// default: allow it for every epilogue on the current device, before any
// launch (and outside any stream capture).
cudaError_t gemm_set_attributes() {
    const void *fns[] = {(const void *)mlp_gemm<EPI_F32>, (const void *)mlp_gemm<EPI_FWD_HIDDEN>,
                         (const void *)mlp_gemm<EPI_FWD_OUT>, (const void *)mlp_gemm<EPI_BWD_HIDDEN>};
    for (const void *f : fns) {
        const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int EPI>
cudaError_t gemm(const GemmArgs &a, cudaStream_t s) {
    const dim3 grid(a.m / TM, a.n / a.nt);
    mlp_gemm<EPI><<<grid, 128, GEMM_SMEM, s>>>(a);
    return cudaGetLastError();
}

GemmArgs args(const bf16 *a, int lda, const bf16 *b, int ldb, int m, int n, int k, int *err,
              long long wait_cycles = ek::tc::WAIT_CYCLES_DEFAULT) {
    GemmArgs g{};
    g.wait_cycles = wait_cycles;
    g.a = a;
    g.lda = lda;
    g.b = b;
    g.ldb = ldb;
    g.m = m;
    g.n = n;
    g.k = k;
    g.nt = std::min(n, NT_MAX);
    g.err = err;
    return g;
}

// Forward of the current batch (x): Z, H of the hidden layers and Y.
int forward(ek_mlp *q) {
    const int B = q->B;
    const bf16 *in = q->x;
    int ldin = INP;
    for (int l = 0; l < 3; ++l) {
        GemmArgs a = args(in, ldin, q->wb[l], DIM_IN[l], B, HID, DIM_IN[l], q->err, q->wait_cycles);
        a.bias = q->p + q->off_b[l];
        a.z = q->z[l];
        a.ldz = HID;
        a.h = q->h[l];
        a.ldh = HID;
        a.ht = q->ht[l];
        a.ldht = B;
        EK_MCUDA(gemm<EPI_FWD_HIDDEN>(a, q->stream), "forward GEMM");
        in = q->h[l];
        ldin = HID;
    }
    GemmArgs a = args(in, HID, q->wb[3], HID, B, OUT, HID, q->err, q->wait_cycles);
    a.bias = q->p + q->off_b[3];
    a.c = q->y;
    a.ldc = OUT;
    EK_MCUDA(gemm<EPI_FWD_OUT>(a, q->stream), "output GEMM");
    q->launches += 4;
    return EK_OK;
}

// Loss gradient, backward GEMMs and bias gradients into q->g.
int backward(ek_mlp *q, bool counted) {
    const int B = q->B;
    mse_grad<<<B, 256, 0, q->stream>>>(q->y, q->t, B, q->dy, q->dyt, q->loss, counted ? q->step : nullptr,
                                      counted ? q->base : nullptr);
    EK_MCUDA(cudaGetLastError(), "loss kernel");
    // layer 3: dW3 = dY^T H2, dZ2 = (dY W3) * silu'(Z2)
    {
        GemmArgs a = args(q->dyt, B, q->ht[2], B, OUT, HID, B, q->err, q->wait_cycles);
        a.c = q->g + q->off_w[3];
        a.ldc = HID;
        EK_MCUDA(gemm<EPI_F32>(a, q->stream), "weight-gradient GEMM");
    }
    const bf16 *up = q->dy;
    int ldup = OUT;
    for (int l = 2; l >= 0; --l) {
        // dZ_l = (dZ_{l+1} W_{l+1}) * silu'(Z_l)
        GemmArgs a = args(up, ldup, q->wt[l + 1], DIM_OUT[l + 1], B, HID, DIM_OUT[l + 1], q->err, q->wait_cycles);
        a.z = q->z[l];
        a.ldz = HID;
        a.h = q->dz[l];
        a.ldh = HID;
        a.ht = q->dzt[l];
        a.ldht = B;
        EK_MCUDA(gemm<EPI_BWD_HIDDEN>(a, q->stream), "backward GEMM");
        // dW_l = dZ_l^T H_{l-1} (H_{-1} = X)
        const bf16 *hin_t = l > 0 ? q->ht[l - 1] : q->xt;
        GemmArgs w = args(q->dzt[l], B, hin_t, B, HID, DIM_IN[l], B, q->err, q->wait_cycles);
        w.c = q->g + q->off_w[l];
        w.ldc = DIM_IN[l];
        EK_MCUDA(gemm<EPI_F32>(w, q->stream), "weight-gradient GEMM");
        up = q->dz[l];
        ldup = HID;
    }
    BiasSeg s{};
    int rows = 0;
    for (int l = 0; l < NL; ++l) {
        s.dzt[l] = l < 3 ? q->dzt[l] : q->dyt;
        s.db[l] = q->g + q->off_b[l];
        s.rows[l] = DIM_OUT[l];
        rows += DIM_OUT[l];
    }
    bias_grads<<<(rows * 32 + 255) / 256, 256, 0, q->stream>>>(s, B);
    EK_MCUDA(cudaGetLastError(), "bias gradients");
    q->launches += 9;
    return EK_OK;
}

int cast_all(ek_mlp *q, bool advance) {
    CastSeg s{};
    int total = 0;
    for (int l = 0; l < NL; ++l) {
        s.w[l] = q->p + q->off_w[l];
        s.wb[l] = q->wb[l];
        s.wt[l] = q->wt[l];
        s.out[l] = DIM_OUT[l];
        s.in[l] = DIM_IN[l];
        total += DIM_OUT[l] * DIM_IN[l];
    }
    cast_weights<<<(total + 255) / 256, 256, 0, q->stream>>>(s, advance ? q->step : nullptr, total);
    EK_MCUDA(cudaGetLastError(), "weight casts");
    ++q->launches;
    return EK_OK;
}

int train_iteration(ek_mlp *q, float lr) {
    gather_batch<<<q->B, 256, 0, q->stream>>>(q->xs, q->ts, q->idx, q->step, q->base, q->B, q->x, q->xt, q->t);
    EK_MCUDA(cudaGetLastError(), "batch gather");
    ++q->launches;
    int rc = forward(q);
    if (rc == EK_OK) rc = backward(q, true);
    if (rc != EK_OK) return rc;
    adam_update<<<(int)((q->nparam + 255) / 256), 256, 0, q->stream>>>(q->p, q->g, q->m, q->v, q->nparam, lr, 0.9f,
                                                                     0.999f, 1e-8f, q->step);
    EK_MCUDA(cudaGetLastError(), "Adam");
    ++q->launches;
    return cast_all(q, true);
}

int check_err(ek_mlp *q) {
    int v = 0;
    EK_MCUDA(cudaMemcpyAsync(&v, q->err, sizeof(int), cudaMemcpyDeviceToHost, q->stream), "error word");
    EK_MCUDA(cudaStreamSynchronize(q->stream), "error word");
    if (v) {
        EK_MCUDA(cudaMemsetAsync(q->err, 0, sizeof(int), q->stream), "error word");
        return ek::ctx_fail(EK_ERR_TIMEOUT, "a bounded wait for the tensor cores gave up");
    }
    return EK_OK;
}

}  // namespace

extern "C" {

int ek_mlp_create(int32_t batch, uint64_t seed, ek_mlp **out) {
    if (!out || batch <= 0 || batch % TM) return ek::ctx_fail(EK_ERR_INVALID, "batch must be a positive multiple of 128");
    *out = nullptr;
    EK_MCUDA(gemm_set_attributes(), "GEMM attributes");
    ek_mlp *q = new ek_mlp();
    q->B = batch;
    q->rng.seed(seed);
    int64_t off = 0;
    for (int l = 0; l < NL; ++l) {
        q->off_w[l] = off;
        off += (int64_t)DIM_OUT[l] * DIM_IN[l];
        q->off_b[l] = off;
        off += DIM_OUT[l];
    }
    q->nparam = off;
    const int B = batch;
    struct A { void **p; size_t bytes; };
    std::vector<A> al = {
        {(void **)&q->p, (size_t)off * 4}, {(void **)&q->g, (size_t)off * 4}, {(void **)&q->m, (size_t)off * 4},
        {(void **)&q->v, (size_t)off * 4},
        {(void **)&q->x, (size_t)B * INP * 2}, {(void **)&q->xt, (size_t)B * INP * 2},
        {(void **)&q->t, (size_t)B * OUT * 4}, {(void **)&q->y, (size_t)B * OUT * 4},
        {(void **)&q->dy, (size_t)B * OUT * 2}, {(void **)&q->dyt, (size_t)B * OUT * 2},
        {(void **)&q->step, 8}, {(void **)&q->base, 8}, {(void **)&q->err, 4},
    };
    for (int l = 0; l < NL; ++l) {
        al.push_back({(void **)&q->wb[l], (size_t)DIM_OUT[l] * DIM_IN[l] * 2});
        al.push_back({(void **)&q->wt[l], (size_t)DIM_OUT[l] * DIM_IN[l] * 2});
    }
    for (int l = 0; l < 3; ++l) {
        al.push_back({(void **)&q->z[l], (size_t)B * HID * 4});
        al.push_back({(void **)&q->h[l], (size_t)B * HID * 2});
        al.push_back({(void **)&q->ht[l], (size_t)B * HID * 2});
        al.push_back({(void **)&q->dz[l], (size_t)B * HID * 2});
        al.push_back({(void **)&q->dzt[l], (size_t)B * HID * 2});
    }
    cudaError_t e = cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
    for (auto &a : al) {
        if (e == cudaSuccess) e = cudaMalloc(a.p, a.bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(*a.p, 0, a.bytes, q->stream);
    }
    if (e != cudaSuccess) {
        ek_mlp_destroy(q);
        return cuda_err(e, "MLP allocation");
    }
    // Glorot-uniform weights over the true fan-in (4 for layer 0), zero biases
    std::vector<float> p(off, 0.0f);
    for (int l = 0; l < NL; ++l) {
        const int fin = l == 0 ? IN : DIM_IN[l];
        const float a = std::sqrt(6.0f / (float)(fin + DIM_OUT[l]));
        std::uniform_real_distribution<float> u(-a, a);
        for (int o = 0; o < DIM_OUT[l]; ++o)
            for (int i = 0; i < fin; ++i) p[q->off_w[l] + (int64_t)o * DIM_IN[l] + i] = u(q->rng);
    }
    int rc = ek_mlp_set_params(q, p.data());
    if (rc != EK_OK) {
        ek_mlp_destroy(q);
        return rc;
    }
    *out = q;
    return EK_OK;
}

int ek_mlp_destroy(ek_mlp *q) {
    if (!q) return ek::ctx_fail(EK_ERR_INVALID, "null MLP");
    if (q->stream) cudaStreamSynchronize(q->stream);
    if (q->graph) cudaGraphExecDestroy(q->graph);
    void *bufs[] = {q->p, q->g, q->m, q->v, q->x, q->xt, q->t, q->y, q->dy, q->dyt, q->step, q->base, q->err,
                    q->xs, q->ts, q->idx, q->loss};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (int l = 0; l < NL; ++l) {
        if (q->wb[l]) cudaFree(q->wb[l]);
        if (q->wt[l]) cudaFree(q->wt[l]);
    }
    for (int l = 0; l < 3; ++l) {
        void *b2[] = {q->z[l], q->h[l], q->ht[l], q->dz[l], q->dzt[l]};
        for (void *b : b2)
            if (b) cudaFree(b);
    }
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
    return EK_OK;
}

int ek_mlp_param_count(const ek_mlp *q, int64_t *n) {
    if (!q || !n) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *n = q->nparam;
    return EK_OK;
}

int ek_mlp_get_params(ek_mlp *q, float *flat) {
    if (!q || !flat) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    EK_MCUDA(cudaMemcpyAsync(flat, q->p, q->nparam * 4, cudaMemcpyDeviceToHost, q->stream), "parameters");
    EK_MCUDA(cudaStreamSynchronize(q->stream), "parameters");
    return EK_OK;
}

int ek_mlp_set_params(ek_mlp *q, const float *flat) {
    if (!q || !flat) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    for (int64_t i = 0; i < q->nparam; ++i)
        if (!std::isfinite(flat[i])) return ek::ctx_fail(EK_ERR_INVALID, "non-finite parameter");
    EK_MCUDA(cudaMemcpyAsync(q->p, flat, q->nparam * 4, cudaMemcpyHostToDevice, q->stream), "parameters");
    EK_MCUDA(cudaMemsetAsync(q->m, 0, q->nparam * 4, q->stream), "Adam state");
    EK_MCUDA(cudaMemsetAsync(q->v, 0, q->nparam * 4, q->stream), "Adam state");
    EK_MCUDA(cudaMemsetAsync(q->step, 0, 8, q->stream), "step");
    q->host_step = 0;
    int rc = cast_all(q, false);
    if (rc != EK_OK) return rc;
    EK_MCUDA(cudaStreamSynchronize(q->stream), "parameters");
    return EK_OK;
}

int ek_mlp_set_data(ek_mlp *q, const float *x, const float *t, int64_t n) {
    if (!q || !x || !t || n < q->B) return ek::ctx_fail(EK_ERR_INVALID, "need at least one batch of rows");
    for (int64_t i = 0; i < n * IN; ++i)
        if (!std::isfinite(x[i])) return ek::ctx_fail(EK_ERR_INVALID, "non-finite input");
    for (int64_t i = 0; i < n * OUT; ++i)
        if (!std::isfinite(t[i])) return ek::ctx_fail(EK_ERR_INVALID, "non-finite target");
    EK_MCUDA(cudaStreamSynchronize(q->stream), "data");
    if (q->graph) cudaGraphExecDestroy(q->graph);  // it holds the old data pointers
    q->graph = nullptr;
    q->perm.clear();
    if (q->xs) cudaFree(q->xs);
    if (q->ts) cudaFree(q->ts);
    q->xs = q->ts = nullptr;
    EK_MCUDA(cudaMalloc(&q->xs, n * IN * 4), "data set");
    EK_MCUDA(cudaMalloc(&q->ts, n * OUT * 4), "data set");
    EK_MCUDA(cudaMemcpyAsync(q->xs, x, n * IN * 4, cudaMemcpyHostToDevice, q->stream), "data set");
    EK_MCUDA(cudaMemcpyAsync(q->ts, t, n * OUT * 4, cudaMemcpyHostToDevice, q->stream), "data set");
    EK_MCUDA(cudaStreamSynchronize(q->stream), "data set");
    q->nrows = n;
    return EK_OK;
}

// `iters` Adam iterations over shuffled batches (a new permutation of the data
// set every epoch, from the MLP's seeded generator); loss_out (optional) gets
// each iteration's mean squared error.
int ek_mlp_train(ek_mlp *q, int32_t iters, float lr, double *loss_out) {
    if (!q || iters < 0 || !(lr > 0.0f)) return ek::ctx_fail(EK_ERR_INVALID, "bad training arguments");
    if (!q->xs) return ek::ctx_fail(EK_ERR_INVALID, "call ek_mlp_set_data first");
    const int64_t per_epoch = q->nrows / q->B;
    constexpr int64_t CHUNK = 1024;  // iterations per index upload
    if (!q->idx) {
        EK_MCUDA(cudaMalloc(&q->idx, CHUNK * q->B * sizeof(int)), "index buffer");
        EK_MCUDA(cudaMalloc(&q->loss, CHUNK * sizeof(double)), "loss buffer");
        q->idx_cap = CHUNK;
    }
    if (q->graph && q->graph_lr != lr) {
        cudaGraphExecDestroy(q->graph);
        q->graph = nullptr;
    }
    std::vector<int> idx;
    std::vector<double> losses;
    int64_t done = 0;
    while (done < iters) {
        const int64_t n = std::min<int64_t>(CHUNK, iters - done);
        idx.clear();
        for (int64_t it = 0; it < n; ++it) {
            const int64_t e = (q->host_step + it) % per_epoch;
            if (e == 0 || (int64_t)q->perm.size() != q->nrows) {
                q->perm.resize(q->nrows);
                for (int64_t i = 0; i < q->nrows; ++i) q->perm[i] = (int)i;
                std::shuffle(q->perm.begin(), q->perm.end(), q->rng);
            }
            for (int b = 0; b < q->B; ++b) idx.push_back(q->perm[(size_t)(e * q->B + b)]);
        }
        EK_MCUDA(cudaMemcpyAsync(q->idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, q->stream),
                 "batch indices");
        EK_MCUDA(cudaMemcpyAsync(q->base, q->step, 8, cudaMemcpyDeviceToDevice, q->stream), "iteration base");
        EK_MCUDA(cudaMemsetAsync(q->loss, 0, n * sizeof(double), q->stream), "loss buffer");
        if (!q->graph) {
            cudaGraph_t g = nullptr;
            const int64_t l0 = q->launches;
            EK_MCUDA(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
            int rc = train_iteration(q, lr);
            cudaError_t e = cudaStreamEndCapture(q->stream, &g);
            q->launches = l0;
            if (rc != EK_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            EK_MCUDA(e, "graph capture");
            e = cudaGraphInstantiate(&q->graph, g, 0);
            cudaGraphDestroy(g);
            EK_MCUDA(e, "graph instantiate");
            q->graph_lr = lr;
        }
        for (int64_t it = 0; it < n; ++it) {
            EK_MCUDA(cudaGraphLaunch(q->graph, q->stream), "graph launch");
            q->launches += 16;
        }
        if (loss_out) {
            losses.resize(n);
            EK_MCUDA(cudaMemcpyAsync(losses.data(), q->loss, n * sizeof(double), cudaMemcpyDeviceToHost, q->stream),
                     "losses");
        }
        int rc = check_err(q);
        if (rc != EK_OK) return rc;
        if (loss_out) std::copy(losses.begin(), losses.end(), loss_out + done);
        q->host_step += n;
        done += n;
    }
    return EK_OK;
}

// Gradients (flat, the layout of the parameters) and loss of one batch of B
// rows, without an update.
int ek_mlp_gradients(ek_mlp *q, const float *x, const float *t, float *grads, double *loss) {
    if (!q || !x || !t || !grads) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    float *xs = nullptr, *ts = nullptr;
    int *idx = nullptr;
    double *l = nullptr;
    std::vector<int> id(q->B);
    for (int i = 0; i < q->B; ++i) id[i] = i;
    auto run = [&]() -> int {
        EK_MCUDA(cudaMalloc(&xs, (size_t)q->B * IN * 4), "staging");
        EK_MCUDA(cudaMalloc(&ts, (size_t)q->B * OUT * 4), "staging");
        EK_MCUDA(cudaMalloc(&idx, (size_t)q->B * 4), "staging");
        EK_MCUDA(cudaMalloc(&l, 8), "staging");
        EK_MCUDA(cudaMemcpyAsync(xs, x, (size_t)q->B * IN * 4, cudaMemcpyHostToDevice, q->stream), "staging");
        EK_MCUDA(cudaMemcpyAsync(ts, t, (size_t)q->B * OUT * 4, cudaMemcpyHostToDevice, q->stream), "staging");
        EK_MCUDA(cudaMemcpyAsync(idx, id.data(), (size_t)q->B * 4, cudaMemcpyHostToDevice, q->stream), "staging");
        EK_MCUDA(cudaMemsetAsync(l, 0, 8, q->stream), "staging");
        gather_batch<<<q->B, 256, 0, q->stream>>>(xs, ts, idx, nullptr, nullptr, q->B, q->x, q->xt, q->t);
        EK_MCUDA(cudaGetLastError(), "batch gather");
        int rc = forward(q);
        if (rc != EK_OK) return rc;
        double *saved = q->loss;
        q->loss = l;
        rc = backward(q, false);
        q->loss = saved;
        if (rc != EK_OK) return rc;
        EK_MCUDA(cudaMemcpyAsync(grads, q->g, q->nparam * 4, cudaMemcpyDeviceToHost, q->stream), "gradients");
        if (loss) EK_MCUDA(cudaMemcpyAsync(loss, l, 8, cudaMemcpyDeviceToHost, q->stream), "loss");
        return check_err(q);
    };
    const int rc = run();
    cudaFree(xs);
    cudaFree(ts);
    cudaFree(idx);
    cudaFree(l);
    return rc;
}

// y (n x 512) = network(x (n x 4)), in batches of B rows.
int ek_mlp_forward(ek_mlp *q, const float *x, int64_t n, float *y) {
    if (!q || !x || !y || n < 0) return ek::ctx_fail(EK_ERR_INVALID, "bad forward arguments");
    float *xs = nullptr, *ts = nullptr;
    int *idx = nullptr;
    std::vector<int> id(q->B);
    for (int i = 0; i < q->B; ++i) id[i] = i;
    std::vector<float> xb((size_t)q->B * IN);
    auto run = [&]() -> int {
        EK_MCUDA(cudaMalloc(&xs, (size_t)q->B * IN * 4), "staging");
        EK_MCUDA(cudaMalloc(&ts, (size_t)q->B * OUT * 4), "staging");
        EK_MCUDA(cudaMalloc(&idx, (size_t)q->B * 4), "staging");
        EK_MCUDA(cudaMemsetAsync(ts, 0, (size_t)q->B * OUT * 4, q->stream), "staging");
        EK_MCUDA(cudaMemcpyAsync(idx, id.data(), (size_t)q->B * 4, cudaMemcpyHostToDevice, q->stream), "staging");
        for (int64_t r0 = 0; r0 < n; r0 += q->B) {
            const int64_t cnt = std::min<int64_t>(q->B, n - r0);
            std::fill(xb.begin(), xb.end(), 0.0f);
            std::copy(x + r0 * IN, x + (r0 + cnt) * IN, xb.begin());
            EK_MCUDA(cudaMemcpyAsync(xs, xb.data(), xb.size() * 4, cudaMemcpyHostToDevice, q->stream), "staging");
            gather_batch<<<q->B, 256, 0, q->stream>>>(xs, ts, idx, nullptr, nullptr, q->B, q->x, q->xt, q->t);
            EK_MCUDA(cudaGetLastError(), "batch gather");
            int rc = forward(q);
            if (rc != EK_OK) return rc;
            EK_MCUDA(cudaMemcpyAsync(y + r0 * OUT, q->y, cnt * OUT * 4, cudaMemcpyDeviceToHost, q->stream), "output");
            EK_MCUDA(cudaStreamSynchronize(q->stream), "output");
        }
        return check_err(q);
    };
    const int rc = run();
    cudaFree(xs);
    cudaFree(ts);
    cudaFree(idx);
    return rc;
}

int ek_mlp_launch_count(const ek_mlp *q, int64_t *out) {
    if (!q || !out) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *out = q->launches;
    return EK_OK;
}

int ek_mlp_set_wait_cycles(ek_mlp *q, int64_t cycles) {
    if (!q || cycles < 1) return ek::ctx_fail(EK_ERR_INVALID, "need a network and cycles >= 1");
    EK_MCUDA(cudaStreamSynchronize(q->stream), "wait bound");
    if (q->graph) cudaGraphExecDestroy(q->graph);  // it holds the old bound
    q->graph = nullptr;
    q->wait_cycles = cycles;
    return EK_OK;
}

}  // extern "C"

namespace {
// One block of 64 threads: thread 0 waits, at most `cycles`, on an mbarrier
// that expects one arrival; thread 32 (another warp) arrives only if
// `arrive`.  out[0] = 1 if the wait gave up, out[1] = 1 when thread 0 is done.
__global__ void __launch_bounds__(64) wait_selftest(long long cycles, int arrive, int *out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        ek::tc::mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 32 && arrive)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(ek::tc::smem_u32(&bar)) : "memory");
    if (threadIdx.x == 0) {
        const bool ok = ek::tc::mbar_wait_bounded(&bar, 0, cycles);
        out[0] = ok ? 0 : 1;
        out[1] = 1;
    }
}
}  // namespace

extern "C" {

int ek_wait_selftest(int64_t cycles, int32_t arrive) {
    if (cycles < 1) return ek::ctx_fail(EK_ERR_INVALID, "need cycles >= 1");
    int *out = nullptr;
    EK_MCUDA(cudaMalloc(&out, 2 * sizeof(int)), "self-test word");
    cudaError_t e = cudaMemset(out, 0, 2 * sizeof(int));
    if (e == cudaSuccess) {
        wait_selftest<<<1, 64>>>((long long)cycles, arrive ? 1 : 0, out);
        e = cudaGetLastError();
    }
    int h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, out, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(out);
    EK_MCUDA(e, "self-test kernel");
    if (h[1] != 1) return ek::ctx_fail(EK_ERR_CUDA, "self-test kernel did not finish");
    if (h[0]) return ek::ctx_fail(EK_ERR_TIMEOUT, "the bounded wait gave up (as asked: nothing arrived)");
    return EK_OK;
}

// C (m x n, FP32, row stride ldc) = A (m x k) B (n x k)^T on the tensor cores;
// BF16 device operands, m a multiple of 128, n a multiple of 16 (and of 128
// above 128), k a multiple of 16, lda and ldb multiples of 8.
int ek_gemm_bf16(const uint16_t *a, int32_t lda, const uint16_t *b, int32_t ldb, float *c, int32_t ldc, int32_t m,
                 int32_t n, int32_t k, void *stream) {
    if (!a || !b || !c || m <= 0 || n <= 0 || k <= 0) return ek::ctx_fail(EK_ERR_INVALID, "bad GEMM arguments");
    if (m % TM || n % 16 || (n > NT_MAX && n % NT_MAX) || k % 16 || lda % 8 || ldb % 8 || lda < k || ldb < k ||
        ldc < n)
        return ek::ctx_fail(EK_ERR_UNSUPPORTED, "GEMM shape outside the supported tiling");
    if (((uintptr_t)a | (uintptr_t)b) & 15) return ek::ctx_fail(EK_ERR_INVALID, "operands must be 16-byte aligned");
    static int *err = nullptr;
    if (!err) {
        EK_MCUDA(cudaMalloc(&err, 4), "error word");
        EK_MCUDA(cudaMemset(err, 0, 4), "error word");
    }
    EK_MCUDA(gemm_set_attributes(), "GEMM attributes");
    GemmArgs g = args((const bf16 *)a, lda, (const bf16 *)b, ldb, m, n, k, err);
    g.c = c;
    g.ldc = ldc;
    EK_MCUDA(gemm<EPI_F32>(g, (cudaStream_t)stream), "GEMM");
    int v = 0;
    EK_MCUDA(cudaMemcpyAsync(&v, err, 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream), "error word");
    EK_MCUDA(cudaStreamSynchronize((cudaStream_t)stream), "GEMM");
    if (v) {
        cudaMemset(err, 0, 4);
        return ek::ctx_fail(EK_ERR_TIMEOUT, "a bounded wait for the tensor cores gave up");
    }
    return EK_OK;
}

}  // extern "C"
