// ek_batch.cu -- many independent channels stepped together (new; the
// reference runs one channel per process).
//
// Each channel keeps its own context (ek_ctx: populations, fields, Poisson
// plan, wall profiles, reference rows) and all of them step in lockstep with
// four launches per step, whatever the number of channels:
//   LBM      one persistent kernel over a host-built tile work-list.  A tile is
//            {channel, first row, first column, width}; channels narrower
//            than the block put several rows into one tile.  Blocks claim
//            runs of tiles from a queue (one wave: the grid is the number of
//            blocks that fit on the GPU) and stage the current channel's
//            constants in shared memory when the channel changes.
//   Poisson  the batched passes of ek_poisson.cu: each block's item names its
//            channel and its first row pair (row FFTs) or first x-mode
//            (column solve; a channel's FP64 zero mode is an item of its own).
// Steps run in cycles of an even number R of steps.  The last step of a cycle
// writes the moments and, with re-basing on, the cycle ends with the re-basing
// of every channel's shifted populations to its new row means (three more
// launches, done in place so that device pointers never change).  A whole
// cycle is captured once in a CUDA graph and replayed.  The block shape of the
// LBM kernel (threads, tile width, blocks per SM) is picked by timing the
// candidates (ek_batch_autotune).
//
// Per step and channel the arithmetic is that of ek_step: the node update is
// the same device function (ek_lbm_f32.cuh), the Poisson passes the same
// device bodies, the re-basing the same formula, so a batch gives each
// channel the bits that ek_step with the same re-base interval gives it.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "ek_ctx.h"
#include "ek_lbm_f32.cuh"

using namespace ek;

namespace {

constexpr int REFS_TPB = 256;

// ---- kernels ---------------------------------------------------------------

// Persistent LBM kernel over the tile list; TXB threads = tile width x rows.
// MINB: blocks per SM the register allocation must allow (the block shapes,
// kShapes below, pair a width with it).
// Tiles are handed out from a queue, TILE_CHUNK consecutive tiles (same
// channel, adjacent rows) at a time: queue[0] is the next unclaimed tile,
// queue[1] counts the blocks that found the list empty; the last of them
// puts both back to zero for the next launch (every other block has made its
// last claim by then), so the queue needs no reset between launches or graph
// replays.
constexpr int TILE_CHUNK = 4;

template <typename S, bool FIRST, bool EE, int TXB, int MINB>
__global__ void __launch_bounds__(TXB, MINB)
batch_lbm(const ChanF *__restrict__ chans, const S *const *__restrict__ src, S *const *__restrict__ dst,
          double *const *__restrict__ fields, const int4 *__restrict__ tiles, int ntiles, int *__restrict__ queue,
          bool mom, int sbuf) {
    __shared__ ChanF ks;
    __shared__ int claim;
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) claim = atomicAdd(queue, TILE_CHUNK);
        __syncthreads();
        const int t0 = claim;
        if (t0 >= ntiles) break;  // the same for every thread of the block
        const int t1 = min(ntiles, t0 + TILE_CHUNK);
        for (int t = t0; t < t1; ++t) {
            const int4 tl = tiles[t];  // {channel, y0, x0, width}
            if (tl.x != cur) {
                __syncthreads();
                if (threadIdx.x == 0) ks = chans[tl.x];
                __syncthreads();
                cur = tl.x;
            }
            const int r = threadIdx.x / tl.w;
            const int x = tl.z + (threadIdx.x - r * tl.w), y = tl.y + r;
            if (r < TXB / tl.w && x < ks.nx && y < ks.ny)
                // 32-bit indexing: batched channels are at most 4096 x 8194 (ek_batch_create)
                node_shifted<S, FIRST, EE, uint32_t>(ks, src[cur], dst[cur], fields[cur], x, y, mom, sbuf);
        }
        __syncthreads();  // every thread has read `claim` before thread 0 claims again
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
            queue[0] = 0;
            queue[1] = 0;
            __threadfence();
        }
    }
}

// New reference rows of every channel into its spare buffer: item {channel, row}.
__global__ void __launch_bounds__(REFS_TPB)
batch_row_refs(const ChanF *__restrict__ chans, double *const *__restrict__ fields, const int4 *__restrict__ kq,
               float *const *__restrict__ spare, const int2 *__restrict__ rows) {
    const int2 it = rows[blockIdx.x];
    const ChanF &k = chans[it.x];
    const int4 q = kq[it.x];
    row_refs_dev(k.nx, k.nxp, k.ny, k.plane, fields[it.x], q.x, q.y, q.z, spare[it.x], it.y);
}

// Re-basing of all 27 planes of every node of a tile to the spare rows.
template <typename S, int TXB>
__global__ void __launch_bounds__(TXB)
batch_rebase(const ChanF *__restrict__ chans, S *const *__restrict__ pops, float *const *__restrict__ spare,
             const int4 *__restrict__ tiles) {
    const int4 tl = tiles[blockIdx.x];
    const ChanF &k = chans[tl.x];
    const int r = threadIdx.x / tl.w;
    const int x = tl.z + (threadIdx.x - r * tl.w), y = tl.y + r;
    if (r >= TXB / tl.w || x >= k.nx || y >= k.ny) return;  // each node of the tile once
    S *base = pops[tl.x] + (size_t)y * k.nxp + x;
    for (int pl = 0; pl < 27; ++pl) rebase_dev<S>(base + (size_t)pl * k.plane, pl, k.ny, y, k.kref, spare[tl.x]);
}

// The spare rows become the current ones: item {channel, row}, 3 species.
__global__ void batch_commit_refs(const ChanF *__restrict__ chans, float *const *__restrict__ spare,
                                  const int2 *__restrict__ rows, int nrows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nrows) return;
    const int2 it = rows[i / 3];
    const int s = i - 3 * (i / 3);
    const ChanF &k = chans[it.x];
    const size_t o = (size_t)s * k.ny + it.y;
    const_cast<float *>(k.kref)[o] = spare[it.x][o];
}

// ---- launchers --------------------------------------------------------------

template <typename S, int TXB, int MINB>
cudaError_t lbm_t(const ChanF *chans, const void *src, void *dst, double *const *fields, const int4 *tiles,
                  int ntiles, int *queue, int grid, bool first, bool ee, bool mom, int sbuf, cudaStream_t s) {
    const S *const *a = (const S *const *)src;
    S *const *b = (S *const *)dst;
#define EK_BL(F, E) \
    batch_lbm<S, F, E, TXB, MINB><<<grid, TXB, 0, s>>>(chans, a, b, fields, tiles, ntiles, queue, mom, sbuf)
    if (first) {
        if (ee) EK_BL(true, true);
        else EK_BL(true, false);
    } else {
        if (ee) EK_BL(false, true);
        else EK_BL(false, false);
    }
#undef EK_BL
    return cudaGetLastError();
}

// Block shapes of the batched LBM kernel: threads, the widest tile (a tile is
// min(width, nx) columns by threads / that many rows) and the blocks per SM
// that the register allocation must allow.  At 72 registers (7 blocks of 128,
// 14 of 64) the batched node update spills a little; 10 blocks of 64, 5 of
// 128 and 3 of 256 do not.  Narrower tiles than threads give 2-D tiles whose
// rows share their pulled neighbours in L1.
struct Shape {
    int threads, width, minb;
};
constexpr Shape kShapes[EK_BATCH_SHAPES] = {{64, 64, 10},   {128, 128, 5}, {128, 128, 7},
                                             {256, 256, 3}, {256, 64, 3},  {256, 128, 3}};

#define EK_SHAPE_CASES(F) F(0) F(1) F(2) F(3) F(4) F(5)
static_assert(EK_BATCH_SHAPES == 6, "one case per shape");

template <typename S>
cudaError_t lbm_s(int shape, const ChanF *chans, const void *src, void *dst, double *const *fields,
                  const int4 *tiles, int ntiles, int *queue, int grid, bool first, bool ee, bool mom, int sbuf,
                  cudaStream_t s) {
    switch (shape) {
#define EK_CASE(I)                                                                                           \
    case I:                                                                                                  \
        return lbm_t<S, kShapes[I].threads, kShapes[I].minb>(chans, src, dst, fields, tiles, ntiles, queue, grid, \
                                                             first, ee, mom, sbuf, s);
        EK_SHAPE_CASES(EK_CASE)
#undef EK_CASE
        default: return cudaErrorInvalidValue;
    }
}

template <typename S>
cudaError_t rebase_s(int txb, const ChanF *chans, void *pops, float *const *spare, const int4 *tiles, int ntiles,
                     cudaStream_t s) {
    S *const *p = (S *const *)pops;
    if (txb == 64) batch_rebase<S, 64><<<ntiles, 64, 0, s>>>(chans, p, spare, tiles);
    else if (txb == 256) batch_rebase<S, 256><<<ntiles, 256, 0, s>>>(chans, p, spare, tiles);
    else batch_rebase<S, 128><<<ntiles, 128, 0, s>>>(chans, p, spare, tiles);
    return cudaGetLastError();
}

// Blocks of the (non-first) LBM kernel of a shape resident per SM.
template <typename S>
int lbm_occupancy(int shape) {
    int occ = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (shape) {
#define EK_CASE(I)                                                                                                  \
    case I:                                                                                                         \
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                                          \
            &occ, batch_lbm<S, false, false, kShapes[I].threads, kShapes[I].minb>, kShapes[I].threads, 0);          \
        break;
        EK_SHAPE_CASES(EK_CASE)
#undef EK_CASE
        default: break;
    }
    return e == cudaSuccess && occ > 0 ? occ : 1;
}

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

}  // namespace

struct ek_batch {
    std::vector<ek_ctx *> ch;
    std::vector<int> kcur;           // each channel's current reference buffer when the tables were built
    std::vector<char> active;        // channels that step (frozen ones keep their state)
    std::vector<int64_t> ch_steps;   // steps each channel has taken in the batch
    int storage = EK_STORE_F32;
    cudaStream_t stream = nullptr;
    int cur = 0;                     // population buffer holding the current state (all channels)
    bool state_pre = false;
    bool explicit_e_once = false;
    int64_t steps = 0;
    int64_t nodes = 0;
    int cycle = 200;                 // steps per cycle (even)
    bool rebase = true;
    bool use_graph = true;
    bool poisson_f32 = false;        // every channel runs the FP32 Poisson form
    cudaGraphExec_t graph = nullptr;
    int graph_cur = -1;              // parity the graph was captured for
    int64_t launches = 0;
    // device tables
    ChanF *d_chanf = nullptr;
    Chan *d_chan = nullptr;
    PoissonPlan *d_plans = nullptr;
    void **d_pops[2] = {nullptr, nullptr};  // per parity: channel -> population buffer
    double **d_fields = nullptr;
    float **d_spare = nullptr;
    int4 *d_kq = nullptr;
    int4 *d_tiles = nullptr;
    int ntiles = 0, shape = 1, txb = 128, grid = 0;  // kShapes[shape], txb = its threads
    int *d_queue = nullptr;          // LBM tile queue: next tile, finished blocks (zero between launches)
    int2 *d_pairs = nullptr;         // Poisson row-pair items
    int npairs = 0;
    int3 *d_modes = nullptr;         // Poisson x-mode items
    int nmodes = 0;
    int2 *d_rows = nullptr;          // {channel, row} of every row
    int nrows = 0;
    // residuals
    double **d_snaps = nullptr;
    int4 *d_ritems = nullptr;
    int nritems = 0;
    int2 *d_rranges = nullptr;
    double *d_rpart = nullptr;       // partials, then 8 sums per channel
    int nrpart = 0;
};

namespace {

int cuda_err(cudaError_t e, const char *what) {
    return ek::ctx_fail(e == cudaErrorMemoryAllocation ? EK_ERR_NOMEM : EK_ERR_CUDA,
                        (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

#define EK_BCUDA(call, what)                              \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_err(e_, what); \
    } while (0)

template <typename T>
int upload(T **dst, const std::vector<T> &v, cudaStream_t s) {
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    if (v.empty()) return EK_OK;
    EK_BCUDA(cudaMalloc(dst, v.size() * sizeof(T)), "batch table");
    EK_BCUDA(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "batch table");
    EK_BCUDA(cudaStreamSynchronize(s), "batch table");
    return EK_OK;
}

// LBM + three Poisson passes; the FP32 form's column solve is two kernels.
int launches_per_step(const ek_batch *) { return 4; }

void release_graph(ek_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_cur = -1;
}

// LBM tiles of a block shape: min(width, nx) columns by threads / that many
// rows; the grid is one wave.
int build_tiles(ek_batch *b, int shape) {
    if (shape < 0 || shape >= EK_BATCH_SHAPES) return ek::ctx_fail(EK_ERR_INVALID, "no such block shape");
    const int txb = kShapes[shape].threads;
    std::vector<int4> tiles;
    for (size_t i = 0; i < b->ch.size(); ++i) {
        if (!b->active[i]) continue;
        const ek_params &p = b->ch[i]->p;
        const int w = std::min(kShapes[shape].width, p.nx);
        const int rows = txb / w;
        for (int y = 0; y < p.ny; y += rows)
            for (int x0 = 0; x0 < p.nx; x0 += w) tiles.push_back(make_int4((int)i, y, x0, w));
    }
    release_graph(b);
    int rc = upload(&b->d_tiles, tiles, b->stream);
    if (rc != EK_OK) return rc;
    if (!b->d_queue) {
        EK_BCUDA(cudaMalloc(&b->d_queue, 2 * sizeof(int)), "tile queue");
        EK_BCUDA(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(int), b->stream), "tile queue");
    }
    b->ntiles = (int)tiles.size();
    b->txb = txb;
    b->shape = shape;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int occ = b->storage == EK_STORE_F16 ? lbm_occupancy<__half>(shape) : lbm_occupancy<float>(shape);
    b->grid = std::max(1, std::min((b->ntiles + TILE_CHUNK - 1) / TILE_CHUNK, sms * occ));
    return EK_OK;
}

// Per-channel tables and the Poisson / row / residual item lists.
int build_tables(ek_batch *b) {
    std::vector<ChanF> cf;
    std::vector<Chan> cc;
    std::vector<PoissonPlan> pl;
    std::vector<void *> p0, p1;
    std::vector<double *> fl, sn;
    std::vector<float *> sp;
    std::vector<int4> kq, ritems;
    std::vector<int2> pairs, rows, rranges;
    std::vector<int3> modes, zeros;  // column items: zero modes first (the longer blocks start first)
    release_graph(b);
    b->kcur.clear();
    int nrpart = 0;
    bool f32 = true;
    for (ek_ctx *c : b->ch) f32 = f32 && ek::ctx_poisson_f32(c);
    b->poisson_f32 = f32;
    if (!f32)
        return ek::ctx_fail(EK_ERR_UNSUPPORTED, "batched channels run the FP32 Poisson form (EK_OPT_POISSON 0 or 2)");
    size_t field_bytes = 0;  // right-hand side + psi (FP32 planes) of the stepping channels
    for (size_t i = 0; i < b->ch.size(); ++i)
        if (b->active[i]) field_bytes += 2 * b->ch[i]->plane * sizeof(float);
    for (ek_ctx *c : b->ch) c->keep_l2 = keep_l2_fits(field_bytes);
    for (size_t i = 0; i < b->ch.size(); ++i) {
        ek_ctx *c = b->ch[i];
        ek::ctx_refresh(c);
        int rc = ek::ctx_residual_buffers(c);
        if (rc != EK_OK) return rc;
        b->kcur.push_back(c->kcur);
        cf.push_back(make_chanf(c->chan));
        cc.push_back(c->chan);
        pl.push_back(c->pp);
        p0.push_back(c->pops[0]);
        p1.push_back(c->pops[1]);
        fl.push_back(c->fields);
        sn.push_back(c->snap);
        sp.push_back(c->kref[c->kcur ^ 1]);
        kq.push_back(make_int4(c->kq[0], c->kq[1], c->kq[2], 0));
        const int nx = c->p.nx, n = c->pp.n;
        if (b->active[i]) {
            const int per = 256 / (nx >> 4);
            for (int q = 0; q < (n + 1) / 2; q += per) pairs.push_back(make_int2((int)i, q));
            const int M = poisson_tridiag_modes(n);
            // the zero mode in FP64 (an item with 0 modes per block); modes 1.. in FP32
            zeros.push_back(make_int3((int)i, 0, 0));
            for (int m0 = 1; m0 <= nx / 2; m0 += M) modes.push_back(make_int3((int)i, m0, M));
            for (int y = 0; y < c->p.ny; ++y) rows.push_back(make_int2((int)i, y));
        }
        const int nb = residual_blocks(c->chan);
        for (int k = 0; k < nb; ++k) ritems.push_back(make_int4((int)i, k, nb, nrpart));
        rranges.push_back(make_int2(nrpart, nb));
        nrpart += nb;
    }
    int rc;
    if ((rc = upload(&b->d_chanf, cf, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_chan, cc, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_plans, pl, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_pops[0], p0, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_pops[1], p1, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_fields, fl, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_snaps, sn, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_spare, sp, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_kq, kq, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_pairs, pairs, b->stream)) != EK_OK) return rc;
    modes.insert(modes.begin(), zeros.begin(), zeros.end());
    if ((rc = upload(&b->d_modes, modes, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_rows, rows, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_ritems, ritems, b->stream)) != EK_OK) return rc;
    if ((rc = upload(&b->d_rranges, rranges, b->stream)) != EK_OK) return rc;
    b->npairs = (int)pairs.size();
    b->nmodes = (int)modes.size();
    b->nrows = (int)rows.size();
    b->nritems = (int)ritems.size();
    if (b->d_rpart) cudaFree(b->d_rpart);
    b->d_rpart = nullptr;
    EK_BCUDA(cudaMalloc(&b->d_rpart, ((size_t)nrpart + b->ch.size()) * 8 * sizeof(double)), "residual partials");
    b->nrpart = nrpart;
    return EK_OK;
}

// One step of every channel: LBM, then the three Poisson passes.
int launch_step(ek_batch *b, bool first, bool ee, bool mom) {
    const void *src = b->d_pops[b->cur];
    void *dst = b->d_pops[b->cur ^ 1];
    cudaError_t e = b->storage == EK_STORE_F16
                        ? lbm_s<__half>(b->shape, b->d_chanf, src, dst, b->d_fields, b->d_tiles, b->ntiles,
                                        b->d_queue, b->grid, first, ee, mom, b->cur, b->stream)
                        : lbm_s<float>(b->shape, b->d_chanf, src, dst, b->d_fields, b->d_tiles, b->ntiles,
                                       b->d_queue, b->grid, first, ee, mom, b->cur, b->stream);
    EK_BCUDA(e, "batch LBM kernel");
    EK_BCUDA(batch_poisson(0, b->d_plans, b->d_chan, b->d_fields, b->d_pairs, b->npairs, false, b->stream),
             "batch rows");
    EK_BCUDA(batch_tridiag_f32(b->d_plans, b->d_modes, b->nmodes, b->stream), "batch modes");
    // the FP64 psi planes follow on the steps that write the moments
    EK_BCUDA(batch_poisson(2, b->d_plans, b->d_chan, b->d_fields, b->d_pairs, b->npairs, mom, b->stream),
             "batch rows");
    b->launches += launches_per_step(b);
    b->cur ^= 1;
    return EK_OK;
}

// Re-base every channel's current populations to its new row means, in place.
int launch_rebase(ek_batch *b) {
    if (b->nrows == 0) return EK_OK;  // every channel frozen
    batch_row_refs<<<b->nrows, REFS_TPB, 0, b->stream>>>(b->d_chanf, b->d_fields, b->d_kq, b->d_spare, b->d_rows);
    EK_BCUDA(cudaGetLastError(), "batch row references");
    void *pops = b->d_pops[b->cur];
    EK_BCUDA(b->storage == EK_STORE_F16 ? rebase_s<__half>(b->txb, b->d_chanf, pops, b->d_spare, b->d_tiles,
                                                           b->ntiles, b->stream)
                                        : rebase_s<float>(b->txb, b->d_chanf, pops, b->d_spare, b->d_tiles,
                                                          b->ntiles, b->stream),
             "batch rebase");
    batch_commit_refs<<<(3 * b->nrows + 255) / 256, 256, 0, b->stream>>>(b->d_chanf, b->d_spare, b->d_rows,
                                                                         b->nrows);
    EK_BCUDA(cudaGetLastError(), "batch reference commit");
    b->launches += 3;
    return EK_OK;
}

// Graph of one full cycle starting at parity b->cur: R steps, moments on the
// last, then the re-basing.
int capture_graph(ek_batch *b) {
    release_graph(b);
    const int saved_cur = b->cur;
    const int64_t saved_launches = b->launches;
    cudaGraph_t g = nullptr;
    EK_BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    int rc = EK_OK;
    for (int i = 0; i < b->cycle && rc == EK_OK; ++i) rc = launch_step(b, false, false, i == b->cycle - 1);
    if (rc == EK_OK && b->rebase) rc = launch_rebase(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->cur = saved_cur;
    b->launches = saved_launches;
    if (rc != EK_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    EK_BCUDA(e, "graph capture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    EK_BCUDA(e, "graph instantiate");
    b->graph_cur = b->cur;
    return EK_OK;
}

// Per-channel state after `advanced` batch steps of the active channels.
void sync_channel_state(ek_batch *b, int64_t advanced) {
    for (size_t i = 0; i < b->ch.size(); ++i) {
        if (!b->active[i]) continue;
        ek_ctx *c = b->ch[i];
        b->ch_steps[i] += advanced;
        c->cur = b->cur;
        c->state_pre = b->state_pre;
        c->explicit_e_once = b->explicit_e_once;
        c->steps = b->ch_steps[i];
        c->e_stale = true;
    }
}

// The channels must not have been stepped or re-based on their own since the
// tables were built.
int check_channels(ek_batch *b) {
    for (size_t i = 0; i < b->ch.size(); ++i) {
        const ek_ctx *c = b->ch[i];
        if (!c->initialised) return ek::ctx_fail(EK_ERR_INVALID, "call ek_batch_init_equilibrium before stepping");
        if (!b->active[i]) continue;
        if (c->cur != b->cur || c->kcur != b->kcur[i] || c->steps != b->ch_steps[i])
            return ek::ctx_fail(EK_ERR_INVALID,
                                "a channel was stepped or re-based on its own; call ek_batch_init_equilibrium");
    }
    return EK_OK;
}

int launches_per_cycle(const ek_batch *b) { return b->cycle * launches_per_step(b) + (b->rebase ? 3 : 0); }

}  // namespace

extern "C" {

int ek_batch_create(const ek_params *params, int32_t count, ek_batch **out) {
    if (!params || !out || count <= 0) return ek::ctx_fail(EK_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    for (int32_t i = 0; i < count; ++i) {
        const ek_params &p = params[i];
        if (p.storage != params[0].storage)
            return ek::ctx_fail(EK_ERR_INVALID, "all channels of a batch need one storage mode");
        if (p.storage != EK_STORE_F32 && p.storage != EK_STORE_F16)
            return ek::ctx_fail(EK_ERR_UNSUPPORTED, "batches use FP32 or FP16 storage");
        static_assert(index32_fits((size_t)4096 * 8194), "batched channels use 32-bit indexing");
        if (!pow2(p.nx) || p.nx < 16 || p.nx > 4096)
            return ek::ctx_fail(EK_ERR_UNSUPPORTED, "batched channels need nx a power of two in [16, 4096]");
        if (p.flags & EK_FLAG_EXPLICIT_E) return ek::ctx_fail(EK_ERR_UNSUPPORTED, "batches derive E from psi");
        if (p.ny < 3 || poisson_tridiag_modes(p.ny - 2) == 0)
            return ek::ctx_fail(EK_ERR_UNSUPPORTED, "batched channels need 3 <= ny <= 8194");
    }
    ek_batch *b = new ek_batch();
    b->storage = params[0].storage;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        b->stream = nullptr;
        ek_batch_destroy(b);
        return cuda_err(e, "stream create");
    }
    for (int32_t i = 0; i < count; ++i) {
        ek_ctx *c = nullptr;
        int rc = ek_create(&params[i], &c);
        if (rc == EK_OK) rc = ek_set_stream(c, b->stream);
        if (rc != EK_OK) {
            if (c) ek_destroy(c);
            ek_batch_destroy(b);
            return rc;
        }
        b->ch.push_back(c);
        b->active.push_back(1);
        b->ch_steps.push_back(0);
        b->nodes += (int64_t)params[i].nx * params[i].ny;
    }
    int rc = build_tables(b);
    if (rc == EK_OK) rc = build_tiles(b, 1);
    if (rc != EK_OK) {
        ek_batch_destroy(b);
        return rc;
    }
    *out = b;
    return EK_OK;
}

int ek_batch_destroy(ek_batch *b) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    if (b->stream) cudaStreamSynchronize(b->stream);
    release_graph(b);
    for (ek_ctx *c : b->ch) ek_destroy(c);  // the channels do not own the batch's stream
    void *tables[] = {b->d_chanf, b->d_chan,  b->d_plans,  b->d_pops[0],  b->d_pops[1], b->d_fields,
                      b->d_spare, b->d_kq,    b->d_tiles,  b->d_pairs,    b->d_modes,   b->d_rows,
                      b->d_snaps, b->d_ritems, b->d_rranges, b->d_rpart,  b->d_queue};
    for (void *t : tables)
        if (t) cudaFree(t);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EK_OK;
}

int ek_batch_count(const ek_batch *b, int32_t *count, int64_t *nodes) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    if (count) *count = (int32_t)b->ch.size();
    if (nodes) *nodes = b->nodes;
    return EK_OK;
}

int ek_batch_channel(ek_batch *b, int32_t i, ek_ctx **out) {
    if (!b || !out || i < 0 || i >= (int32_t)b->ch.size()) return ek::ctx_fail(EK_ERR_INVALID, "bad channel index");
    *out = b->ch[i];
    return EK_OK;
}

int ek_batch_set_cycle(ek_batch *b, int32_t steps, int32_t rebase, int32_t use_graph) {
    if (!b || steps < 2 || (steps & 1)) return ek::ctx_fail(EK_ERR_INVALID, "a cycle is an even number >= 2 of steps");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    b->cycle = steps;
    b->rebase = rebase != 0;
    b->use_graph = use_graph != 0;
    release_graph(b);
    return EK_OK;
}

int ek_batch_init_equilibrium(ek_batch *b) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    // one first-step variant for all: if any channel carries explicit E
    // (reference Poisson-Boltzmann start, fields loaded with E), the others get
    // the E of their psi written to their E planes
    std::fill(b->active.begin(), b->active.end(), 1);
    std::fill(b->ch_steps.begin(), b->ch_steps.end(), 0);
    bool ee = false;
    for (ek_ctx *c : b->ch) ee = ee || c->explicit_e_once;
    for (ek_ctx *c : b->ch) {
        if (ee && !c->explicit_e_once) {
            EK_BCUDA(launch_efield_f64(c->chan, c->fields, b->stream), "efield kernel");
            c->explicit_e_once = true;
        }
        c->cur = b->cur;
        const int rc = ek_init_equilibrium(c);
        if (rc != EK_OK) return rc;
    }
    b->state_pre = true;
    b->explicit_e_once = ee;
    b->steps = 0;
    int rc = build_tables(b);  // reference buffers may have changed
    if (rc == EK_OK) rc = build_tiles(b, b->shape);
    if (rc != EK_OK) return rc;
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch init");
    sync_channel_state(b, 0);
    return EK_OK;
}

int ek_batch_step(ek_batch *b, int32_t nsteps) {
    if (!b || nsteps < 0) return ek::ctx_fail(EK_ERR_INVALID, "bad batch step arguments");
    int rc = check_channels(b);
    if (rc != EK_OK) return rc;
    int32_t done = 0;
    while (done < nsteps) {
        const int32_t left = nsteps - done;
        const bool special = b->state_pre || b->explicit_e_once;
        if (b->use_graph && !special && b->steps % b->cycle == 0 && left >= b->cycle) {
            if (!b->graph || b->graph_cur != b->cur) {
                rc = capture_graph(b);
                if (rc != EK_OK) return rc;
            }
            EK_BCUDA(cudaGraphLaunch(b->graph, b->stream), "graph launch");
            b->launches += launches_per_cycle(b);
            done += b->cycle;
            b->steps += b->cycle;
            continue;
        }
        const bool cycle_end = (b->steps + 1) % b->cycle == 0;
        rc = launch_step(b, b->state_pre, b->explicit_e_once, left == 1 || cycle_end);
        if (rc != EK_OK) return rc;
        if (b->rebase && cycle_end) {
            rc = launch_rebase(b);
            if (rc != EK_OK) return rc;
        }
        b->state_pre = false;
        b->explicit_e_once = false;
        ++done;
        ++b->steps;
    }
    sync_channel_state(b, done);
    return EK_OK;
}

int ek_batch_sync(ek_batch *b) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    return EK_OK;
}

int ek_batch_step_count(const ek_batch *b, int64_t *out) {
    if (!b || !out) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *out = b->steps;
    return EK_OK;
}

int ek_batch_launch_count(const ek_batch *b, int64_t *out) {
    if (!b || !out) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *out = b->launches;
    return EK_OK;
}

int ek_batch_shape_info(int32_t index, int32_t *threads, int32_t *width, int32_t *blocks_per_sm) {
    if (index < 0 || index >= EK_BATCH_SHAPES) return ek::ctx_fail(EK_ERR_INVALID, "no such block shape");
    if (threads) *threads = kShapes[index].threads;
    if (width) *width = kShapes[index].width;
    if (blocks_per_sm) *blocks_per_sm = kShapes[index].minb;
    return EK_OK;
}

int ek_batch_shape(const ek_batch *b, int32_t *out) {
    if (!b || !out) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *out = b->shape;
    return EK_OK;
}

int ek_batch_set_shape(ek_batch *b, int32_t index) {
    if (!b || index < 0 || index >= EK_BATCH_SHAPES) return ek::ctx_fail(EK_ERR_INVALID, "no such block shape");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    return build_tiles(b, index);
}

int ek_batch_stream(const ek_batch *b, void **out) {
    if (!b || !out) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    *out = (void *)b->stream;
    return EK_OK;
}

// The batch adopts its channels' current states (set through their own
// handles, e.g. by ek_tile_x): same parity and state flags for all, step
// counts taken from the channels, tables rebuilt.
int ek_batch_resync(ek_batch *b) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    const ek_ctx *c0 = b->ch[0];
    for (const ek_ctx *c : b->ch) {
        if (!c->initialised) return ek::ctx_fail(EK_ERR_INVALID, "call ek_batch_init_equilibrium first");
        if (c->cur != c0->cur || c->state_pre != c0->state_pre || c->explicit_e_once != c0->explicit_e_once)
            return ek::ctx_fail(EK_ERR_INVALID, "the channels are not at one step parity and state");
    }
    b->cur = c0->cur;
    b->state_pre = c0->state_pre;
    b->explicit_e_once = c0->explicit_e_once;
    for (size_t i = 0; i < b->ch.size(); ++i) b->ch_steps[i] = b->ch[i]->steps;
    int rc = build_tables(b);  // reference rows and exponents may have changed
    if (rc == EK_OK) rc = build_tiles(b, b->shape);
    return rc;
}

// Channels with mask[i] == 0 stop stepping and keep their state (and step
// count); mask[i] != 0 steps them again, which needs their state in the
// batch's current buffer parity (an even number of batch steps since they
// were frozen).  Launches per step stay the same; the work shrinks to the
// active channels.
int ek_batch_restart(ek_batch *b, const uint8_t *mask) {
    if (!b || !mask) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    bool any = false;
    for (size_t i = 0; i < b->ch.size(); ++i) {
        if (!mask[i]) continue;
        ek_ctx *c = b->ch[i];
        if (!c->initialised) return ek::ctx_fail(EK_ERR_INVALID, "call ek_batch_init_equilibrium first");
        // equilibrium populations of the channel's loaded fields, written to
        // the buffer the batch steps from next; that step pulls them
        c->cur = b->cur;
        const int rc = ek_init_equilibrium(c);
        if (rc != EK_OK) return rc;
        EK_BCUDA(cudaStreamSynchronize(c->stream), "restart sync");
        c->state_pre = b->state_pre;
        c->explicit_e_once = b->explicit_e_once;
        b->ch_steps[i] = 0;
        c->steps = 0;
        b->active[i] = 1;
        any = true;
    }
    if (!any) return EK_OK;
    int rc = build_tables(b);  // reference rows and exponents of the restarted channels changed
    if (rc == EK_OK) rc = build_tiles(b, b->shape);
    return rc;
}

int ek_batch_set_active(ek_batch *b, const uint8_t *mask) {
    if (!b || !mask) return ek::ctx_fail(EK_ERR_INVALID, "null argument");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "batch sync");
    for (size_t i = 0; i < b->ch.size(); ++i)
        if (mask[i] && !b->active[i] && b->ch[i]->cur != b->cur)
            return ek::ctx_fail(EK_ERR_INVALID, "a frozen channel can rejoin only after an even number of batch steps");
    bool changed = false;
    for (size_t i = 0; i < b->ch.size(); ++i) {
        const char a = mask[i] ? 1 : 0;
        changed = changed || a != b->active[i];
        b->active[i] = a;
    }
    if (!changed) return EK_OK;
    int rc = build_tables(b);
    if (rc == EK_OK) rc = build_tiles(b, b->shape);
    return rc;
}

int ek_batch_active(const ek_batch *b, uint8_t *mask, int64_t *active_nodes) {
    if (!b) return ek::ctx_fail(EK_ERR_INVALID, "null batch");
    int64_t n = 0;
    for (size_t i = 0; i < b->ch.size(); ++i) {
        if (mask) mask[i] = (uint8_t)b->active[i];
        if (b->active[i]) n += (int64_t)b->ch[i]->p.nx * b->ch[i]->p.ny;
    }
    if (active_nodes) *active_nodes = n;
    return EK_OK;
}

// Residuals of every channel (as ek_residual, one snapshot per channel):
// out5 gets 5 values per channel, worst5 (optional) the maxima over channels.
int ek_batch_residual(ek_batch *b, int32_t interval, double *out5, double *worst5) {
    if (!b || !out5 || interval <= 0) return ek::ctx_fail(EK_ERR_INVALID, "bad residual arguments");
    const int nch = (int)b->ch.size();
    double *sums = b->d_rpart + (size_t)b->nrpart * 8;
    EK_BCUDA(launch_batch_residual(b->d_chan, b->d_fields, b->d_snaps, b->d_ritems, b->nritems, b->d_rranges, nch,
                                   b->d_rpart, sums, b->stream),
             "batch residual");
    b->launches += 2;
    std::vector<double> h((size_t)nch * 8);
    EK_BCUDA(cudaMemcpyAsync(h.data(), sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream),
             "residual copy");
    EK_BCUDA(cudaStreamSynchronize(b->stream), "residual sync");
    double w[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < nch; ++i) {
        double *o = out5 + (size_t)i * 5;
        const double *sums = &h[(size_t)i * 8];
        if (!std::all_of(sums, sums + 8, [](double v) { return std::isfinite(v); })) {
            // a diverged channel: NaN residuals, the others carry on
            std::fill(o, o + 5, std::nan(""));
            b->ch[i]->snap_valid = false;
            continue;
        }
        const int rc = ek::ctx_residual_finish(b->ch[i], sums, interval, o);
        if (rc != EK_OK) return rc;
        for (int k = 0; k < 5; ++k) w[k] = std::max(w[k], o[k]);
    }
    if (worst5)
        for (int k = 0; k < 5; ++k) worst5[k] = w[k];
    return EK_OK;
}

// Time each block shape for `steps` steps (the state advances by
// EK_BATCH_SHAPES (steps + 2) steps) and keep the fastest; ms (optional) gets
// the ms per step of every shape.
int ek_batch_autotune(ek_batch *b, int32_t steps, int32_t *chosen, double *ms) {
    if (!b || steps <= 0) return ek::ctx_fail(EK_ERR_INVALID, "bad autotune arguments");
    int rc = check_channels(b);
    if (rc != EK_OK) return rc;
    double best = 1e300;
    int best_w = b->shape;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    EK_BCUDA(cudaEventCreate(&e0), "event");
    EK_BCUDA(cudaEventCreate(&e1), "event");
    const bool saved_graph = b->use_graph;
    b->use_graph = false;  // time the kernels, not a graph captured for one width
    for (int k = 0; k < EK_BATCH_SHAPES && rc == EK_OK; ++k) {
        rc = build_tiles(b, k);
        if (rc == EK_OK) rc = ek_batch_step(b, 2);  // warm-up
        if (rc != EK_OK) break;
        cudaEventRecord(e0, b->stream);
        rc = ek_batch_step(b, steps);
        if (rc != EK_OK) break;
        cudaEventRecord(e1, b->stream);
        const cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            rc = cuda_err(e, "autotune");
            break;
        }
        float elapsed = 0.0f;
        cudaEventElapsedTime(&elapsed, e0, e1);
        const double per = elapsed / steps;
        if (ms) ms[k] = per;
        if (per < best) {
            best = per;
            best_w = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->use_graph = saved_graph;
    if (rc != EK_OK) return rc;
    rc = build_tiles(b, best_w);
    if (rc != EK_OK) return rc;
    if (chosen) *chosen = best_w;
    return EK_OK;
}

}  // extern "C"
