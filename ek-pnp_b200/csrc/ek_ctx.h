// ek_ctx.h -- the channel context behind the C ABI's ek_ctx handle (host
// side; shared by ek_api.cu and the batched solver in ek_batch.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "ek_internal.h"

struct ek_ctx {
    ek_params p{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nxp = 0, mp = 0, n = 0;
    size_t plane = 0;
    void *pops[2] = {nullptr, nullptr};
    int cur = 0;
    bool initialised = false;  // populations exist
    bool state_pre = false;    // pops[cur] holds pre-collision populations in place
    bool explicit_e_once = false;
    bool e_stale = false;      // E planes older than psi
    bool split_stale = false;  // shifted storage: psif/psim older than the FP64 psi plane
    double *fields = nullptr;
    double *wall = nullptr;    // 6 x nx
    std::vector<double> wall_host;  // host copy of the wall profiles
    double *snap = nullptr;    // residual snapshot, 4 planes
    double *part = nullptr;    // residual partial sums
    bool snap_valid = false;
    float *kref[2] = {nullptr, nullptr};  // shifted storage: row references /36, double-buffered
    float *kwall = nullptr;               // shifted storage: wall ions' per-x frames (ChanF::kwall)
    float *wdelta = nullptr;              // and half their defect (ChanF::wdelta)
    float *lift = nullptr;                // shifted storage: the wall lifting's x-fluctuation (Chan::lift)
    int kcur = 0;
    int kq[3] = {0, 0, 0};                // binary exponents of the reference grids
    int32_t rebase_every = 0;
    CUtensorMap tmaps[2];                 // shifted storage: TMA descriptors of pops[0], pops[1]
    bool tma_ok = false;
    int lbm_kernel = 0;                   // EK_OPT_LBM_KERNEL
    int poisson_mode = 0;                 // EK_OPT_POISSON
    bool last_moments = true;             // EK_OPT_LAST_STEP_MOMENTS
    long long wait_cycles = 1ll << 31;    // EK_OPT_WAIT_CYCLES
    bool keep_l2 = false;                 // rhs + psi planes fit the L2 share kept for them
    int *err_dev = nullptr;               // set by bounded device waits
    unsigned long long *jacobi_word = nullptr;  // ek_poisson_jacobi: largest change of a sweep
    ek::Rates *rates_dev = nullptr;
    ek::Rates rates{};
    ek::PoissonPlan pp{};
    ek::Chan chan{};
    int64_t steps = 0;
    int64_t launches = 0;
    // profiling
    bool prof = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    std::vector<int> ev_phase;
    size_t ev_used = 0;
    cudaEvent_t marks[16] = {};
};

// Shared with ek_batch.cu (defined in ek_api.cu).
namespace ek {
int ctx_fail(int code, const char *msg);
int ctx_refs_from_fields(ek_ctx *c, float *out);
void ctx_refresh(ek_ctx *c);
int ctx_residual_buffers(ek_ctx *c);
int ctx_residual_finish(ek_ctx *c, const double *sums, int32_t interval, double *out5);
bool ctx_poisson_f32(const ek_ctx *c);  // the FP32 form runs for this context
// After psi was set on the device outside a step (a grid relaxation): the E
// planes from psi, and the FP32 planes of shifted storage marked stale.
int ctx_after_psi(ek_ctx *c);
}  // namespace ek
