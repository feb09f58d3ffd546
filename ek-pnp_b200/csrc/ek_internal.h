// ek_internal.h -- shared definitions of libekpnp's kernels and C ABI.
//
// Device memory of one channel (all planes ny rows x nxp columns, nxp = nx
// rounded up to 32 so every row starts 256-byte aligned):
//   pops[2]   27 planes each, ping-pong: species-major (fluid f, c+ h, c- t),
//             then direction 0..8 in the reference numbering (LBM.cu:831-834).
//             Between steps a buffer holds POST-collision populations; the next
//             step pulls them (streaming fused into the load).  Right after
//             ek_init_equilibrium it holds pre-collision populations at their
//             own node ("state_pre"), and the first step reads them in place.
//   fields    9 planes: rho, ux, uy, c+, c-, psi, Ex, Ey, and the Poisson
//             right-hand side.
//   spec      (ny-2) x mp complex: x-spectrum of the interior rows (mp >= nx/2+1)
//   piv       (ny-2) x mp: pivots of the per-mode tridiagonal y-solve
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/ekpnp.h"

namespace ek {

// Programmatic dependent launch.  A kernel started by launch_pdl may be
// scheduled while the kernel before it in the stream is still draining; its
// first statement is pdl_wait(), which waits for that kernel's completion
// and the visibility of its writes, then lets the next kernel be scheduled
// in turn.  A kernel launched the ordinary way passes pdl_wait() at once.
// Used for a channel's one-wave row transform after the LBM step (measured
// at 4096 x 1024: -2.6 us a step); on the many-wave LBM kernel the per-block
// wait cost ~40 us a step, and next to the column pass's fork/join events it
// cost more than it saved (the batched passes run many waves: not used there).
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Field-plane bytes (right-hand side + psi of every channel stepped together)
// that the evict_last stores may pin, out of the 126 MB L2: above it the
// planes are stored the ordinary way.
constexpr size_t KEEP_L2_BYTES = (size_t)80 << 20;
inline bool keep_l2_fits(size_t bytes) { return bytes <= KEEP_L2_BYTES; }

// Stores of field planes that the next kernel reads back (the Poisson
// right-hand side written by the LBM step, psi written by the inverse row
// pass): with keep set they carry an L2 evict_last policy, so the plane
// stays in L2 while the step's populations stream through it.
__device__ __forceinline__ void st_field(double *p, double v, bool keep) {
#if defined(__CUDA_ARCH__)
    if (keep) {
        unsigned long long pol;
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
        return;
    }
#endif
    *p = v;
}

__device__ __forceinline__ void st_field_f(float *p, float v, bool keep) {
#if defined(__CUDA_ARCH__)
    if (keep) {
        unsigned long long pol;
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
        return;
    }
#endif
    *p = v;
}

template <typename... Exp, typename... Act>
cudaError_t launch_pdl(void (*kern)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Act &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Act>(args)...);
}

// D2Q9 velocity set in the reference numbering:  6 2 5 / 3 0 1 / 7 4 8
__host__ __device__ constexpr int cxd(int d) {
    return d == 1 || d == 5 || d == 8 ? 1 : (d == 3 || d == 6 || d == 7 ? -1 : 0);
}
__host__ __device__ constexpr int cyd(int d) {
    return d == 2 || d == 5 || d == 6 ? 1 : (d == 4 || d == 7 || d == 8 ? -1 : 0);
}
__host__ __device__ constexpr int oppd(int d) { return d == 0 ? 0 : (d <= 4 ? (d + 1) % 4 + 1 : (d - 3) % 4 + 5); }
static_assert(oppd(1) == 3 && oppd(2) == 4 && oppd(3) == 1 && oppd(4) == 2, "opp straight");
static_assert(oppd(5) == 7 && oppd(6) == 8 && oppd(7) == 5 && oppd(8) == 6, "opp diagonal");

constexpr double W0 = 4.0 / 9.0, WS = 1.0 / 9.0, WD = 1.0 / 36.0;  // LBM.h:105-107

// Relaxation and wall constants, evaluated on the device with the reference's
// expressions (LBM.cu:336-341, 745-746, 812-813) so they round as it does.
struct Rates {
    double wp, wm;    // fluid omega+*dt, omega-*dt
    double wcp, wcm;  // c+  (minus set by diffu, plus by VC)
    double wtp, wtm;  // c-  (minus set by D, plus by VT)
    double sp, sm;    // Guo source factors 1 - dt*omega/2
    double ms, md;    // moving top wall terms
};

// Per-channel constants, passed by value to every kernel.
struct Chan {
    int nx, ny, nxp, flags;
    size_t plane;  // ny * nxp
    double dx, dy, dt, cfl, cs2, rho0, c0;
    double mob_p, mob_n, f_charge, eps, ext_x, exf;
    Rates r;
    const double *zlo, *zhi, *cplo, *cphi, *cnlo, *cnhi;  // per-x wall values (nx each)
    // Shifted storage only: per-row reference densities divided by 36, three
    // rows of ny floats (fluid, c+, c-).  A population of species s stored at
    // row y holds f - w_i * 36 * kref[s*ny + y]; every kref value is a
    // multiple of 2^-q, so 36 w_i (kref[y'] - kref[y]) is exact in FP32.
    const float *kref;
    // Shifted storage only: per-x ion frames of the wall nodes (/36), per
    // population buffer, and half their defect (see ChanF::kwall).
    const float *kwall;
    const float *wdelta;
    // Shifted storage only: the step's field planes (PoissonPlan::rhsf, psif, psim),
    // and the x-fluctuation of the wall lifting, (zeta(x) - zeta_mean)/dy^2,
    // lower wall then upper (2 nx floats), which rows 1 and ny-2 subtract
    // from rhsf.
    float *rhsf;
    const float *psif;
    const double *psim;
    const float *lift;
    int keep_l2;   // right-hand side and psi planes held in L2 between kernels
};

enum Field { F_RHO = 0, F_UX, F_UY, F_CP, F_CN, F_PSI, F_EX, F_EY, F_RHS, F_COUNT };

// ---- launchers (ek_lbm_f64.cu) ----
cudaError_t launch_rates(const ek_params &p, Rates *dev_out, cudaStream_t s);
cudaError_t launch_init_f64(const Chan &c, double *pops, const double *fields, bool explicit_e,
                            cudaStream_t s);
cudaError_t launch_step_f64(const Chan &c, const double *src, double *dst, double *fields,
                            bool first, bool explicit_e, bool moments, cudaStream_t s);
cudaError_t launch_efield_f64(const Chan &c, double *fields, cudaStream_t s);
cudaError_t launch_rhs_from_moments_f64(const Chan &c, double *fields, cudaStream_t s);

// ---- Poisson-Boltzmann start (ek_init.cu) ----
cudaError_t launch_pb_fill(const Chan &c, double *fields, double *psi_old, cudaStream_t s);
cudaError_t launch_pb_conc(const Chan &c, double e_kt, double *fields, cudaStream_t s);
cudaError_t launch_pb_relax(const Chan &c, double omega, double *fields, double *psi_old, cudaStream_t s);
// Newton Poisson-Boltzmann start: ncol columns (walls[q] = {zeta_lo, zeta_hi})
// solved on the device (psi, cp, dp: ny x ncol scratch, ok: ncol flags), then
// the fields of every node from its column colmap[x].
cudaError_t launch_pb_newton(const Chan &c, double dy, double g, double a, const double2 *walls, int ncol,
                             double *psi, double *cp, double *dp, int *ok, const int *colmap, double *fields,
                             cudaStream_t s);

// ---- shifted-storage forms (ek_lbm_f32.cu); storage = EK_STORE_F32 or _F16 ----
// sbuf: index (0/1) of the population buffer that src is (it names the wall
// ions' frames); buf: the buffer that pops is.
cudaError_t launch_step_shifted(const Chan &c, int storage, const void *src, void *dst, double *fields,
                                bool first, bool explicit_e, bool moments, int sbuf, cudaStream_t s);
cudaError_t launch_init_shifted(const Chan &c, int storage, void *pops, const double *fields, bool explicit_e,
                                int buf, cudaStream_t s);
// Wall frames of the ions from the fields' wall rows (initialisation; buf is
// the buffer the initial populations go to), and their defect after the wall
// concentrations change.
cudaError_t launch_wall_frames(const Chan &c, const double *fields, int qp, int qn, int buf, float *kwall,
                               float *wdelta, cudaStream_t s);
cudaError_t launch_wall_delta(const Chan &c, const float *kwall, float *wdelta, cudaStream_t s);
// Row means of rho, c+, c- rounded to the grid K 2^-q, stored /36 in
// kout[3*ny] (ek_lbm_f32.cu); q per species.
cudaError_t launch_row_refs(const Chan &c, const double *fields, int qf, int qp, int qn, float *kout,
                            cudaStream_t s);
// Re-express stored shifted populations against a new reference profile.
cudaError_t launch_rebase(const Chan &c, int storage, void *pops, const float *kold, const float *knew,
                          cudaStream_t s);
// ---- TMA-fed persistent form of the shifted step (ek_lbm_tma.cu) ----
// map_out: a 128-byte CUtensorMap (64-byte aligned) over one population buffer.
cudaError_t make_pop_tensor_map(int storage, const void *pops, int nxp, int ny, void *map_out);
cudaError_t launch_step_tma(const Chan &c, int storage, const void *map, const void *src, void *dst, double *fields,
                            bool first, bool explicit_e, bool moments, int sbuf, int *err, long long wait_cycles,
                            cudaStream_t s);
inline size_t pop_elem_bytes(int storage) { return storage == EK_STORE_F64 ? 8 : (storage == EK_STORE_F32 ? 4 : 2); }

// ---- Poisson (ek_poisson.cu) ----
struct PoissonPlan {
    int nx, ny, n, mp, log2nx;  // n = ny-2 interior rows
    bool pow2;
    double dy2;                 // dy*dy
    double2 *tw;                // nx twiddles exp(-2 pi i k/nx)
    double *piv;                // n x mp pivots
    double2 *spec;              // n x mp spectrum
    // FP32 form (shifted storage): modes >= 1 in FP32, the zero mode in FP64
    // (column 0 of spec); null where the form is not set up
    float2 *twf;                // FP32 row transforms: per-pass twiddle tables (< nx entries)
    float *pivf;                // n x mp pivots, FP32
    float2 *specf;              // n x mp spectrum, FP32
    double *rowmean;            // n row means of the last solve: the offset removed before the FP32 FFT
    int *rowmean_ok;            // set by the first solve's pass C; before it pass A takes exact means
    // Field planes of the shifted-storage step (every shifted context; the
    // FP32 form reads and writes them directly, the FP64 form through
    // compose/split kernels):
    //   rhsf  (ny x nxp) FP32: the right-hand side minus its row constant,
    //         rhs_q (c+ - c- - (R+ - R-)); the constant rhs_q (R+ - R-) of the
    //         row references and the wall lifting are added in FP64 by pass A
    //   psif  (ny x nxp) FP32: psi minus its row mean
    //   psim  (ny) FP64: the row means of psi (the zero mode, walls included)
    float *rhsf;
    float *psif;
    double *psim;
    double zlo_mean, zhi_mean;  // x-means of the wall potentials (psim of the wall rows)
    int keep_l2;                // psi stores ask L2 to keep the plane (see st_field)
};
// pass 0: row FFTs, 1: tridiagonal column solve, 2: inverse row FFTs + walls
cudaError_t poisson_pass_f64(int pass, const PoissonPlan &pp, const Chan &c, double *fields, cudaStream_t s);
// Same passes with the right-hand side and psi planes given directly.
cudaError_t poisson_pass_f64_at(int pass, const PoissonPlan &pp, const Chan &c, const double *rhs, double *psi,
                                cudaStream_t s);
size_t poisson_smem_bytes_f64(int nx);
// FP32 form of the passes (power-of-two nx >= 16, n <= 8192, twf/pivf/specf
// set): the row FFTs and the column solves of the modes >= 1 in FP32 on the
// fluctuation about each row's mean; the row sums (the zero mode), its
// column solve and the mean of psi in FP64.
bool poisson_f32_supported(const PoissonPlan &pp);
// Passes 0 and 2 (pass 1 is poisson_tridiag_f32): pass 0 reads
// pp.rhsf with the row constants of c.kref and the wall lifting; pass 2 writes
// pp.psif and pp.psim, and the FP64 psi plane too when write_f64.
cudaError_t poisson_pass_f32(int pass, const PoissonPlan &pp, const Chan &c, double *psi, bool write_f64,
                             cudaStream_t s);
// Shifted storage with the FP64 passes: the FP64 right-hand side from rhsf
// (before pass 0), and psif/psim from the FP64 psi (after pass 2, and
// whenever psi was set from outside).
cudaError_t launch_compose_rhs(const PoissonPlan &pp, const Chan &c, double *rhs, cudaStream_t s);
// The FP64 row constant of the right-hand side of row y (1 <= y <= ny-2):
// rhs_q (R+ - R-) of the row references, minus zeta_mean/dy^2 on rows 1 and
// ny-2 (the x-mean of the wall lifting; its fluctuation is Chan::lift).
__host__ __device__ inline double rhs_row_constant(const PoissonPlan &pp, const Chan &c, int y) {
    const double rq = -c.f_charge / c.eps, inv_dy2 = 1.0 / (c.dy * c.dy);
    double v = rq * (36.0 * (double)c.kref[c.ny + y] - 36.0 * (double)c.kref[2 * c.ny + y]);
    if (y == 1) v -= pp.zlo_mean * inv_dy2;
    if (y == c.ny - 2) v -= pp.zhi_mean * inv_dy2;
    return v;
}
cudaError_t launch_split_psi(const PoissonPlan &pp, const Chan &c, const double *psi, cudaStream_t s);
// rhsf from the c+, c- moments (a solve outside the step, FP32 form).
cudaError_t launch_rhsf_from_moments(const PoissonPlan &pp, const Chan &c, const double *fields, cudaStream_t s);
// Pass B of the FP32 form, one kernel: the FP64 zero mode in its first
// block, the FP32 modes in the others.  Batched: items int3 {channel, first
// mode, modes per block}, modes per block 0 naming a channel's zero mode.
cudaError_t poisson_tridiag_f32(const PoissonPlan &pp, cudaStream_t s);
cudaError_t batch_tridiag_f32(const PoissonPlan *plans, const void *items, int nitems, cudaStream_t s);
// Batched Poisson passes of the FP32 form over many channels (ek_batch.cu
// builds the items): pass 0/2 items int2 {channel, first row pair}
// (256-thread blocks, each 256/(nx/16) row pairs; power-of-two nx from 16 to
// 4096); pass 1 is batch_tridiag_f32.  write_f64 as poisson_pass_f32.
cudaError_t batch_poisson(int pass, const PoissonPlan *plans, const Chan *chans, double *const *fields,
                          const void *items, int nitems, bool write_f64, cudaStream_t s);
int poisson_tridiag_modes(int n);
// Steady-state residual sums (ek_residual.cu): per channel 8 FP64 sums,
// (q - q_snap)^2 then q^2 for q in (ux, c+, c-, psi); the snapshot is updated.
cudaError_t launch_residual_f64(const Chan &c, const double *fields, double *snap, double *part,
                                int nblocks, double *out8, cudaStream_t s);
int residual_blocks(const Chan &c);
// Many channels: items int4 {channel, block, blocks of the channel, first
// partial}, ranges int2 {first partial, blocks} per channel, out8 8 per channel.
cudaError_t launch_batch_residual(const Chan *chans, double *const *fields, double *const *snaps, const int4 *items,
                                  int nitems, const int2 *ranges, int nch, double *part, double *out8,
                                  cudaStream_t s);
// Record an error message for ek_last_error() (ek_api.cu).
void set_last_error(const char *msg);
cudaError_t poisson_set_smem_limits();

}  // namespace ek
