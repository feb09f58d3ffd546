/*
 * ekpnp.h -- C ABI of the B200 EK-PNP channel solver (libekpnp.so).
 *
 * One solver context ("channel") holds a 2D channel of nx*ny lattice nodes,
 * periodic in x, with walls at y = 0 and y = ny-1.  Each time step is the
 * coupled update of the reference code (gyf135/EK-PNP):
 *   - TRT D2Q9 fluid with Guo forcing by the electric body force,
 *   - TRT D2Q9 Nernst-Planck populations for c+ and c-,
 *   - wall boundary conditions (fluid full-way bounce-back, ion Dirichlet
 *     anti-bounce-back),
 *   - spectral Poisson solve for the potential psi and the field E = -grad psi.
 *
 * Every entry point returns an int status (EK_OK = 0, see ek_status_string)
 * instead of calling exit() as the reference does (LBM.cu:44-62, LBM.h:182-203).
 * All field arrays are row-major nx*ny doubles, index = nx*y + x, the
 * reference's scalar_index (LBM.h:172-175).  Pointers are host pointers unless
 * the call says otherwise.  No torch or CUDA types appear in the signatures;
 * streams are passed as void* (a cudaStream_t).
 */
#ifndef EKPNP_H
#define EKPNP_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
    EK_OK = 0,
    EK_ERR_INVALID = 1,     /* bad argument or parameter (rejected on the host) */
    EK_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    EK_ERR_NOMEM = 3,       /* device allocation failed */
    EK_ERR_NAN = 4,         /* non-finite value found by a residual/health reduction */
    EK_ERR_TIMEOUT = 5,     /* a bounded device wait gave up (batched work queue) */
    EK_ERR_UNSUPPORTED = 6, /* configuration outside what this build supports */
    EK_ERR_TOO_LARGE = 7    /* size above the documented maximum of the call */
};

/* ---- population storage ---------------------------------------------- */
enum {
    EK_STORE_F64 = 0,       /* FP64 populations, reference arithmetic order      */
    EK_STORE_F32 = 1,       /* FP32 deviations f - w_i*rho0, h - w_i*c0          */
    EK_STORE_F16 = 2        /* FP16 deviations, FP32 arithmetic                  */
};

/* ---- behaviour flags (ek_params.flags) --------------------------------- */
enum {
    /* Electric body force on the fluid, F = f_charge*(c+ - c-)*(E + ext_x) + exf.
     * The reference ships it commented out (LBM.cu:388-389, 438-439); set this
     * to run the driven flow the commented expression describes. */
    EK_FLAG_FORCE = 1 << 0,
    /* Negative-ion rest equilibrium uses the fluid's 1 - u^2/(2cs^2) instead
     * of the c- drift velocity, as gpu_collide_save does (LBM.cu:493).  Off
     * gives the consistent form used by gpu_init_equilibrium (LBM.cu:242). */
    EK_FLAG_REST_QUIRK = 1 << 1,
    /* Write rho, ux, uy, c+, c- of every step to the context's field buffers
     * (the reference writes them every step, LBM.cu:447-451).  Without it they
     * are written only on the steps that need them (residual, ek_get_fields). */
    EK_FLAG_MOMENTS_EVERY_STEP = 1 << 2,
    /* Keep explicit Ex/Ey arrays written by the Poisson step and read by the
     * collision (reference data flow, poisson.cu:132-174).  Without it the
     * collision differentiates psi itself with the same stencil. */
    EK_FLAG_EXPLICIT_E = 1 << 3
};

/* Physical and numerical constants of one channel.  Names follow the
 * reference's LBM.h symbols (cited per field); any consistent unit system
 * works, lattice units being dx = dy = dt = cfl = 1, cs2 = 1/3. */
typedef struct ek_params {
    int32_t nx;          /* NX (LBM.h:35); x is periodic                       */
    int32_t ny;          /* NY (LBM.h:36); walls at y = 0 and ny-1, ny >= 4    */
    int32_t storage;     /* EK_STORE_*                                         */
    int32_t flags;       /* EK_FLAG_*                                          */
    double dx, dy;       /* dx, dy (LBM.h:42-43)                               */
    double dt;           /* dt (LBM.h:51)                                      */
    double cfl;          /* CFL = dt/dx (LBM.h:50)                             */
    double cs2;          /* cs_square (LBM.h:52)                               */
    double lx;           /* Lx, x period of the spectral symbol (LBM.h:40)     */
    double rho0;         /* rho0 (LBM.h:53); fluid shift of the FP32/16 forms  */
    double c0;           /* bulk concentration; ion shift of the FP32/16 forms */
    double nu;           /* nu (LBM.h:65-66)                                   */
    double magic_f;      /* V, fluid TRT magic parameter (LBM.h:110)           */
    double diff_p;       /* diffu, c+ diffusivity (LBM.h:64)                   */
    double magic_p;      /* VC (LBM.h:111)                                     */
    double mob_p;        /* K, c+ mobility (LBM.h:67-68)                       */
    double diff_n;       /* D, c- diffusivity (LBM.h:71-72)                    */
    double magic_n;      /* VT (LBM.h:112)                                     */
    double mob_n;        /* Kn, c- mobility (LBM.h:74-75)                      */
    double eps;          /* eps, permittivity (LBM.h:63)                       */
    double f_charge;     /* convertCtoCharge (LBM.h:90)                        */
    double zeta_lo;      /* voltage, wall potential at y = 0 (LBM.h:58)        */
    double zeta_hi;      /* voltage2, wall potential at y = ny-1 (LBM.h:60)    */
    double cp_lo, cp_hi; /* charge0, charge1: c+ at the walls (LBM.h:55-56)    */
    double cn_lo, cn_hi; /* charge0n, charge1n: c- at the walls (LBM.h:81-83)  */
    double ext_x;        /* Ext, applied field along x (LBM.h:62)              */
    double exf;          /* exf, extra body force along x (LBM.h:47-49)        */
    double uw;           /* uw, top wall velocity (LBM.h:46-48)                */
} ek_params;

typedef struct ek_ctx ek_ctx;

/* Library version (major*10000 + minor*100 + patch). */
int ek_version(void);
const char *ek_status_string(int status);
/* Message of the last failing call on this host thread ("" if none). */
const char *ek_last_error(void);

/* Fill *p with lattice-unit defaults (dx=dy=dt=cfl=1, cs2=1/3, nu=1/6,
 * magic 1/4, FP64 storage, force and rest quirk on).  nx, ny are set. */
int ek_params_default(ek_params *p, int32_t nx, int32_t ny);

/* Make `device` the current CUDA device of this library on the calling host
 * thread (the library carries its own CUDA runtime state, so a device chosen
 * through another runtime instance, e.g. a Python framework's, does not apply). */
int ek_set_device(int32_t device);
int ek_get_device_count(int32_t *out);

/* Create a context on the current CUDA device.  Replaces the allocation and
 * set-up block of main.cu:89-142 (population and field buffers, cuFFT plan,
 * wavenumber tables).  Rejects invalid parameters with EK_ERR_INVALID. */
int ek_create(const ek_params *p, ek_ctx **out);
int ek_destroy(ek_ctx *ctx);
/* Run all later work of ctx on this stream (a cudaStream_t; NULL = legacy). */
int ek_set_stream(ek_ctx *ctx, void *stream);
int ek_get_params(const ek_ctx *ctx, ek_params *out);

/* Load macroscopic fields (host pointers, nx*ny doubles each).  ex/ey may be
 * NULL: the field is then taken from psi.  Mirrors read_data (LBM.cu:1350-1391)
 * minus the file parsing. */
int ek_set_fields(ek_ctx *ctx, const double *rho, const double *ux,
                  const double *uy, const double *cp, const double *cn,
                  const double *psi, const double *ex, const double *ey);
/* Same as ek_set_fields from device buffers of nx*ny doubles (index nx*y + x),
 * e.g. the caller's own rho_gpu, charge_gpu, ... of main.cu:102-110. */
int ek_set_fields_device(ek_ctx *ctx, const double *rho, const double *ux,
                         const double *uy, const double *cp, const double *cn,
                         const double *psi, const double *ex, const double *ey);

/* Per-x wall potential and wall concentrations (nx doubles each, any may be
 * NULL to keep the uniform value).  Extends the uniform voltage/charge0
 * constants of LBM.h:55-83 to a wall zeta that varies along x. */
int ek_set_wall_profile(ek_ctx *ctx, const double *zeta_lo, const double *zeta_hi,
                        const double *cp_lo, const double *cp_hi,
                        const double *cn_lo, const double *cn_hi);

/* Poisson-Boltzmann start: sets rho = rho0, u = 0, c+- = c0 exp(-+ e_kt psi)
 * and psi (E follows from psi).  e_kt is e/kT in the units of psi (1 when psi
 * is in thermal volts).
 *   method EK_PB_REFERENCE: the reference's own start (initialization,
 *     LBM.cu:95-145): psi = zeta_lo everywhere, then `iterations` rounds of
 *     {c+- from psi, Poisson solve, psi = omega psi + (1-omega) psi_old}.  It
 *     converges only for weak coupling (roughly kappa*H below 10 at |zeta| = 2).
 *   method EK_PB_NEWTON: damped Newton iteration of the discrete 1D
 *     Poisson-Boltzmann equation down every x-column (rows 1..ny-2, Dirichlet
 *     wall values), iterations/omega ignored, on the device (one thread per
 *     distinct pair of wall potentials, 3 ny doubles of scratch each).  Exact
 *     for walls uniform in x, the column-local solution otherwise.
 * Follow with ek_init_equilibrium (optionally after perturbing the fields). */
enum { EK_PB_REFERENCE = 0, EK_PB_NEWTON = 1 };
int ek_init_poisson_boltzmann(ek_ctx *ctx, int32_t method, int32_t iterations,
                              double omega, double e_kt);

/* Populations at equilibrium with the loaded fields: init_equilibrium /
 * gpu_init_equilibrium (LBM.cu:183-305). */
int ek_init_equilibrium(ek_ctx *ctx);

/* Copy the state of src into dst repeated along x: populations, fields,
 * shifted-storage reference rows and the FP32 Poisson form's row offsets.
 * Needs the same ny and storage and dst's nx a multiple of src's.  With
 * walls uniform along x a channel's steady state does not depend on x, so a
 * narrow channel relaxed to it starts a wide one there (the reference only
 * restarts a channel of the same size, from data_end.dat).  dst keeps its
 * step count and parameters. */
int ek_tile_x(ek_ctx *dst, const ek_ctx *src);

/* Advance nsteps coupled steps.  One step = stream_collide_save
 * (LBM.cu:307-329: collide, fluid walls, stream, ion walls) followed by
 * fast_Poisson (poisson.cu:180-208), fused as one pull-scheme LBM kernel plus
 * a three-pass Poisson solve. */
int ek_step(ek_ctx *ctx, int32_t nsteps);

/* Shifted storage (FP32/FP16) keeps each population as a deviation from a
 * per-row reference density (fluid, c+, c-) set from the fields' row means by
 * ek_init_equilibrium.  ek_rebase re-derives the references from the moments
 * of the last step and re-expresses the stored populations against them
 * (exactly); ek_set_rebase_interval(ctx, n) does that every n steps inside
 * ek_step (0 = never, the default).  No effect in FP64. */
int ek_rebase(ek_ctx *ctx);
int ek_set_rebase_interval(ek_ctx *ctx, int32_t steps);

/* Tuning options (ek_set_option).  EK_OPT_LBM_KERNEL selects the form of the
 * shifted-storage LBM kernel: 0 = automatic (currently the plain form, the
 * faster one on B200), 1 = plain per-node loads, 2 = TMA-fed pipeline
 * (producer warp + mbarrier ring of tensor copies).  Both forms give
 * bit-identical results.
 * Returns EK_ERR_UNSUPPORTED for a form that this context cannot run. */
enum { EK_OPT_LBM_KERNEL = 1, EK_OPT_POISSON = 2, EK_OPT_LAST_STEP_MOMENTS = 3, EK_OPT_WAIT_CYCLES = 4 };
/* EK_OPT_POISSON selects the arithmetic of the Poisson solve (ek_step and
 * ek_poisson): 0 = automatic (the FP32 form for FP32/FP16 storage where it
 * applies, FP64 otherwise), 1 = FP64, 2 = FP32 form: row FFTs and column
 * solves of the x-modes >= 1 in FP32 on the fluctuation about each row's
 * mean, the zero mode (row sums, its column solve, the mean of psi) in FP64.
 * The FP32 form needs shifted storage, a power-of-two nx >= 16 and
 * ny <= 8194 (EK_ERR_UNSUPPORTED otherwise).
 * EK_OPT_LAST_STEP_MOMENTS: 1 (default) = the last step of every ek_step call
 * writes the moments rho, ux, uy, c+, c- to the field planes; 0 = only the
 * steps that need them anyway (re-basing, EK_FLAG_MOMENTS_EVERY_STEP) write
 * them, and the planes keep the moments of the last step that did.  psi and
 * E follow every step either way.  A caller that steps one step per call and
 * reads the moments only now and then (the reference's loop, main.cu:190-233)
 * sets 0 and switches to 1 for the steps whose moments it reads; the choice
 * never changes the arithmetic of a step.
 * EK_OPT_WAIT_CYCLES: bound, in SM clock cycles (>= 1), of each wait of the
 * TMA-fed kernel's pipeline (default 2^31, about a second).  A wait that runs
 * out sets the context's error word; the producer still waits, at the
 * default bound, for the copies it issued; the next ek_sync or
 * ek_get_fields returns EK_ERR_TIMEOUT and the context stays usable. */
int ek_set_option(ek_ctx *ctx, int32_t option, int64_t value);

/* Poisson solve for the current c+, c- moments, then psi and E:
 * fast_Poisson (poisson.cu:180-208) without its per-call cudaMalloc/Free. */
int ek_poisson(ek_ctx *ctx);

/* Grid relaxation of the same Poisson equation for the current c+, c-
 * moments: poisson_phi / gpu_poisson (poisson.cu:35-130), the reference's
 * iterative solver, which its time loop does not call.  Weighted Jacobi
 * sweeps (omega in (0, 2), 1 = the reference's update) from the current
 * psi, walls at the wall potentials, until the largest change of a sweep is
 * below tol (the reference: 1e-9) or max_sweeps (the reference: 1e6); the
 * change is measured every check_every sweeps and on the last.  Unlike the
 * reference's in-place update, every sweep reads one buffer and writes
 * another, so the result does not depend on the schedule.  The fixed point
 * is the five-point discretisation (three-point along x too), not the
 * spectral-x one of ek_poisson.  Then E from psi.  sweeps / change (optional): sweeps done and the last measured change
 * (-1 if none was measured).  Returns EK_OK whether or not tol was reached. */
int ek_poisson_jacobi(ek_ctx *ctx, int32_t max_sweeps, double tol, double omega, int32_t check_every,
                      int32_t *sweeps, double *change);

/* Copy the macroscopic fields of the last step to host arrays (any pointer may
 * be NULL).  rho, ux, uy, cp, cn are the moments of the last step's
 * pre-collision populations, psi/ex/ey the Poisson result from them, as the
 * reference's buffers hold after its loop (main.cu:190-233). */
int ek_get_fields(ek_ctx *ctx, double *rho, double *ux, double *uy, double *cp,
                  double *cn, double *psi, double *ex, double *ey);

/* Same as ek_get_fields but into device buffers of nx*ny doubles. */
int ek_get_fields_device(ek_ctx *ctx, double *rho, double *ux, double *uy,
                         double *cp, double *cn, double *psi, double *ex,
                         double *ey);

/* Steady-state residual over the last `interval` steps (new; the reference has
 * none): out[q] = ||q^n - q^{n-interval}||_2 / (interval * max(||q^n||_2, floor_q))
 * for q = ux, c+, c-, psi (FP64 reductions on the device); out[4] = max.
 * Returns EK_ERR_NAN if a field holds a non-finite value.  The first call only
 * records the snapshot and reports out[] = +inf. */
int ek_residual(ek_ctx *ctx, int32_t interval, double *out5);

/* Steps taken since ek_create / ek_init_equilibrium. */
int ek_step_count(const ek_ctx *ctx, int64_t *out);

/* Wait for the context's stream.  Returns EK_ERR_TIMEOUT if a bounded device
 * wait of a pipelined kernel gave up since the last check (the error word is
 * then cleared). */
int ek_sync(ek_ctx *ctx);

/* Device pointers of the field planes (zero-copy readers).  Order: rho, ux,
 * uy, cp, cn, psi, ex, ey; each plane has ny rows of *pitch doubles (pitch >=
 * nx), index = pitch*y + x. */
int ek_field_pointers(ek_ctx *ctx, double **out8, int32_t *pitch);

/* ---- Poisson solve without device allocation --------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory inside their time loop (the reference allocates and frees four
 * buffers in every Poisson call, poisson.cu:182-207; a host program whose
 * device memory belongs to its own pool, or is fully committed, cannot).
 * Computes psi (and, if ex/ey are given, E = -grad psi) from c+ and c- for the
 * channel described by p, exactly as ek_poisson does, with every scratch
 * buffer in device arrays built into the library (10.9 MB per GPU, held until
 * the process exits).  cp, cn, psi, ex, ey: device arrays of nx*ny doubles,
 * index nx*y + x.  Uses nx, ny, dx, dy, lx, eps, f_charge, zeta_lo, zeta_hi of p.
 * Limit: nx*ny <= 524288 nodes (nx a power of two <= 8192, or nx <= 2048)
 * and ny <= 65535; larger channels return EK_ERR_TOO_LARGE before any work
 * is queued.  All calls on a GPU share the scratch: calls that overlap on the
 * GPU race, so order them on one stream.  The first call on a device looks up
 * the scratch addresses; make it before any stream capture.  After
 * cudaDeviceReset the next call looks them up again (also outside a capture).
 * A launch error pending from the caller's earlier work is cleared on entry;
 * on EK_ERR_CUDA part of the call may be queued and psi, ex, ey are undefined.
 * stream: a cudaStream_t, NULL for the legacy stream. */
int ek_poisson_noalloc(const ek_params *p, const double *cp, const double *cn,
                       double *psi, double *ex, double *ey, void *stream);

/* ---- profiling (CUDA events on the context's stream) ------------------
 * Phases of a step: 0 = fused LBM kernel, 1 = Poisson pass A (row FFTs),
 * 2 = pass B (tridiagonal y-solve), 3 = pass C (inverse row FFTs).
 * ek_profile_enable(ctx, 1) resets and starts per-launch timing;
 * ek_profile_read waits for the stream and returns, per phase, the summed
 * kernel milliseconds and the launch count since the last enable. */
int ek_profile_enable(ek_ctx *ctx, int32_t on);
int ek_profile_read(ek_ctx *ctx, double *ms4, int64_t *launches4);
/* Record event `slot` (0..15) on the context's stream; elapsed ms between two
 * recorded slots (waits for the later one). */
int ek_mark(ek_ctx *ctx, int32_t slot);
int ek_elapsed(ek_ctx *ctx, int32_t slot_a, int32_t slot_b, double *ms);
/* Total number of kernels this context has launched. */
int ek_launch_count(const ek_ctx *ctx, int64_t *out);

/* ---- the reference's file formats and diagnostics (host arrays) ---------
 * Field arrays are nx*ny doubles, index nx*y + x; no device work.  The
 * reference extrapolates wall rows of its own host copies in place; these
 * calls leave the caller's arrays unchanged. */
/* data_end.dat restart: nx*ny lines "%10.6f" x 9: time ux uy rho c+ phi Ex Ey
 * c- (save_data_end LBM.cu:1272-1312; read_data LBM.cu:1350-1392). */
int ek_write_restart(const char *path, int32_t nx, int32_t ny, double time, const double *ux, const double *uy,
                     const double *rho, const double *cp, const double *psi, const double *ex, const double *ey,
                     const double *cn);
int ek_read_restart(const char *path, int32_t nx, int32_t ny, double *time, double *ux, double *uy, double *rho,
                    double *cp, double *psi, double *ex, double *ey, double *cn);
/* A context's fields to / from that file (ek_load_restart also loads E,
 * which the next step then uses, as read_data's Ex/Ey are). */
int ek_save_restart(ek_ctx *ctx, const char *path, double time);
int ek_load_restart(ek_ctx *ctx, const char *path, double *time);
/* One Tecplot POINT zone with the reference's derived fields (charge
 * gradient, vorticity and its Laplacian, curl of the electric force); the
 * VARIABLES header and a new file when first != 0, appended otherwise
 * (save_data_tecplot LBM.cu:1100-1270).  nx >= 3, ny >= 6. */
int ek_write_tecplot(const char *path, int32_t first, double time, int32_t nx, int32_t ny, double dx, double dy,
                     const double *ux, const double *uy, const double *rho, const double *cp, const double *psi,
                     const double *ex, const double *ey, const double *cn);
/* c+ snapshot for DMD, top row extrapolated, "%10.6f \n" per node
 * (save_data_dmd LBM.cu:1314-1348). */
int ek_write_dmd(const char *path, int32_t append, int32_t nx, int32_t ny, const double *cp);
/* Electric current through the top wall, K dy sum_x c+ Ey on the
 * extrapolated wall row (current LBM.cu:1394-1417); mob_p is K. */
int ek_diag_current(int32_t nx, int32_t ny, const double *cp, const double *ey, double mob_p, double dy, double *out);
/* The reference's "umax": the maximum of u_y (not |u|) with the top row
 * extrapolated, never below 0 (record_umax LBM.cu:1419-1451). */
int ek_diag_umax(int32_t nx, int32_t ny, const double *uy, double *out);

/* ---- batches of independent channels ------------------------------------
 * No counterpart in the reference (one channel per run of main.cu).  A batch
 * steps many channels of different sizes and parameters in lockstep, four
 * kernel launches per step for all of them: one persistent LBM kernel over a
 * tile work-list and three batched Poisson passes.  Each channel is an ek_ctx
 * owned by the batch (ek_batch_channel); use it for ek_set_fields,
 * ek_set_wall_profile, ek_init_poisson_boltzmann, ek_get_fields and
 * ek_residual, but step it only through the batch.  Per channel, a batch step
 * gives the bits of ek_step with ek_set_rebase_interval(cycle) (cycle below).
 * Channels: FP32 or FP16 storage (one for all), nx a power of two in
 * [16, 4096], ny <= 8194, E derived from psi (no EK_FLAG_EXPLICIT_E).
 * All calls on one batch use the batch's own stream (ek_batch_stream). */
typedef struct ek_batch ek_batch;
int ek_batch_create(const ek_params *params, int32_t count, ek_batch **out);
int ek_batch_destroy(ek_batch *b);
int ek_batch_count(const ek_batch *b, int32_t *count, int64_t *nodes);
int ek_batch_channel(ek_batch *b, int32_t index, ek_ctx **out);
int ek_batch_stream(const ek_batch *b, void **stream);
/* Steps run in cycles of `steps` (even, >= 2; default 200): the last step of a
 * cycle writes the moments and, if rebase != 0 (default), re-bases the
 * shifted populations to the new row means.  use_graph != 0 (default) replays
 * whole cycles from a CUDA graph captured on first use. */
int ek_batch_set_cycle(ek_batch *b, int32_t steps, int32_t rebase, int32_t use_graph);
/* ek_init_equilibrium of every channel from its fields; step count to 0. */
int ek_batch_init_equilibrium(ek_batch *b);
/* nsteps coupled steps of every channel; the moments (fields) are current
 * when the call's work ends.  Asynchronous: ek_batch_sync waits. */
int ek_batch_step(ek_batch *b, int32_t nsteps);
int ek_batch_sync(ek_batch *b);
int ek_batch_step_count(const ek_batch *b, int64_t *out);
int ek_batch_launch_count(const ek_batch *b, int64_t *out);
/* Block shapes of the batched LBM kernel, indices 0 .. EK_BATCH_SHAPES-1:
 * threads per block, the widest tile (a tile is min(width, nx) columns by
 * threads / min(width, nx) rows) and the blocks per SM that the kernel's
 * register allocation allows.  Every shape gives the same bits. */
#define EK_BATCH_SHAPES 6
int ek_batch_shape_info(int32_t index, int32_t *threads, int32_t *width, int32_t *blocks_per_sm);
int ek_batch_shape(const ek_batch *b, int32_t *index);
int ek_batch_set_shape(ek_batch *b, int32_t index);
/* Times `steps` steps in each block shape (the state advances by
 * EK_BATCH_SHAPES (steps + 2) steps) and keeps the fastest; chosen: its
 * index; ms (optional, EK_BATCH_SHAPES values): ms per step of each shape. */
int ek_batch_autotune(ek_batch *b, int32_t steps, int32_t *chosen, double *ms);
/* Freeze (mask[i] == 0) or step (mask[i] != 0) each channel; a frozen
 * channel keeps its state and step count, the launches per step stay the
 * same and the work shrinks to the active channels (a run to steady state freezes
 * the channels that have converged).  A frozen channel rejoins only after an
 * even number of batch steps.  ek_batch_init_equilibrium activates all. */
int ek_batch_set_active(ek_batch *b, const uint8_t *mask);
/* Adopt the channels' current states after they were set through their own
 * handles (ek_tile_x): all channels must be initialised and at one step
 * parity and state; the batch steps on from there. */
int ek_batch_resync(ek_batch *b);
/* Restart the channels with mask[i] != 0 in place from the fields loaded
 * through their own handles (ek_set_fields): their populations become the
 * equilibrium of those fields in the buffer the batch steps from next (that
 * step pulls them, as every step but a batch's first does), their step counts
 * start over and they step on with the others; the other channels are not
 * touched.  A run to steady state uses it to send a channel whose start went
 * wrong back to the cold start without waiting for the rest of the batch.
 * A restarted channel's next residual compares with its state before the
 * restart. */
int ek_batch_restart(ek_batch *b, const uint8_t *mask);
/* mask (optional, count bytes) and the number of active nodes (optional). */
int ek_batch_active(const ek_batch *b, uint8_t *mask, int64_t *active_nodes);
/* ek_residual of every channel: out5 gets 5 doubles per channel (u_x, c+,
 * c-, psi, max), worst5 (optional) the maxima over the finite channels.  A
 * channel holding non-finite values gets NaN residuals (the call succeeds). */
int ek_batch_residual(ek_batch *b, int32_t interval, double *out5, double *worst5);

/* ---- learned warm start: MLP on the tensor cores ------------------------
 * No counterpart in the reference.  A 4 -> 256 -> 256 -> 256 -> 512 network
 * with SiLU activations (inputs: the four normalised channel descriptors;
 * outputs: four 128-point profiles across the channel).  Forward, backward
 * and Adam run in hand-written kernels: BF16 operands on the tensor cores
 * (tcgen05, FP32 accumulation in tensor memory), FP32 master weights.
 * Parameters are one flat FP32 array, per layer W (out x in, row-major; the
 * first layer's 4 inputs padded to 16 with zero weights) then b (out). */
typedef struct ek_mlp ek_mlp;
/* batch: rows per training step, a multiple of 128; seed: weight
 * initialisation (Glorot uniform, zero biases) and batch shuffling. */
int ek_mlp_create(int32_t batch, uint64_t seed, ek_mlp **out);
int ek_mlp_destroy(ek_mlp *m);
int ek_mlp_param_count(const ek_mlp *m, int64_t *n);
int ek_mlp_get_params(ek_mlp *m, float *flat);
/* Replaces the parameters and resets the Adam state and step count. */
int ek_mlp_set_params(ek_mlp *m, const float *flat);
/* Training set: x n x 4, t n x 512 (host, FP32), n >= batch. */
int ek_mlp_set_data(ek_mlp *m, const float *x, const float *t, int64_t n);
/* iters Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) on shuffled batches
 * (a new permutation every epoch); loss_out (optional, iters doubles) gets
 * each step's mean squared error. */
int ek_mlp_train(ek_mlp *m, int32_t iters, float lr, double *loss_out);
/* Gradients of the mean squared error of one batch (x batch x 4, t batch x
 * 512) into grads (param_count floats), loss optional; no update. */
int ek_mlp_gradients(ek_mlp *m, const float *x, const float *t, float *grads, double *loss);
/* y (n x 512) = network(x (n x 4)), host arrays. */
int ek_mlp_forward(ek_mlp *m, const float *x, int64_t n, float *y);
int ek_mlp_launch_count(const ek_mlp *m, int64_t *out);
/* Bound, in SM clock cycles (>= 1), of each wait for the tensor cores inside
 * the network's GEMMs (default 2^31, about a second).  A wait that runs out
 * makes the call return EK_ERR_TIMEOUT; MMAs still in flight are waited for
 * at the default bound before the tensor memory is freed. */
int ek_mlp_set_wait_cycles(ek_mlp *m, int64_t cycles);
/* Device self-test of the bounded wait used by the GEMMs: one thread waits,
 * at most `cycles`, on a shared-memory barrier that another thread completes
 * only if arrive != 0.  Returns EK_OK when the wait saw the arrival and
 * EK_ERR_TIMEOUT when it gave up; either way the kernel ends and the device
 * stays usable. */
int ek_wait_selftest(int64_t cycles, int32_t arrive);
/* C (m x n, FP32, row stride ldc) = A (m x k) * B (n x k)^T on the tensor
 * cores; A, B BF16 (uint16 bit patterns), device pointers 16-byte aligned;
 * m a multiple of 128, n a multiple of 16 (of 128 above 128), k a multiple of
 * 16, lda and ldb multiples of 8.  Synchronises the stream. */
int ek_gemm_bf16(const uint16_t *a, int32_t lda, const uint16_t *b, int32_t ldb, float *c, int32_t ldc,
                 int32_t m, int32_t n, int32_t k, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EKPNP_H */
