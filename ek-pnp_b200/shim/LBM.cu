// LBM.cu (drop-in) -- the host entry points that the reference's LBM.h
// declares (LBM.h:149-169), implemented over libekpnp's C ABI
// (include/ekpnp.h).  Together with the poisson.cu of this folder it replaces
// the reference's LBM.cu and poisson.cu; the reference's main.cu and LBM.h
// compile against it unchanged.
//
// main.cu includes LBM.h, LBM.cu and poisson.cu textually (main.cu:18-20), so
// this file is compiled inside main.cu's translation unit: it sees the sizes
// and constants of the caller's LBM.h (NX, NY, the __constant__ physics, the
// *_host values) and its globals (phi_gpu, Ex_gpu, Ey_gpu).  Build:
//   nvcc -O3 -gencode arch=compute_100a,code=sm_100a -I<repo>/include \
//        main.cu seconds.cpp -L<repo>/ek-pnp_b200/ekpnp -lekpnp -lcufft
// with this folder's LBM.cu and poisson.cu beside main.cu and LBM.h.
//
// What each entry point does:
//   initialization      ek_init_poisson_boltzmann(EK_PB_REFERENCE): the
//                       reference's 501 under-relaxed rounds (LBM.cu:95-130)
//   read_data           data_end.dat through ek_read_restart into the
//                       caller's device buffers (LBM.cu:1350-1391)
//   init_equilibrium    the caller's fields into the library
//                       (ek_set_fields_device), then ek_init_equilibrium
//   stream_collide_save one coupled step, ek_step(ctx, 1): the fused LBM
//                       kernel and the Poisson solve of the same loop body
//   fast_Poisson        right after stream_collide_save: completes that step
//                       (its solve already ran); on its own: ek_poisson on the
//                       caller's c+ and c-, psi and E into phi_gpu, Ex_gpu, Ey_gpu
//   writers, current    the library's writers of the reference formats
//                       (ek_write_tecplot, ek_write_restart, ek_write_dmd,
//                       ek_diag_current, ek_diag_umax) and save_scalar
//
// Buffers.  The library keeps its own populations (27 planes, ping-pong) and
// field planes; the caller's f/h/temp population buffers (main.cu:93-101) are
// neither read nor written.  The caller's rho, ux, uy, charge, T, phi, Ex, Ey
// buffers receive the library's fields only on the steps after which
// main.cu's loop reads them (main.cu:205-231): i % printCurrent == 1 (charge
// and Ey copied to the host directly), i % NSAVE == 1, i % NDMD == 1 and the
// last step (i == NSTEPS).  Only those steps write the moments at all
// (EK_OPT_LAST_STEP_MOMENTS), so the other steps move no field plane beyond
// the solve's own.  Every writer below copies the fields back first if they
// are older than the library's, so a loop that calls the writers at other
// steps still writes psi and E of the current step; its rho, u, c+, c- are
// those of the last scheduled step unless this file is compiled with
// -DEKPNP_SHIM_MOMENTS_EVERY_STEP (moments on every step).
//
// Precision: FP64 populations by default (-DEKPNP_SHIM_STORAGE=1 for the
// FP32 shifted form).  The electric body force that the reference ships
// commented out (LBM.cu:388-389, 438-439) is on; -DEKPNP_SHIM_FORCE=0 turns
// it off.
//
// Errors end the process with the library's message, as the reference's
// checks do (LBM.cu:44-62).  The library runs on its own CUDA stream; the
// entry points synchronise with the caller's legacy stream where the caller's
// buffers change hands.
#ifndef EKPNP_SHIM_LBM_CU
#define EKPNP_SHIM_LBM_CU

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "LBM.h"
#include "ekpnp.h"

#ifndef EKPNP_SHIM_FORCE
#define EKPNP_SHIM_FORCE 1
#endif
#ifndef EKPNP_SHIM_STORAGE
#define EKPNP_SHIM_STORAGE EK_STORE_F64
#endif

// main.cu checks its own CUDA calls with this macro (main.cu:76-111).
#define checkCudaErrors(err) ekshim_cuda_check((err), #err, __FILE__, __LINE__)
#define getLastCudaError(msg) ekshim_cuda_check(cudaGetLastError(), (msg), __FILE__, __LINE__)

inline void ekshim_cuda_check(cudaError_t err, const char *what, const char *file, int line) {
    if (err != cudaSuccess) {
        fprintf(stderr, "CUDA error at %s(%d) \"%s\": [%d] %s.\n", file, line, what, (int)err,
                cudaGetErrorString(err));
        exit(-1);
    }
}

namespace ekshim {

inline void check(int rc, const char *what) {
    if (rc != EK_OK) {
        fprintf(stderr, "libekpnp: %s failed: %s (%s)\n", what, ek_status_string(rc), ek_last_error());
        exit(-1);
    }
}

template <typename T>
T from_symbol(const T &symbol) {
    T v;
    checkCudaErrors(cudaMemcpyFromSymbol(&v, symbol, sizeof(T), 0, cudaMemcpyDeviceToHost));
    return v;
}

struct State {
    ek_ctx *ctx = nullptr;
    unsigned iter = 0;         // stream_collide_save calls since init_equilibrium
    bool step_open = false;    // a step whose fast_Poisson call has not come yet
    bool write_back = false;   // that step's fields go to the caller's buffers
    bool stale = false;        // the caller's buffers are older than the library's fields
    // the caller's moment buffers, as passed to stream_collide_save
    double *rho = nullptr, *ux = nullptr, *uy = nullptr, *cp = nullptr, *cn = nullptr;
};
inline State &st() {
    static State s;
    return s;
}

// ek_params from the caller's LBM.h (the constants main.cu also copies into
// the device variables nu, K, D, Kn, uw, exf, main.cu:36-42).
inline ek_params params() {
    ek_params p;
    check(ek_params_default(&p, (int32_t)NX, (int32_t)NY), "ek_params_default");
    p.storage = EKPNP_SHIM_STORAGE;
    p.flags = EK_FLAG_REST_QUIRK | (EKPNP_SHIM_FORCE ? EK_FLAG_FORCE : 0);
    p.dx = from_symbol(dx);
    p.dy = from_symbol(dy);
    p.dt = from_symbol(dt);
    p.cfl = from_symbol(CFL);
    p.cs2 = from_symbol(cs_square);
    p.lx = from_symbol(Lx);
    p.rho0 = from_symbol(rho0);
    p.c0 = from_symbol(chargeinf);
    p.nu = nu_host;
    p.magic_f = from_symbol(V);
    p.diff_p = from_symbol(diffu);
    p.magic_p = from_symbol(VC);
    p.mob_p = K_host;
    p.diff_n = D_host;
    p.magic_n = from_symbol(VT);
    p.mob_n = Kn_host;
    p.eps = from_symbol(eps);
    p.f_charge = from_symbol(convertCtoCharge);
    p.zeta_lo = from_symbol(voltage);
    p.zeta_hi = from_symbol(voltage2);
    p.cp_lo = from_symbol(charge0);
    p.cp_hi = from_symbol(charge1);
    p.cn_lo = from_symbol(charge0n);
    p.cn_hi = from_symbol(charge1n);
    p.ext_x = from_symbol(Ext);
    p.exf = exf_host;
    p.uw = uw_host;
    return p;
}

inline ek_ctx *ctx() {
    State &s = st();
    if (!s.ctx) {
        const ek_params p = params();
        check(ek_create(&p, &s.ctx), "ek_create");
#ifndef EKPNP_SHIM_MOMENTS_EVERY_STEP
        check(ek_set_option(s.ctx, EK_OPT_LAST_STEP_MOMENTS, 0), "ek_set_option");
#endif
    }
    return s.ctx;
}

// Does main.cu's loop read the caller's buffers after iteration i?
inline bool loop_reads_after(unsigned i) {
    auto hit = [i](unsigned every) { return every != 0 && i % every == 1; };
    return hit(printCurrent) || hit(NSAVE) || hit(NDMD) || i == NSTEPS;
}

// The library's fields into the caller's buffers (moments into the buffers
// last given to stream_collide_save, psi and E into phi_gpu, Ex_gpu, Ey_gpu).
inline void write_back_now() {
    State &s = st();
    check(ek_get_fields_device(ctx(), s.rho, s.ux, s.uy, s.cp, s.cn, phi_gpu, Ex_gpu, Ey_gpu),
          "ek_get_fields_device");
    check(ek_sync(ctx()), "ek_sync");
    s.stale = false;
}

inline void fresh() {
    if (st().stale) write_back_now();
}

// Host copy of one device field of the caller.
struct HostField {
    double *h;
    explicit HostField(const double *dev) : h((double *)malloc(mem_size_scalar)) {
        if (!h) {
            fprintf(stderr, "unable to allocate %zu bytes of host memory\n", (size_t)mem_size_scalar);
            exit(-1);
        }
        checkCudaErrors(cudaMemcpy(h, dev, mem_size_scalar, cudaMemcpyDeviceToHost));
    }
    ~HostField() { free(h); }
};

// Append the file that a library writer produced to the caller's open FILE*.
inline void append_file(FILE *out, const char *path) {
    FILE *in = fopen(path, "rb");
    if (!in) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(-1);
    }
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), in)) > 0) fwrite(buf, 1, n, out);
    fclose(in);
    remove(path);
}

inline void temp_path(char *out, size_t cap) {
    static unsigned serial = 0;
    snprintf(out, cap, ".ekpnp_shim_%d_%u.tmp", (int)getpid(), serial++);
}

}  // namespace ekshim

// ---- start-up ---------------------------------------------------------------

__host__ void initialization(double *r, double *c, double *fi, double *u, double *v, double *ex, double *ey,
                             double *temp, double *kx_, double *ky_, cufftHandle plan_) {
    (void)kx_;
    (void)ky_;
    (void)plan_;
    using namespace ekshim;
    const double e_kt = from_symbol(electron) / from_symbol(kB) / from_symbol(roomT);
    check(ek_init_poisson_boltzmann(ctx(), EK_PB_REFERENCE, 501, from_symbol(PB_omega), e_kt),
          "ek_init_poisson_boltzmann");
    check(ek_get_fields_device(ctx(), r, u, v, c, temp, fi, ex, ey), "ek_get_fields_device");
    check(ek_sync(ctx()), "ek_sync");
}

__host__ void read_data(double *time, double *rho_d, double *charge_d, double *phi_d, double *ux_d,
                        double *uy_d, double *Ex_d, double *Ey_d, double *T_d) {
    using namespace ekshim;
    const size_t n = (size_t)NX * NY;
    double *h = (double *)malloc(8 * n * sizeof(double));
    if (!h) {
        fprintf(stderr, "unable to allocate host memory for data_end.dat\n");
        exit(-1);
    }
    double *ux = h, *uy = h + n, *rho = h + 2 * n, *cp = h + 3 * n, *psi = h + 4 * n, *ex = h + 5 * n,
           *ey = h + 6 * n, *cn = h + 7 * n;
    check(ek_read_restart("data_end.dat", (int32_t)NX, (int32_t)NY, time, ux, uy, rho, cp, psi, ex, ey, cn),
          "ek_read_restart");
    double *dst[8] = {rho_d, charge_d, phi_d, T_d, ux_d, uy_d, Ex_d, Ey_d};
    double *src[8] = {rho, cp, psi, cn, ux, uy, ex, ey};
    for (int k = 0; k < 8; ++k) checkCudaErrors(cudaMemcpy(dst[k], src[k], mem_size_scalar, cudaMemcpyHostToDevice));
    free(h);
}

__host__ void init_equilibrium(double *f0, double *f1, double *h0, double *h1, double *temp0, double *temp1,
                               double *r, double *c, double *u, double *v, double *ex, double *ey, double *temp) {
    (void)f0, (void)f1, (void)h0, (void)h1, (void)temp0, (void)temp1;
    using namespace ekshim;
    State &s = st();
    checkCudaErrors(cudaDeviceSynchronize());  // the caller's buffers are complete
    check(ek_set_fields_device(ctx(), r, u, v, c, temp, phi_gpu, ex, ey), "ek_set_fields_device");
    check(ek_init_equilibrium(ctx()), "ek_init_equilibrium");
    s.iter = 0;
    s.step_open = false;
    s.stale = false;
    s.rho = r;
    s.ux = u;
    s.uy = v;
    s.cp = c;
    s.cn = temp;
}

// ---- the time step ----------------------------------------------------------

__host__ void stream_collide_save(double *f0, double *f1, double *f2, double *h0, double *h1, double *h2,
                                  double *temp0, double *temp1, double *temp2, double *r, double *c, double *u,
                                  double *v, double *ex, double *ey, double *Temp, double t_, double *f0bc_) {
    (void)f0, (void)f1, (void)f2, (void)h0, (void)h1, (void)h2, (void)temp0, (void)temp1, (void)temp2;
    (void)ex, (void)ey, (void)t_, (void)f0bc_;
    using namespace ekshim;
    State &s = st();
    if (!s.ctx) {
        fprintf(stderr, "stream_collide_save: call init_equilibrium first\n");
        exit(-1);
    }
    s.rho = r;
    s.ux = u;
    s.uy = v;
    s.cp = c;
    s.cn = Temp;
    s.write_back = loop_reads_after(s.iter);
#ifndef EKPNP_SHIM_MOMENTS_EVERY_STEP
    check(ek_set_option(s.ctx, EK_OPT_LAST_STEP_MOMENTS, s.write_back ? 1 : 0), "ek_set_option");
#endif
    check(ek_step(s.ctx, 1), "ek_step");
    s.step_open = true;
    s.stale = true;
    ++s.iter;
}

// ---- writers of the reference's file formats and diagnostics --------------

__host__ void report_flow_properties(unsigned int n, double t_, double *rho_, double *charge_, double *phi_,
                                     double *ux_, double *uy_, double *Ex_, double *Ey_) {
    (void)rho_, (void)charge_, (void)phi_, (void)ux_, (void)uy_, (void)Ex_, (void)Ey_;
    printf("Iteration: %u, physical time: %g.\n", n, t_);
}

// The dimensionless groups of compute_parameters (LBM.cu:1026-1060).
__host__ void compute_parameters(double *T_, double *M_, double *C_, double *Fe_) {
    using namespace ekshim;
    const double k = from_symbol(K), e = from_symbol(eps), zeta = from_symbol(voltage), nuv = from_symbol(nu);
    const double ly = from_symbol(Ly), d = from_symbol(diffu), c0w = from_symbol(charge0), r0 = from_symbol(rho0);
    *M_ = sqrt(e / r0) / k;
    *T_ = e * zeta / k / nuv / r0;
    *C_ = c0w * ly * ly / (zeta * e);
    *Fe_ = k * zeta / d;
}

// Raw doubles of one field, file "<name><n, zero-padded to the digits of
// NSTEPS>.bin" (the reference's save_scalar naming, LBM.cu:1062-1098).
__host__ void save_scalar(const char *name, double *scalar_gpu, double *scalar_host, unsigned int n) {
    using namespace ekshim;
    fresh();
    const int digits = (int)floor(log10((double)NSTEPS) + 1.0);
    char path[160];
    snprintf(path, sizeof(path), "%s%0*u.bin", name, digits, n);
    checkCudaErrors(cudaMemcpy(scalar_host, scalar_gpu, mem_size_scalar, cudaMemcpyDeviceToHost));
    FILE *f = fopen(path, "wb+");
    if (!f) {
        fprintf(stderr, "Error saving to %s\n", path);
        return;
    }
    fwrite(scalar_host, 1, mem_size_scalar, f);
    fclose(f);
}

__host__ void save_data_tecplot(FILE *fout, double time, double *rho_d, double *charge_d, double *phi_d,
                                double *ux_d, double *uy_d, double *Ex_d, double *Ey_d, double *T_d, int first) {
    using namespace ekshim;
    fresh();
    HostField rho(rho_d), cp(charge_d), psi(phi_d), ux(ux_d), uy(uy_d), ex(Ex_d), ey(Ey_d), cn(T_d);
    char path[96];
    temp_path(path, sizeof(path));
    check(ek_write_tecplot(path, first, time, (int32_t)NX, (int32_t)NY, from_symbol(dx), from_symbol(dy), ux.h,
                           uy.h, rho.h, cp.h, psi.h, ex.h, ey.h, cn.h),
          "ek_write_tecplot");
    append_file(fout, path);
}

__host__ void save_data_end(FILE *fend, double time, double *rho_d, double *charge_d, double *phi_d,
                            double *ux_d, double *uy_d, double *Ex_d, double *Ey_d, double *T_d) {
    using namespace ekshim;
    fresh();
    HostField rho(rho_d), cp(charge_d), psi(phi_d), ux(ux_d), uy(uy_d), ex(Ex_d), ey(Ey_d), cn(T_d);
    char path[96];
    temp_path(path, sizeof(path));
    check(ek_write_restart(path, (int32_t)NX, (int32_t)NY, time, ux.h, uy.h, rho.h, cp.h, psi.h, ex.h, ey.h, cn.h),
          "ek_write_restart");
    append_file(fend, path);
}

__host__ void save_data_dmd(FILE *fend, double time, double *ux_d, double *uy_d, double *charge_d,
                            double *phi_d) {
    (void)time, (void)ux_d, (void)uy_d, (void)phi_d;
    using namespace ekshim;
    fresh();
    HostField cp(charge_d);
    char path[96];
    temp_path(path, sizeof(path));
    check(ek_write_dmd(path, 0, (int32_t)NX, (int32_t)NY, cp.h), "ek_write_dmd");
    append_file(fend, path);
}

__host__ double current(double *c, double *ey) {
    using namespace ekshim;
    double i_wall = 0.0;
    check(ek_diag_current((int32_t)NX, (int32_t)NY, c, ey, K_host, from_symbol(dy), &i_wall), "ek_diag_current");
    return i_wall;
}

__host__ void record_umax(FILE *fend, double time, double *ux_d, double *uy_d) {
    (void)ux_d;
    using namespace ekshim;
    fresh();
    HostField uy(uy_d);
    double umax = 0.0;
    check(ek_diag_umax((int32_t)NX, (int32_t)NY, uy.h, &umax), "ek_diag_umax");
    fprintf(fend, "%10.6f %10.6f\n", time, umax);
}

#endif  // EKPNP_SHIM_LBM_CU
