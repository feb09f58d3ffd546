// ek_api.cu -- the C ABI of libekpnp (declared in include/ekpnp.h).
//
// Host-side owner of a channel: allocation, parameter checks, the step loop
// (one fused LBM launch + three Poisson passes per step) and field I/O.
// Replaces the host code of main.cu:28-307 and the host wrappers of LBM.cu /
// poisson.cu; every failure is returned as a status instead of exit().
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "ek_internal.h"

using namespace ek;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? EK_ERR_NOMEM : EK_ERR_CUDA;
}

#define EK_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

#include "ek_ctx.h"

namespace {

int validate(const ek_params *p) {
    if (!p) return fail(EK_ERR_INVALID, "null parameters");
    if (p->nx < 2 || p->ny < 4) return fail(EK_ERR_INVALID, "need nx >= 2 and ny >= 4");
    if (p->storage != EK_STORE_F64 && p->storage != EK_STORE_F32 && p->storage != EK_STORE_F16)
        return fail(EK_ERR_INVALID, "unknown storage mode");
    if (is_pow2(p->nx) ? p->nx > 8192 : p->nx > 2048)
        return fail(EK_ERR_UNSUPPORTED, "nx above 8192 (powers of two) or 2048 (other lengths)");
    if (p->ny > 65535) return fail(EK_ERR_UNSUPPORTED, "ny above 65535");
    const double pos[] = {p->dx, p->dy, p->dt, p->cfl, p->cs2, p->lx, p->nu, p->diff_p, p->diff_n,
                          p->magic_f, p->magic_p, p->magic_n};
    for (double v : pos)
        if (!(v > 0.0) || !std::isfinite(v)) return fail(EK_ERR_INVALID, "non-positive or non-finite scale/rate parameter");
    const double fin[] = {p->rho0, p->c0, p->mob_p, p->mob_n, p->eps, p->f_charge, p->zeta_lo,
                          p->zeta_hi, p->cp_lo, p->cp_hi, p->cn_lo, p->cn_hi, p->ext_x, p->exf, p->uw};
    for (double v : fin)
        if (!std::isfinite(v)) return fail(EK_ERR_INVALID, "non-finite parameter");
    if (p->eps == 0.0) return fail(EK_ERR_INVALID, "eps must be non-zero");
    if (p->flags & ~(EK_FLAG_FORCE | EK_FLAG_REST_QUIRK | EK_FLAG_MOMENTS_EVERY_STEP | EK_FLAG_EXPLICIT_E))
        return fail(EK_ERR_INVALID, "unknown flag bits");
    return EK_OK;
}

void free_ctx(ek_ctx *c) {
    if (!c) return;
    cudaFree(c->pops[0]);
    cudaFree(c->pops[1]);
    cudaFree(c->fields);
    cudaFree(c->wall);
    cudaFree(c->snap);
    cudaFree(c->part);
    cudaFree(c->rates_dev);
    cudaFree(c->kref[0]);
    cudaFree(c->kref[1]);
    cudaFree(c->kwall);
    cudaFree(c->wdelta);
    cudaFree(c->lift);
    cudaFree(c->err_dev);
    cudaFree(c->jacobi_word);
    cudaFree(c->pp.tw);
    cudaFree(c->pp.piv);
    cudaFree(c->pp.spec);
    cudaFree(c->pp.twf);
    cudaFree(c->pp.pivf);
    cudaFree(c->pp.specf);
    cudaFree(c->pp.rowmean);
    cudaFree(c->pp.rowmean_ok);
    cudaFree(c->pp.rhsf);
    cudaFree(c->pp.psif);
    cudaFree(c->pp.psim);
    for (auto &pr : c->ev_pool) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (auto &m : c->marks)
        if (m) cudaEventDestroy(m);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// Pivots of the per-mode tridiagonal solve: b_m = -(2 + kx_m^2 dy^2),
// kx_m = 2 pi m / Lx (main.cu:120-123); piv_0 = 1/b, piv_j = 1/(b - piv_{j-1}).
std::vector<double> make_pivots(const ek_params &p, int n, int mp) {
    std::vector<double> piv((size_t)n * mp, 0.0);
    for (int m = 0; m <= p.nx / 2; ++m) {
        const double kx = (double)m * 2.0 * M_PI / p.lx;
        const double b = -(2.0 + kx * kx * p.dy * p.dy);
        double c = 0.0;
        for (int j = 0; j < n; ++j) {
            c = 1.0 / (b - c);
            piv[(size_t)j * mp + m] = c;
        }
    }
    return piv;
}

std::vector<double2> make_twiddles(int nx) {
    std::vector<double2> tw(nx);
    for (int k = 0; k < nx; ++k) {
        const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)nx;
        tw[k] = make_double2((double)cosl(a), (double)-sinl(a));
    }
    return tw;
}

void refresh_chan(ek_ctx *c) {
    Chan &h = c->chan;
    const ek_params &p = c->p;
    h.nx = p.nx;
    h.ny = p.ny;
    h.nxp = c->nxp;
    h.flags = p.flags;
    h.plane = c->plane;
    h.dx = p.dx;
    h.dy = p.dy;
    h.dt = p.dt;
    h.cfl = p.cfl;
    h.cs2 = p.cs2;
    h.rho0 = p.rho0;
    h.c0 = p.c0;
    h.mob_p = p.mob_p;
    h.mob_n = p.mob_n;
    h.f_charge = p.f_charge;
    h.eps = p.eps;
    h.ext_x = p.ext_x;
    h.exf = p.exf;
    h.r = c->rates;
    h.zlo = c->wall;
    h.zhi = c->wall + p.nx;
    h.cplo = c->wall + 2 * p.nx;
    h.cphi = c->wall + 3 * p.nx;
    h.cnlo = c->wall + 4 * p.nx;
    h.cnhi = c->wall + 5 * p.nx;
    h.kref = c->kref[c->kcur];
    h.kwall = c->kwall;
    h.wdelta = c->wdelta;
    h.rhsf = c->pp.rhsf;
    h.psif = c->pp.psif;
    h.psim = c->pp.psim;
    h.lift = c->lift;
    h.keep_l2 = c->keep_l2;
    c->pp.keep_l2 = c->keep_l2;
    double zl = 0.0, zh = 0.0;  // x-means of the wall potentials (psim of the wall rows)
    for (int x = 0; x < p.nx; ++x) {
        zl += c->wall_host[x];
        zh += c->wall_host[(size_t)p.nx + x];
    }
    c->pp.zlo_mean = zl / p.nx;
    c->pp.zhi_mean = zh / p.nx;
}

// Binary exponent q of a reference grid K 2^-q (values stored /36) for
// values up to vmax: 36 K stays below 2^22, so 36 K 2^-q and every
// (16|4|1) (K' - K) 2^-q are exact in FP32.
int ref_exponent(double vmax) {
    int e = 1;
    while ((double)(1 << e) < vmax && e < 20) ++e;
    return 22 - e;
}

int shifted(const ek_ctx *c) { return c->p.storage != EK_STORE_F64; }

// Shifted storage: the x-fluctuation of the wall lifting, (zeta(x) -
// zeta_mean)/dy^2 per wall, from the host copy of the wall profiles (the
// x-means themselves are refreshed by refresh_chan).
int upload_lift(ek_ctx *c) {
    if (!shifted(c)) return EK_OK;
    const int nx = c->p.nx;
    const double inv_dy2 = 1.0 / (c->p.dy * c->p.dy);
    std::vector<float> l(2 * (size_t)nx);
    for (int x = 0; x < nx; ++x) {
        l[x] = (float)((c->wall_host[x] - c->pp.zlo_mean) * inv_dy2);
        l[(size_t)nx + x] = (float)((c->wall_host[(size_t)nx + x] - c->pp.zhi_mean) * inv_dy2);
    }
    EK_CUDA(cudaMemcpyAsync(c->lift, l.data(), l.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream), "lift");
    EK_CUDA(cudaStreamSynchronize(c->stream), "lift");
    return EK_OK;
}

// The TMA-fed form runs four compute warps per block; on the measured B200
// the node update is issue-bound and the plain form (more resident warps) is
// faster (0.196 against 0.38 ms on 4096x1024), so "automatic" picks plain.
bool use_tma(const ek_ctx *c) {
    if (!shifted(c) || !c->tma_ok) return false;
    return c->lbm_kernel == 2;
}

// Device error word of the pipelined kernels -> EK_ERR_TIMEOUT (cleared).
int check_device_error(ek_ctx *c) {
    int v = 0;
    EK_CUDA(cudaMemcpyAsync(&v, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "error word");
    EK_CUDA(cudaStreamSynchronize(c->stream), "error word");
    if (v != 0) {
        EK_CUDA(cudaMemsetAsync(c->err_dev, 0, sizeof(int), c->stream), "error word");
        return fail(EK_ERR_TIMEOUT, "a bounded device wait of the TMA pipeline gave up");
    }
    return EK_OK;
}

// New reference profile from the fields' row means into the spare buffer.
int refs_from_fields(ek_ctx *c, float *out) {
    EK_CUDA(launch_row_refs(c->chan, c->fields, c->kq[0], c->kq[1], c->kq[2], out, c->stream), "row refs");
    ++c->launches;
    return EK_OK;
}

int rebase_now(ek_ctx *c) {
    float *kold = c->kref[c->kcur], *knew = c->kref[c->kcur ^ 1];
    int rc = refs_from_fields(c, knew);
    if (rc != EK_OK) return rc;
    EK_CUDA(launch_rebase(c->chan, c->p.storage, c->pops[c->cur], kold, knew, c->stream), "rebase");
    ++c->launches;
    c->kcur ^= 1;
    refresh_chan(c);
    return EK_OK;
}

int copy_in(ek_ctx *c, int plane_idx, const double *src, cudaMemcpyKind kind = cudaMemcpyHostToDevice) {
    if (!src) return EK_OK;
    const size_t w = (size_t)c->p.nx * sizeof(double);
    EK_CUDA(cudaMemcpy2DAsync(c->fields + plane_idx * c->plane, (size_t)c->nxp * sizeof(double), src, w, w,
                              c->p.ny, kind, c->stream),
            "copy field to device");
    return EK_OK;
}

int copy_out(ek_ctx *c, int plane_idx, double *dst, cudaMemcpyKind kind) {
    if (!dst) return EK_OK;
    const size_t w = (size_t)c->p.nx * sizeof(double);
    EK_CUDA(cudaMemcpy2DAsync(dst, w, c->fields + plane_idx * c->plane, (size_t)c->nxp * sizeof(double), w,
                              c->p.ny, kind, c->stream),
            "copy field from device");
    return EK_OK;
}

int refresh_e(ek_ctx *c) {
    if (c->e_stale && !(c->p.flags & EK_FLAG_EXPLICIT_E)) {
        EK_CUDA(launch_efield_f64(c->chan, c->fields, c->stream), "efield kernel");
        ++c->launches;
        c->e_stale = false;
    }
    return EK_OK;
}

// Launch one kernel of `phase` through fn(); with profiling on, bracket it
// with a pair of events from the context's pool.
template <typename Fn>
int timed(ek_ctx *c, int phase, const char *what, Fn fn, int kernels = 1) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (c->prof) {
        if (c->ev_used == c->ev_pool.size()) {
            cudaEvent_t e0, e1;
            EK_CUDA(cudaEventCreate(&e0), "event create");
            EK_CUDA(cudaEventCreate(&e1), "event create");
            c->ev_pool.emplace_back(e0, e1);
            c->ev_phase.push_back(0);
        }
        a = c->ev_pool[c->ev_used].first;
        b = c->ev_pool[c->ev_used].second;
        c->ev_phase[c->ev_used] = phase;
        ++c->ev_used;
        EK_CUDA(cudaEventRecord(a, c->stream), "event record");
    }
    EK_CUDA(fn(), what);
    c->launches += kernels;
    if (c->prof) EK_CUDA(cudaEventRecord(b, c->stream), "event record");
    return EK_OK;
}

// The Poisson solve of a step (or of a solve outside the step when
// from_moments: the right-hand side from the c+, c- moments).  FP64 storage:
// the FP64 passes on the FP64 planes.  Shifted storage, FP32 form: the passes
// read rhsf and write psif/psim, and the FP64 psi plane too when write_f64.
// Shifted storage, FP64 passes: the FP64 right-hand side composed from rhsf,
// then psif/psim split from the FP64 psi.
int poisson_now(ek_ctx *c, bool write_f64, bool from_moments = false) {
    const bool sh = shifted(c);
    const bool f32 = ek::ctx_poisson_f32(c);
    if (c->p.flags & EK_FLAG_EXPLICIT_E) write_f64 = true;  // the E planes follow psi every step
    double *rhs = c->fields + F_RHS * c->plane, *psi = c->fields + F_PSI * c->plane;
    if (from_moments) {
        if (f32) EK_CUDA(launch_rhsf_from_moments(c->pp, c->chan, c->fields, c->stream), "rhs kernel");
        else EK_CUDA(launch_rhs_from_moments_f64(c->chan, c->fields, c->stream), "rhs kernel");
        ++c->launches;
    } else if (sh && !f32) {
        EK_CUDA(launch_compose_rhs(c->pp, c->chan, rhs, c->stream), "rhs kernel");
        ++c->launches;
    }
    for (int pass = 0; pass < 3; ++pass) {
        int rc = timed(c, 1 + pass, "poisson kernel", [&] {
            // FP32 form, pass B: the FP64 zero mode rides in the FP32 modes' kernel
            if (f32 && pass == 1) return poisson_tridiag_f32(c->pp, c->stream);
            return f32 ? poisson_pass_f32(pass, c->pp, c->chan, psi, write_f64, c->stream)
                       : poisson_pass_f64(pass, c->pp, c->chan, c->fields, c->stream);
        });
        if (rc != EK_OK) return rc;
    }
    if (sh && !f32) {
        EK_CUDA(launch_split_psi(c->pp, c->chan, psi, c->stream), "split psi");
        ++c->launches;
    }
    c->split_stale = false;
    if (c->p.flags & EK_FLAG_EXPLICIT_E) {
        EK_CUDA(launch_efield_f64(c->chan, c->fields, c->stream), "efield kernel");
        ++c->launches;
    } else {
        c->e_stale = true;
    }
    return EK_OK;
}

// Shifted storage: psif/psim from the FP64 psi plane after psi was set from
// outside the step (fields loaded, a Poisson-Boltzmann start).
int split_if_stale(ek_ctx *c) {
    if (!shifted(c) || !c->split_stale) return EK_OK;
    EK_CUDA(launch_split_psi(c->pp, c->chan, c->fields + F_PSI * c->plane, c->stream), "split psi");
    ++c->launches;
    c->split_stale = false;
    return EK_OK;
}


}  // namespace

namespace ek {
void set_last_error(const char *msg) { g_err = msg; }
int ctx_fail(int code, const char *msg) { return fail(code, msg); }
int ctx_refs_from_fields(ek_ctx *c, float *out) { return refs_from_fields(c, out); }
void ctx_refresh(ek_ctx *c) { refresh_chan(c); }
bool ctx_poisson_f32(const ek_ctx *c) {
    if (c->poisson_mode == 1 || c->p.storage == EK_STORE_F64) return false;
    return poisson_f32_supported(c->pp);
}

int ctx_after_psi(ek_ctx *c) {
    EK_CUDA(launch_efield_f64(c->chan, c->fields, c->stream), "efield kernel");
    ++c->launches;
    c->e_stale = false;
    c->split_stale = shifted(c);
    return EK_OK;
}

int ctx_residual_buffers(ek_ctx *c) {
    if (c->snap) return EK_OK;
    EK_CUDA(cudaMalloc(&c->snap, 4 * c->plane * sizeof(double)), "residual snapshot");
    EK_CUDA(cudaMemsetAsync(c->snap, 0, 4 * c->plane * sizeof(double), c->stream), "residual snapshot");
    EK_CUDA(cudaMalloc(&c->part, (size_t)residual_blocks(c->chan) * 8 * sizeof(double) + 8 * sizeof(double)),
            "residual partials");
    return EK_OK;
}

// out5 = per-field residuals |q - q_snap| / (interval |q|) and their maximum
// (infinite before the first snapshot).
int ctx_residual_finish(ek_ctx *c, const double *sums, int32_t interval, double *out5) {
    for (int k = 0; k < 8; ++k)
        if (!std::isfinite(sums[k])) return fail(EK_ERR_NAN, "non-finite value in ux, c+, c- or psi");
    const bool had = c->snap_valid;
    c->snap_valid = true;
    const double nn = (double)c->p.nx * (double)c->p.ny;
    // u_x is normalised by at least the Helmholtz-Smoluchowski speed |eps zeta E/(rho nu)|
    const double uhs = std::fabs(c->p.eps * c->p.zeta_lo * c->p.ext_x / (c->p.rho0 * c->p.nu));
    const double floors[4] = {std::max(uhs * std::sqrt(nn), 1e-300), 1e-300, 1e-300, 1e-300};
    double worst = 0.0;
    for (int q = 0; q < 4; ++q) {
        const double norm = std::max(std::sqrt(sums[4 + q]), floors[q]);
        out5[q] = had ? std::sqrt(sums[q]) / ((double)interval * norm) : INFINITY;
        worst = std::max(worst, out5[q]);
    }
    out5[4] = worst;
    return EK_OK;
}
}  // namespace ek

extern "C" {

int ek_version(void) { return 100; }

const char *ek_status_string(int status) {
    switch (status) {
        case EK_OK: return "ok";
        case EK_ERR_INVALID: return "invalid argument";
        case EK_ERR_CUDA: return "CUDA error";
        case EK_ERR_NOMEM: return "out of device memory";
        case EK_ERR_NAN: return "non-finite value in the solution";
        case EK_ERR_TIMEOUT: return "bounded device wait timed out";
        case EK_ERR_UNSUPPORTED: return "unsupported configuration";
        case EK_ERR_TOO_LARGE: return "size above the call's maximum";
        default: return "unknown status";
    }
}

const char *ek_last_error(void) { return g_err.c_str(); }

int ek_set_device(int32_t device) {
    EK_CUDA(cudaSetDevice(device), "cudaSetDevice");
    return EK_OK;
}

int ek_get_device_count(int32_t *out) {
    if (!out) return fail(EK_ERR_INVALID, "null argument");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *out = 0;
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *out = n;
    return EK_OK;
}

int ek_params_default(ek_params *p, int32_t nx, int32_t ny) {
    if (!p) return fail(EK_ERR_INVALID, "null parameters");
    std::memset(p, 0, sizeof(*p));
    p->nx = nx;
    p->ny = ny;
    p->storage = EK_STORE_F64;
    p->flags = EK_FLAG_FORCE | EK_FLAG_REST_QUIRK;
    p->dx = p->dy = p->dt = p->cfl = 1.0;
    p->cs2 = 1.0 / 3.0;
    p->lx = (double)nx;
    p->rho0 = p->c0 = 1.0;
    p->nu = 1.0 / 6.0;
    p->magic_f = p->magic_p = p->magic_n = 0.25;
    p->diff_p = p->diff_n = 0.05;
    p->mob_p = 0.05;
    p->mob_n = -0.05;
    p->eps = 1.0;
    p->f_charge = 1.0;
    p->cp_lo = p->cp_hi = p->cn_lo = p->cn_hi = 1.0;
    return EK_OK;
}

int ek_create(const ek_params *p, ek_ctx **out) {
    if (!out) return fail(EK_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int rc = validate(p);
    if (rc != EK_OK) return rc;
    ek_ctx *c = new ek_ctx();
    c->p = *p;
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaGetDevice"); }
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "stream create"); }
    c->own_stream = true;
    c->nxp = round_up(p->nx, 32);
    c->plane = (size_t)p->ny * c->nxp;
    c->n = p->ny - 2;
    c->mp = round_up(p->nx / 2 + 1, 16);
    c->keep_l2 = ek::keep_l2_fits(2 * c->plane * (p->storage == EK_STORE_F64 ? sizeof(double) : sizeof(float)));
    const size_t pop_bytes = 27 * c->plane * pop_elem_bytes(p->storage);
    struct Alloc { void **ptr; size_t bytes; } allocs[] = {
        {(void **)&c->pops[0], pop_bytes},
        {(void **)&c->pops[1], pop_bytes},
        {(void **)&c->fields, F_COUNT * c->plane * sizeof(double)},
        {(void **)&c->wall, 6 * (size_t)p->nx * sizeof(double)},
        {(void **)&c->rates_dev, sizeof(Rates)},
        {(void **)&c->pp.tw, (size_t)p->nx * sizeof(double2)},
        {(void **)&c->pp.piv, (size_t)c->n * c->mp * sizeof(double)},
        {(void **)&c->pp.spec, (size_t)c->n * c->mp * sizeof(double2)},
        {(void **)&c->kref[0], 3 * (size_t)p->ny * sizeof(float)},
        {(void **)&c->kref[1], 3 * (size_t)p->ny * sizeof(float)},
        {(void **)&c->kwall, 8 * (size_t)p->nx * sizeof(float)},
        {(void **)&c->wdelta, 4 * (size_t)p->nx * sizeof(float)},
        {(void **)&c->pp.rhsf, p->storage == EK_STORE_F64 ? 0 : c->plane * sizeof(float)},
        {(void **)&c->pp.psif, p->storage == EK_STORE_F64 ? 0 : c->plane * sizeof(float)},
        {(void **)&c->pp.psim, p->storage == EK_STORE_F64 ? 0 : (size_t)p->ny * sizeof(double)},
        {(void **)&c->lift, p->storage == EK_STORE_F64 ? 0 : 2 * (size_t)p->nx * sizeof(float)},
        {(void **)&c->err_dev, sizeof(int)},
    };
    for (auto &a : allocs) {
        if (a.bytes == 0) continue;
        e = cudaMalloc(a.ptr, a.bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(*a.ptr, 0, a.bytes, c->stream);
        if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "device allocation"); }
    }
    // wall profiles start uniform
    std::vector<double> wall(6 * (size_t)p->nx);
    const double uni[6] = {p->zeta_lo, p->zeta_hi, p->cp_lo, p->cp_hi, p->cn_lo, p->cn_hi};
    for (int k = 0; k < 6; ++k)
        for (int x = 0; x < p->nx; ++x) wall[(size_t)k * p->nx + x] = uni[k];
    c->kq[0] = ref_exponent(2.0 * std::fabs(p->rho0));
    c->kq[1] = ref_exponent(2.0 * std::max({std::fabs(p->c0), std::fabs(p->cp_lo), std::fabs(p->cp_hi)}));
    c->kq[2] = ref_exponent(2.0 * std::max({std::fabs(p->c0), std::fabs(p->cn_lo), std::fabs(p->cn_hi)}));
    std::vector<float> kref(3 * (size_t)p->ny);
    const double base[3] = {p->rho0, p->c0, p->c0};
    for (int sp = 0; sp < 3; ++sp) {
        const double K = std::nearbyint(base[sp] / 36.0 * std::ldexp(1.0, c->kq[sp]));
        for (int y = 0; y < p->ny; ++y) kref[(size_t)sp * p->ny + y] = (float)std::ldexp(K, -c->kq[sp]);
    }
    std::vector<double> piv = make_pivots(*p, c->n, c->mp);
    std::vector<double2> tw = make_twiddles(p->nx);
    c->wall_host = wall;
    e = cudaMemcpyAsync(c->wall, wall.data(), wall.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->pp.piv, piv.data(), piv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->kref[0], kref.data(), kref.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->kref[1], kref.data(), kref.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->pp.tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_rates(*p, c->rates_dev, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&c->rates, c->rates_dev, sizeof(Rates), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = poisson_set_smem_limits();
    if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "context set-up"); }
    if (p->storage != EK_STORE_F64) {
        c->tma_ok = make_pop_tensor_map(p->storage, c->pops[0], c->nxp, p->ny, &c->tmaps[0]) == cudaSuccess &&
                    make_pop_tensor_map(p->storage, c->pops[1], c->nxp, p->ny, &c->tmaps[1]) == cudaSuccess;
    }
    c->pp.nx = p->nx;
    c->pp.ny = p->ny;
    c->pp.n = c->n;
    c->pp.mp = c->mp;
    c->pp.pow2 = is_pow2(p->nx);
    int lg = 0;
    while ((1 << lg) < p->nx) ++lg;
    c->pp.log2nx = c->pp.pow2 ? lg : 0;
    c->pp.dy2 = p->dy * p->dy;
    if (p->storage != EK_STORE_F64 && c->pp.pow2 && p->nx >= 16 && poisson_tridiag_modes(c->n) > 0) {
        // FP32 form of the Poisson solve: FP32 pivots and spectrum; the row
        // transforms' twiddles per radix-16 pass on bits [b, b+4), b = lg-4,
        // lg-8, ... >= 1: exp(-2 pi i kb f / 2^(b+4)) at (f-1) 2^b + kb
        std::vector<float> pivf(piv.begin(), piv.end());
        std::vector<float2> twf;
        for (int b = lg - 4; b >= 1; b -= 4)
            for (int f = 1; f < 16; ++f)
                for (int kb = 0; kb < (1 << b); ++kb) {
                    const double2 w = tw[((size_t)kb * f << (lg - b - 4)) % (size_t)p->nx];
                    twf.push_back(make_float2((float)w.x, (float)w.y));
                }
        if (twf.empty()) twf.push_back(make_float2(1.0f, 0.0f));
        e = cudaMalloc(&c->pp.twf, twf.size() * sizeof(float2));
        if (e == cudaSuccess) e = cudaMalloc(&c->pp.pivf, pivf.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&c->pp.specf, (size_t)c->n * c->mp * sizeof(float2));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->pp.specf, 0, (size_t)c->n * c->mp * sizeof(float2), c->stream);
        if (e == cudaSuccess) e = cudaMalloc(&c->pp.rowmean, (size_t)c->n * sizeof(double));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->pp.rowmean, 0, (size_t)c->n * sizeof(double), c->stream);
        if (e == cudaSuccess) e = cudaMalloc(&c->pp.rowmean_ok, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->pp.rowmean_ok, 0, sizeof(int), c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c->pp.twf, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c->pp.pivf, pivf.data(), pivf.size() * sizeof(float), cudaMemcpyHostToDevice,
                                c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "FP32 Poisson set-up"); }
    }
    refresh_chan(c);
    int rcl = upload_lift(c);
    if (rcl != EK_OK) { free_ctx(c); return rcl; }
    *out = c;
    return EK_OK;
}

int ek_destroy(ek_ctx *c) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_ctx(c);
    return EK_OK;
}

int ek_set_stream(ek_ctx *c, void *stream) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    EK_CUDA(cudaStreamSynchronize(c->stream), "stream sync");
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return EK_OK;
}

int ek_get_params(const ek_ctx *c, ek_params *out) {
    if (!c || !out) return fail(EK_ERR_INVALID, "null argument");
    *out = c->p;
    return EK_OK;
}

namespace {
int set_fields_from(ek_ctx *c, const double *const src[F_RHS], cudaMemcpyKind kind) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if ((src[F_EX] == nullptr) != (src[F_EY] == nullptr)) return fail(EK_ERR_INVALID, "give both ex and ey, or neither");
    for (int k = 0; k < F_RHS; ++k) {
        int rc = copy_in(c, k, src[k], kind);
        if (rc != EK_OK) return rc;
    }
    const double *ex = src[F_EX], *psi = src[F_PSI];
    if (psi) c->split_stale = true;
    if (ex) {
        c->explicit_e_once = true;
        c->e_stale = false;
    } else if (psi) {
        c->e_stale = true;
    }
    EK_CUDA(cudaStreamSynchronize(c->stream), "set_fields sync");
    return EK_OK;
}
}  // namespace

int ek_set_fields(ek_ctx *c, const double *rho, const double *ux, const double *uy, const double *cp,
                  const double *cn, const double *psi, const double *ex, const double *ey) {
    const double *src[F_RHS] = {rho, ux, uy, cp, cn, psi, ex, ey};
    return set_fields_from(c, src, cudaMemcpyHostToDevice);
}

int ek_set_fields_device(ek_ctx *c, const double *rho, const double *ux, const double *uy, const double *cp,
                         const double *cn, const double *psi, const double *ex, const double *ey) {
    const double *src[F_RHS] = {rho, ux, uy, cp, cn, psi, ex, ey};
    return set_fields_from(c, src, cudaMemcpyDeviceToDevice);
}

int ek_set_wall_profile(ek_ctx *c, const double *zlo, const double *zhi, const double *cplo,
                        const double *cphi, const double *cnlo, const double *cnhi) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    const double *src[6] = {zlo, zhi, cplo, cphi, cnlo, cnhi};
    for (int k = 0; k < 6; ++k) {
        if (!src[k]) continue;
        for (int x = 0; x < c->p.nx; ++x)
            if (!std::isfinite(src[k][x])) return fail(EK_ERR_INVALID, "non-finite wall value");
        EK_CUDA(cudaMemcpyAsync(c->wall + (size_t)k * c->p.nx, src[k], c->p.nx * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream),
                "copy wall profile");
        std::copy(src[k], src[k] + c->p.nx, c->wall_host.begin() + (size_t)k * c->p.nx);
    }
    refresh_chan(c);  // the wall potentials' x-means
    int rcl = upload_lift(c);
    if (rcl != EK_OK) return rcl;
    // shifted storage after initialisation: the wall ions' frames stay, their
    // defect follows the new wall concentrations
    if (shifted(c) && c->initialised)
        EK_CUDA(launch_wall_delta(c->chan, c->kwall, c->wdelta, c->stream), "wall frames");
    EK_CUDA(cudaStreamSynchronize(c->stream), "wall profile sync");
    return EK_OK;
}

int ek_init_poisson_boltzmann(ek_ctx *c, int32_t method, int32_t iterations, double omega, double e_kt) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (!std::isfinite(e_kt) || e_kt == 0.0) return fail(EK_ERR_INVALID, "e_kt must be finite and non-zero");
    const ek_params &p = c->p;
    if (method == EK_PB_REFERENCE) {
        if (iterations < 0 || !(omega > 0.0) || !(omega <= 1.0)) return fail(EK_ERR_INVALID, "need iterations >= 0, 0 < omega <= 1");
        double *old = nullptr;
        EK_CUDA(cudaMalloc(&old, c->plane * sizeof(double)), "PB scratch");
        int rc = EK_OK;
        auto run = [&]() -> int {
            EK_CUDA(launch_pb_fill(c->chan, c->fields, old, c->stream), "PB fill");
            for (int32_t it = 0; it < iterations; ++it) {
                EK_CUDA(launch_pb_conc(c->chan, e_kt, c->fields, c->stream), "PB concentrations");
                EK_CUDA(launch_rhs_from_moments_f64(c->chan, c->fields, c->stream), "rhs kernel");
                for (int pass = 0; pass < 3; ++pass)
                    EK_CUDA(poisson_pass_f64(pass, c->pp, c->chan, c->fields, c->stream), "poisson kernel");
                EK_CUDA(launch_efield_f64(c->chan, c->fields, c->stream), "efield kernel");
                EK_CUDA(launch_pb_relax(c->chan, omega, c->fields, old, c->stream), "PB relax");
            }
            EK_CUDA(cudaStreamSynchronize(c->stream), "PB sync");
            return EK_OK;
        };
        rc = run();
        cudaFree(old);
        if (rc != EK_OK) return rc;
        // the fields now hold E of the last Poisson solve, as the reference's do
        c->explicit_e_once = iterations > 0;
        c->e_stale = iterations == 0;
        c->split_stale = true;
        return EK_OK;
    }
    if (method != EK_PB_NEWTON) return fail(EK_ERR_INVALID, "unknown Poisson-Boltzmann method");
    const int nx = p.nx, ny = p.ny;
    const double g = p.f_charge * p.c0 / p.eps;
    // one Newton solve per distinct pair of wall potentials, on the device
    std::map<std::pair<double, double>, int> index;
    std::vector<double2> walls;
    std::vector<int> colmap(nx);
    for (int x = 0; x < nx; ++x) {
        const std::pair<double, double> key{c->wall_host[x], c->wall_host[nx + x]};
        auto it = index.find(key);
        if (it == index.end()) {
            it = index.emplace(key, (int)walls.size()).first;
            walls.push_back(make_double2(key.first, key.second));
        }
        colmap[x] = it->second;
    }
    const int ncol = (int)walls.size();
    // one allocation: the 16-byte wall pairs first, then the three ny x ncol
    // columns of doubles, then the ints
    const size_t bytes = (size_t)ncol * sizeof(double2) + 3 * (size_t)ny * ncol * sizeof(double) +
                         (size_t)(nx + ncol) * sizeof(int);
    char *scratch = nullptr;
    EK_CUDA(cudaMalloc(&scratch, bytes), "Newton PB scratch");
    double2 *dwalls = (double2 *)scratch;
    double *psi = (double *)(dwalls + ncol), *cpv = psi + (size_t)ny * ncol, *dpv = cpv + (size_t)ny * ncol;
    int *dmap = (int *)(dpv + (size_t)ny * ncol), *dok = dmap + nx;
    std::vector<int> ok(ncol, 0);
    cudaError_t e = cudaMemcpyAsync(dwalls, walls.data(), walls.size() * sizeof(double2), cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dmap, colmap.data(), (size_t)nx * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = launch_pb_newton(c->chan, p.dy, g, e_kt, dwalls, ncol, psi, cpv, dpv, dok, dmap, c->fields, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ok.data(), dok, (size_t)ncol * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(scratch);
    EK_CUDA(e, "Newton PB");
    for (int v : ok)
        if (!v) return fail(EK_ERR_INVALID, "Poisson-Boltzmann Newton iteration did not converge");
    EK_CUDA(cudaStreamSynchronize(c->stream), "PB upload");
    c->explicit_e_once = false;
    c->e_stale = true;
    c->split_stale = true;
    return EK_OK;
}

int ek_init_equilibrium(ek_ctx *c) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    const bool ee = c->explicit_e_once || (c->p.flags & EK_FLAG_EXPLICIT_E);
    if (c->p.storage == EK_STORE_F64) {
        EK_CUDA(launch_init_f64(c->chan, (double *)c->pops[c->cur], c->fields, ee, c->stream), "init kernel");
    } else {
        int rc = refs_from_fields(c, c->kref[c->kcur]);
        if (rc != EK_OK) return rc;
        EK_CUDA(launch_wall_frames(c->chan, c->fields, c->kq[1], c->kq[2], c->cur, c->kwall, c->wdelta, c->stream),
                "wall frames");
        EK_CUDA(launch_init_shifted(c->chan, c->p.storage, c->pops[c->cur], c->fields, ee, c->cur, c->stream),
                "init kernel");
        c->split_stale = true;  // the first step's E comes from psif/psim of the loaded psi
        rc = split_if_stale(c);
        if (rc != EK_OK) return rc;
    }
    // the FP32 Poisson form's row offsets start over (exact row means on the
    // first solve), so a re-initialised context repeats a fresh one bit for bit
    if (c->pp.rowmean_ok) EK_CUDA(cudaMemsetAsync(c->pp.rowmean_ok, 0, sizeof(int), c->stream), "row offsets");
    c->initialised = true;
    c->state_pre = true;
    c->steps = 0;
    c->snap_valid = false;
    return EK_OK;
}

extern "C++" {
namespace {
// dst[p][y][x] = src[p][y][x mod snx] for planes p < gridDim.z
template <typename T>
__global__ void tile_x_planes(const T *__restrict__ src, size_t splane, int snxp, int snx, T *__restrict__ dst,
                              size_t dplane, int dnxp, int dnx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= dnx) return;
    const size_t y = blockIdx.y, pl = blockIdx.z;
    dst[pl * dplane + y * dnxp + x] = src[pl * splane + y * snxp + x % snx];
}

// dst[r][x] = src[r][x mod snx] for rows r < rows (row pitches snx, dnx)
template <typename T>
__global__ void tile_x_rows(const T *__restrict__ src, int snx, T *__restrict__ dst, int dnx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= dnx) return;
    dst[(size_t)blockIdx.y * dnx + x] = src[(size_t)blockIdx.y * snx + x % snx];
}

template <typename T>
cudaError_t tile_rows(const T *src, int snx, T *dst, int dnx, int rows, cudaStream_t st) {
    tile_x_rows<T><<<dim3((dnx + 255) / 256, rows), 256, 0, st>>>(src, snx, dst, dnx);
    return cudaGetLastError();
}

template <typename T>
cudaError_t tile_planes(const void *src, const ek_ctx *s, void *dst, const ek_ctx *d, int planes, cudaStream_t st) {
    const dim3 g((d->p.nx + 255) / 256, d->p.ny, planes);
    tile_x_planes<T><<<g, 256, 0, st>>>((const T *)src, s->plane, s->nxp, s->p.nx, (T *)dst, d->plane, d->nxp,
                                        d->p.nx);
    return cudaGetLastError();
}
}  // namespace
}

int ek_tile_x(ek_ctx *dst, const ek_ctx *src) {
    if (!dst || !src || dst == src) return fail(EK_ERR_INVALID, "two distinct contexts needed");
    if (!src->initialised) return fail(EK_ERR_INVALID, "the source holds no populations");
    if (dst->p.ny != src->p.ny || dst->p.storage != src->p.storage || dst->p.nx % src->p.nx != 0)
        return fail(EK_ERR_INVALID, "need the same ny and storage and a destination nx that is a multiple of the source's");
    if (dst->device != src->device) return fail(EK_ERR_INVALID, "contexts on different devices");
    EK_CUDA(cudaStreamSynchronize(src->stream), "source sync");
    const int esz = (int)pop_elem_bytes(dst->p.storage);
    cudaError_t e = esz == 8   ? tile_planes<uint64_t>(src->pops[src->cur], src, dst->pops[dst->cur], dst, 27, dst->stream)
                    : esz == 4 ? tile_planes<uint32_t>(src->pops[src->cur], src, dst->pops[dst->cur], dst, 27, dst->stream)
                               : tile_planes<uint16_t>(src->pops[src->cur], src, dst->pops[dst->cur], dst, 27, dst->stream);
    EK_CUDA(e, "tile populations");
    EK_CUDA(tile_planes<double>(src->fields, src, dst->fields, dst, F_COUNT, dst->stream), "tile fields");
    if (dst->p.storage != EK_STORE_F64) {
        EK_CUDA(cudaMemcpyAsync(dst->kref[dst->kcur], src->kref[src->kcur], 3 * (size_t)dst->p.ny * sizeof(float),
                                cudaMemcpyDeviceToDevice, dst->stream),
                "reference rows");
        for (int q = 0; q < 3; ++q) dst->kq[q] = src->kq[q];
        // wall frames: rows of nx floats, buffer-major; the source's buffer
        // cur becomes the destination's buffer cur
        for (int b = 0; b < 2; ++b) {
            const int sb = b ^ src->cur ^ dst->cur;
            EK_CUDA(tile_rows<float>(src->kwall + (size_t)sb * 4 * src->p.nx, src->p.nx,
                                     dst->kwall + (size_t)b * 4 * dst->p.nx, dst->p.nx, 4, dst->stream),
                    "wall frames");
        }
        EK_CUDA(tile_rows<float>(src->wdelta, src->p.nx, dst->wdelta, dst->p.nx, 4, dst->stream), "wall frames");
        // psi of the step: FP32 fluctuations tiled, row means copied
        EK_CUDA(tile_planes<float>(src->pp.psif, src, dst->pp.psif, dst, 1, dst->stream), "psi planes");
        EK_CUDA(cudaMemcpyAsync(dst->pp.psim, src->pp.psim, (size_t)dst->p.ny * sizeof(double),
                                cudaMemcpyDeviceToDevice, dst->stream),
                "psi row means");
    }
    if (dst->pp.rowmean && src->pp.rowmean) {  // offsets of the FP32 Poisson form (row means: x-independent)
        EK_CUDA(cudaMemcpyAsync(dst->pp.rowmean, src->pp.rowmean, (size_t)dst->n * sizeof(double),
                                cudaMemcpyDeviceToDevice, dst->stream),
                "row means");
        EK_CUDA(cudaMemcpyAsync(dst->pp.rowmean_ok, src->pp.rowmean_ok, sizeof(int), cudaMemcpyDeviceToDevice,
                                dst->stream),
                "row means");
    }
    EK_CUDA(cudaStreamSynchronize(dst->stream), "tile");
    dst->initialised = true;
    dst->state_pre = src->state_pre;
    dst->explicit_e_once = src->explicit_e_once;
    dst->e_stale = src->e_stale;
    dst->split_stale = src->split_stale;
    dst->snap_valid = false;
    refresh_chan(dst);
    return EK_OK;
}

int ek_step(ek_ctx *c, int32_t nsteps) {
    if (!c || nsteps < 0) return fail(EK_ERR_INVALID, "null context or negative step count");
    if (!c->initialised) return fail(EK_ERR_INVALID, "call ek_init_equilibrium before ek_step");
    const bool every = (c->p.flags & EK_FLAG_MOMENTS_EVERY_STEP) != 0;
    int rcs = split_if_stale(c);
    if (rcs != EK_OK) return rcs;
    for (int32_t i = 0; i < nsteps; ++i) {
        const bool ee = c->explicit_e_once || (c->p.flags & EK_FLAG_EXPLICIT_E);
        const bool rebase = shifted(c) && c->rebase_every > 0 && (c->steps + 1) % c->rebase_every == 0;
        const bool mom = every || (i == nsteps - 1 && c->last_moments) || rebase;
        int rc0 = timed(c, 0, "LBM step kernel", [&] {
            if (c->p.storage == EK_STORE_F64)
                return launch_step_f64(c->chan, (const double *)c->pops[c->cur], (double *)c->pops[c->cur ^ 1],
                                       c->fields, c->state_pre, ee, mom, c->stream);
            if (use_tma(c))
                return launch_step_tma(c->chan, c->p.storage, &c->tmaps[c->cur], c->pops[c->cur],
                                       c->pops[c->cur ^ 1], c->fields, c->state_pre, ee, mom, c->cur, c->err_dev,
                                       c->wait_cycles, c->stream);
            return launch_step_shifted(c->chan, c->p.storage, c->pops[c->cur], c->pops[c->cur ^ 1], c->fields,
                                       c->state_pre, ee, mom, c->cur, c->stream);
        });
        if (rc0 != EK_OK) return rc0;
        c->cur ^= 1;
        c->state_pre = false;
        c->explicit_e_once = false;
        int rc = poisson_now(c, mom);  // the FP64 psi plane follows on the steps that write the moments
        if (rc != EK_OK) return rc;
        if (rebase) {
            rc = rebase_now(c);
            if (rc != EK_OK) return rc;
        }
        ++c->steps;
    }
    return EK_OK;
}

int ek_rebase(ek_ctx *c) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (!shifted(c) || !c->initialised) return EK_OK;
    return rebase_now(c);
}

int ek_set_rebase_interval(ek_ctx *c, int32_t steps) {
    if (!c || steps < 0) return fail(EK_ERR_INVALID, "null context or negative interval");
    c->rebase_every = steps;
    return EK_OK;
}

int ek_poisson(ek_ctx *c) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    return poisson_now(c, true, true);
}

int ek_get_fields(ek_ctx *c, double *rho, double *ux, double *uy, double *cp, double *cn, double *psi,
                  double *ex, double *ey) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (ex || ey) {
        int rc = refresh_e(c);
        if (rc != EK_OK) return rc;
    }
    double *dst[F_RHS] = {rho, ux, uy, cp, cn, psi, ex, ey};
    for (int k = 0; k < F_RHS; ++k) {
        int rc = copy_out(c, k, dst[k], cudaMemcpyDeviceToHost);
        if (rc != EK_OK) return rc;
    }
    EK_CUDA(cudaStreamSynchronize(c->stream), "get_fields sync");
    return check_device_error(c);
}

int ek_get_fields_device(ek_ctx *c, double *rho, double *ux, double *uy, double *cp, double *cn,
                         double *psi, double *ex, double *ey) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (ex || ey) {
        int rc = refresh_e(c);
        if (rc != EK_OK) return rc;
    }
    double *dst[F_RHS] = {rho, ux, uy, cp, cn, psi, ex, ey};
    for (int k = 0; k < F_RHS; ++k) {
        int rc = copy_out(c, k, dst[k], cudaMemcpyDeviceToDevice);
        if (rc != EK_OK) return rc;
    }
    return EK_OK;
}

int ek_residual(ek_ctx *c, int32_t interval, double *out5) {
    if (!c || !out5 || interval <= 0) return fail(EK_ERR_INVALID, "bad residual arguments");
    int rc = ek::ctx_residual_buffers(c);
    if (rc != EK_OK) return rc;
    double sums[8];
    const int nb = residual_blocks(c->chan);
    EK_CUDA(launch_residual_f64(c->chan, c->fields, c->snap, c->part, nb, c->part + (size_t)nb * 8, c->stream),
            "residual kernels");
    EK_CUDA(cudaMemcpyAsync(sums, c->part + (size_t)nb * 8, sizeof(sums), cudaMemcpyDeviceToHost, c->stream),
            "residual copy");
    EK_CUDA(cudaStreamSynchronize(c->stream), "residual sync");
    return ek::ctx_residual_finish(c, sums, interval, out5);
}

int ek_step_count(const ek_ctx *c, int64_t *out) {
    if (!c || !out) return fail(EK_ERR_INVALID, "null argument");
    *out = c->steps;
    return EK_OK;
}

int ek_sync(ek_ctx *c) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    EK_CUDA(cudaStreamSynchronize(c->stream), "sync");
    return check_device_error(c);
}

int ek_set_option(ek_ctx *c, int32_t option, int64_t value) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    if (option == EK_OPT_LBM_KERNEL) {
        if (value < 0 || value > 2) return fail(EK_ERR_INVALID, "EK_OPT_LBM_KERNEL takes 0, 1 or 2");
        if (value == 2 && !(shifted(c) && c->tma_ok))
            return fail(EK_ERR_UNSUPPORTED, "TMA-fed kernel needs shifted storage and a tensor map");
        c->lbm_kernel = (int)value;
        return EK_OK;
    }
    if (option == EK_OPT_POISSON) {
        if (value < 0 || value > 2) return fail(EK_ERR_INVALID, "EK_OPT_POISSON takes 0, 1 or 2");
        if (value == 2 && !poisson_f32_supported(c->pp))
            return fail(EK_ERR_UNSUPPORTED, "the FP32 Poisson form needs shifted storage, a power-of-two nx >= 16 "
                                            "and ny <= 8194");
        c->poisson_mode = (int)value;
        return EK_OK;
    }
    if (option == EK_OPT_WAIT_CYCLES) {
        if (value < 1) return fail(EK_ERR_INVALID, "EK_OPT_WAIT_CYCLES takes cycles >= 1");
        c->wait_cycles = (long long)value;
        return EK_OK;
    }
    if (option == EK_OPT_LAST_STEP_MOMENTS) {
        if (value < 0 || value > 1) return fail(EK_ERR_INVALID, "EK_OPT_LAST_STEP_MOMENTS takes 0 or 1");
        c->last_moments = value != 0;
        return EK_OK;
    }
    return fail(EK_ERR_INVALID, "unknown option");
}

int ek_profile_enable(ek_ctx *c, int32_t on) {
    if (!c) return fail(EK_ERR_INVALID, "null context");
    EK_CUDA(cudaStreamSynchronize(c->stream), "profile sync");
    c->prof = on != 0;
    c->ev_used = 0;
    return EK_OK;
}

int ek_profile_read(ek_ctx *c, double *ms4, int64_t *launches4) {
    if (!c || !ms4 || !launches4) return fail(EK_ERR_INVALID, "null argument");
    EK_CUDA(cudaStreamSynchronize(c->stream), "profile sync");
    for (int k = 0; k < 4; ++k) {
        ms4[k] = 0.0;
        launches4[k] = 0;
    }
    for (size_t i = 0; i < c->ev_used; ++i) {
        float ms = 0.0f;
        EK_CUDA(cudaEventElapsedTime(&ms, c->ev_pool[i].first, c->ev_pool[i].second), "event elapsed");
        const int ph = c->ev_phase[i];
        if (ph >= 0 && ph < 4) {
            ms4[ph] += ms;
            ++launches4[ph];
        }
    }
    return EK_OK;
}

int ek_mark(ek_ctx *c, int32_t slot) {
    if (!c || slot < 0 || slot >= 16) return fail(EK_ERR_INVALID, "bad event slot");
    if (!c->marks[slot]) EK_CUDA(cudaEventCreate(&c->marks[slot]), "event create");
    EK_CUDA(cudaEventRecord(c->marks[slot], c->stream), "event record");
    return EK_OK;
}

int ek_elapsed(ek_ctx *c, int32_t a, int32_t b, double *ms) {
    if (!c || !ms || a < 0 || a >= 16 || b < 0 || b >= 16 || !c->marks[a] || !c->marks[b])
        return fail(EK_ERR_INVALID, "bad event slots");
    EK_CUDA(cudaEventSynchronize(c->marks[b]), "event sync");
    float f = 0.0f;
    EK_CUDA(cudaEventElapsedTime(&f, c->marks[a], c->marks[b]), "event elapsed");
    *ms = f;
    return EK_OK;
}

int ek_launch_count(const ek_ctx *c, int64_t *out) {
    if (!c || !out) return fail(EK_ERR_INVALID, "null argument");
    *out = c->launches;
    return EK_OK;
}

int ek_field_pointers(ek_ctx *c, double **out8, int32_t *pitch) {
    if (!c || !out8) return fail(EK_ERR_INVALID, "null argument");
    if (pitch) *pitch = c->nxp;
    int rc = refresh_e(c);
    if (rc != EK_OK) return rc;
    for (int k = 0; k < F_RHS; ++k) out8[k] = c->fields + k * c->plane;
    return EK_OK;
}

}  // extern "C"
