// ek_noalloc.cu -- Poisson solve and electric field for callers that must not
// allocate device memory.
//
// Who needs it: the reference's time loop calls its Poisson step once per
// time step, and the reference allocates and frees four device buffers inside
// every call (poisson.cu:182-207).  An allocation on every step synchronises
// the device and, in a host program whose device memory is owned by an arena
// or pool allocator (or is fully committed by the time the loop runs), it can
// fail or fragment that memory.  ek_poisson_noalloc gives such callers the same
// solve with no allocation at all: its scratch (the x-spectrum of the interior
// rows, the tridiagonal pivots, the FFT twiddles, the right-hand side and the
// wall rows) lives in the file-scope device arrays below, which every GPU that
// loads the library holds until the process exits (10.9 MB per GPU).
//
// Limits: nx*ny <= EK_NOALLOC_MAX_NODES (524,288 nodes, e.g. 1024 x 512), nx
// a power of two up to 8192 or any nx up to 2048; larger channels are rejected
// with EK_ERR_TOO_LARGE.  All calls on a GPU share the arrays and the arrays
// keep the last call's contents, so two calls whose kernels overlap on that GPU
// (different streams, or different host threads) race on them; order such
// calls on one stream.  Each call rewrites every part of the scratch it reads
// and clears the spectrum region it uses before use.
//
// First call on a device: the call looks up the device addresses of the arrays
// (cudaGetSymbolAddress, once per device, with that device current) and
// caches them together with the identity of the device's current context.
// Make that first call before any stream capture begins.  After
// cudaDeviceReset the library's module is loaded again into a new context and
// the arrays move; the next call sees the new context and looks the addresses
// up again (that call, too, belongs outside a stream capture).
//
// Errors: a launch error left pending by the caller's own earlier work is
// cleared on entry, so it is not reported as this call's failure.  When the
// call returns EK_ERR_CUDA, part of its work may already be queued on the
// stream and psi, Ex and Ey are undefined.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "ek_internal.h"

#define EK_NOALLOC_MAX_NODES 524288

namespace ek {
namespace {

constexpr int NA_MAX_NX = 8192;
constexpr int NA_TPB = 128;

// Scratch of the no-allocation solve.  Host code must not pass these names to
// a kernel: on the host they are stand-ins, not device addresses.
static __device__ __align__(256) double2 g_na_spec[EK_NOALLOC_MAX_NODES / 2 + 8192];
static __device__ __align__(256) double g_na_piv[EK_NOALLOC_MAX_NODES / 2 + 8192];
static __device__ __align__(256) double g_na_rhs[EK_NOALLOC_MAX_NODES];
static __device__ __align__(256) double2 g_na_tw[NA_MAX_NX];
static __device__ __align__(256) double g_na_wall[2 * NA_MAX_NX];

struct Scratch {
    double2 *spec = nullptr, *tw = nullptr;
    double *piv = nullptr, *rhs = nullptr, *wall = nullptr;
    unsigned long long ctx_id = 0;  // context the addresses belong to
    bool ready = false;
};
constexpr int NA_MAX_DEVICES = 64;
Scratch g_scratch[NA_MAX_DEVICES];
std::mutex g_scratch_mu;

// Identity of the calling thread's current context (cuCtxGetId through the
// runtime's driver entry points; the handle itself where that is missing).
cudaError_t current_ctx_id(unsigned long long *id) {
    typedef CUresult (*GetCurrent)(CUcontext *);
    typedef CUresult (*GetId)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked = false;
    if (!looked) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)f;
        looked = true;
    }
    if (!get_current) return cudaErrorNotSupported;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
    if (get_id && get_id(ctx, id) == CUDA_SUCCESS) return cudaSuccess;
    *id = (unsigned long long)(uintptr_t)ctx;
    return cudaSuccess;
}

// Device addresses of the arrays for the current device: looked up on the
// first call and again whenever the device's context has changed.
cudaError_t scratch_for(int dev, Scratch *out) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    Scratch &s = g_scratch[dev];
    unsigned long long id = 0;
    const cudaError_t have = current_ctx_id(&id);
    const bool checkable = have != cudaErrorNotSupported;  // no driver entry point: no check
    if (s.ready && checkable && (have != cudaSuccess || s.ctx_id != id)) s.ready = false;
    if (!s.ready) {
        cudaError_t e;
        if ((e = cudaGetSymbolAddress((void **)&s.spec, g_na_spec)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void **)&s.piv, g_na_piv)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void **)&s.rhs, g_na_rhs)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void **)&s.tw, g_na_tw)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void **)&s.wall, g_na_wall)) != cudaSuccess) return e;
        // the lookups above made the device's context current if it was not
        if (checkable && (e = current_ctx_id(&id)) != cudaSuccess) return e;
        s.ctx_id = id;
        s.ready = true;
    }
    *out = s;
    return cudaSuccess;
}

// Twiddles exp(-2 pi i k/nx) and the uniform wall rows.
__global__ void na_tables(int nx, double zlo, double zhi, double2 *tw, double *wall) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nx; k += gridDim.x * blockDim.x) {
        double sv, cv;
        sincospi(2.0 * (double)k / (double)nx, &sv, &cv);
        tw[k] = make_double2(cv, -sv);
        wall[k] = zlo;
        wall[nx + k] = zhi;
    }
}

// Pivots of the per-mode tridiagonal solve, one thread per x-mode:
// piv_0 = 1/b, piv_j = 1/(b - piv_{j-1}), b = -(2 + kx^2 dy^2), kx = 2 pi m/Lx.
__global__ void na_pivots(int nx, int n, int mp, double lx, double dy, double *piv) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m > nx / 2) return;
    const double kx = (double)m * 2.0 * 3.141592653589793 / lx;
    const double b = -(2.0 + kx * kx * dy * dy);
    double c = 0.0;
    for (int j = 0; j < n; ++j) {
        c = 1.0 / (b - c);
        piv[(size_t)j * mp + m] = c;
    }
}

// Right-hand side of the interior rows with the Dirichlet lifting
// (odd_extension, poisson.cu:228-241); pitch nx.
__global__ void na_rhs(int nx, int ny, double f_charge, double eps, double dy, double zlo, double zhi,
                       const double *__restrict__ cp, const double *__restrict__ cn, double *__restrict__ rhs) {
    const int x = blockIdx.x * NA_TPB + threadIdx.x;
    const int y = blockIdx.y + 1;
    if (x >= nx) return;
    const size_t o = (size_t)y * nx + x;
    double v = -f_charge * (cp[o] - cn[o]) / eps;
    if (y == 1) v = v - zlo / dy / dy;
    if (y == ny - 2) v = v - zhi / dy / dy;
    rhs[o] = v;
}

// E = -grad psi by central differences, periodic x, wall rows copy the
// adjacent Ey (gpu_efield + gpu_bc, poisson.cu:145-174); pitch nx.
__global__ void na_efield(int nx, int ny, double dx, double dy, const double *__restrict__ psi,
                          double *__restrict__ ex, double *__restrict__ ey) {
    const int x = blockIdx.x * NA_TPB + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= nx) return;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
    const int yc = y == 0 ? 1 : (y == ny - 1 ? ny - 2 : y);
    const size_t r = (size_t)y * nx;
    ex[r + x] = 0.5 * (psi[r + xm] - psi[r + xp]) / dx;
    ey[r + x] = 0.5 * (psi[(size_t)(yc - 1) * nx + x] - psi[(size_t)(yc + 1) * nx + x]) / dy;
}

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

int na_fail(int code, const char *msg) {
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace ek

using namespace ek;

extern "C" int ek_poisson_noalloc(const ek_params *p, const double *cp, const double *cn, double *psi, double *ex,
                                  double *ey, void *stream) {
    if (!p || !cp || !cn || !psi) return na_fail(EK_ERR_INVALID, "null argument");
    if ((ex == nullptr) != (ey == nullptr)) return na_fail(EK_ERR_INVALID, "give both ex and ey, or neither");
    const int nx = p->nx, ny = p->ny;
    if (nx < 2 || ny < 4) return na_fail(EK_ERR_INVALID, "need nx >= 2 and ny >= 4");
    const double pos[] = {p->dx, p->dy, p->lx};
    for (double v : pos)
        if (!(v > 0.0) || !std::isfinite(v)) return na_fail(EK_ERR_INVALID, "non-positive or non-finite dx, dy or lx");
    if (p->eps == 0.0 || !std::isfinite(p->eps) || !std::isfinite(p->f_charge) || !std::isfinite(p->zeta_lo) ||
        !std::isfinite(p->zeta_hi))
        return na_fail(EK_ERR_INVALID, "non-finite eps, f_charge or wall potential, or eps == 0");
    if (ny > 65535) return na_fail(EK_ERR_TOO_LARGE, "ek_poisson_noalloc: ny above 65535");
    if ((long long)nx * ny > EK_NOALLOC_MAX_NODES || (pow2(nx) ? nx > NA_MAX_NX : nx > 2048))
        return na_fail(EK_ERR_TOO_LARGE,
                       "ek_poisson_noalloc: nx*ny above 524288 nodes, or nx above 8192 (2048 if not a power of two)");
    const int n = ny - 2, mp = nx / 2 + 1;
    if ((long long)n * mp > EK_NOALLOC_MAX_NODES / 2 + 8192)
        return na_fail(EK_ERR_TOO_LARGE, "ek_poisson_noalloc: (ny-2)*(nx/2+1) spectrum above the scratch size");
    cudaStream_t s = (cudaStream_t)stream;
    (void)cudaGetLastError();  // a launch error left by the caller's earlier work is not this call's
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return na_fail(EK_ERR_CUDA, "cudaGetDevice");
    Scratch sc;
    if ((e = scratch_for(dev, &sc)) != cudaSuccess) return na_fail(EK_ERR_CUDA, cudaGetErrorString(e));
    if ((e = poisson_set_smem_limits()) != cudaSuccess) return na_fail(EK_ERR_CUDA, cudaGetErrorString(e));

    PoissonPlan pp{};
    pp.nx = nx;
    pp.ny = ny;
    pp.n = n;
    pp.mp = mp;
    pp.pow2 = pow2(nx);
    int lg = 0;
    while ((1 << lg) < nx) ++lg;
    pp.log2nx = pp.pow2 ? lg : 0;
    pp.dy2 = p->dy * p->dy;
    pp.tw = sc.tw;
    pp.piv = sc.piv;
    pp.spec = sc.spec;
    Chan c{};
    c.nx = nx;
    c.ny = ny;
    c.nxp = nx;
    c.plane = (size_t)nx * ny;
    c.zlo = sc.wall;
    c.zhi = sc.wall + nx;

    const dim3 rows((nx + NA_TPB - 1) / NA_TPB, ny - 2);
    const dim3 all((nx + NA_TPB - 1) / NA_TPB, ny);
    e = cudaMemsetAsync(sc.spec, 0, (size_t)n * mp * sizeof(double2), s);
    if (e == cudaSuccess) {
        na_tables<<<(nx + 255) / 256, 256, 0, s>>>(nx, p->zeta_lo, p->zeta_hi, sc.tw, sc.wall);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        na_pivots<<<(mp + 127) / 128, 128, 0, s>>>(nx, n, mp, p->lx, p->dy, sc.piv);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        na_rhs<<<rows, NA_TPB, 0, s>>>(nx, ny, p->f_charge, p->eps, p->dy, p->zeta_lo, p->zeta_hi, cp, cn, sc.rhs);
        e = cudaGetLastError();
    }
    for (int pass = 0; pass < 3 && e == cudaSuccess; ++pass) e = poisson_pass_f64_at(pass, pp, c, sc.rhs, psi, s);
    if (e == cudaSuccess && ex) {
        na_efield<<<all, NA_TPB, 0, s>>>(nx, ny, p->dx, p->dy, psi, ex, ey);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return na_fail(EK_ERR_CUDA, cudaGetErrorString(e));
    return EK_OK;
}
