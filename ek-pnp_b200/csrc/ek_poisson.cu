// ek_poisson.cu -- spectral Poisson solve of the reference's discretisation.
//
// The reference (fast_Poisson, poisson.cu:180-306) odd-extends the interior
// rows to ne = 2(ny-1) rows, runs a 2D complex FFT (cuFFT), divides by
//     mu = kx^2 + (4/dy^2) sin^2(ky dy/2),  kx = 2 pi m/Lx,  ky = 2 pi n/(ne dy)
// and transforms back.  Along y the odd extension makes this a sine transform,
// and (4/dy^2) sin^2(n pi/(2(ny-1))) are exactly the eigenvalues of the
// three-point Dirichlet Laplacian on the ny-2 interior rows.  So, for every
// x-mode m, the reference solves the tridiagonal system
//     phi_{j-1} - (2 + kx_m^2 dy^2) phi_j + phi_{j+1} = dy^2 S_j,  phi_{-1} = phi_{n} = 0
// and this file solves it directly (Thomas recurrence with pivots computed
// once per channel), for any ny, with no FFT in y:
//   pass A  per pair of interior rows: real FFT in x (two rows packed as one
//           complex row, radix-2 in shared memory; direct DFT when nx is not
//           a power of two) -> spec[j][m], m = 0..nx/2
//   pass B  per x-mode m: forward/backward Thomas sweep down the column
//   pass C  per pair of rows: inverse real FFT -> psi; wall rows = zeta(x)
// The result equals the reference's to rounding (the test suite compares).
#include <cuda_runtime.h>

#include "ek_internal.h"

namespace ek {
namespace {

constexpr int PTPB = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// In-place radix-2 decimation-in-time FFT of n = 2^lg points already in
// bit-reversed order in shared memory.  inv selects the +i exponent.
__device__ void fft_smem(double2 *s, int n, const double2 *__restrict__ tw, bool inv) {
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, stride = n / len;
        for (int t = threadIdx.x; t < (n >> 1); t += blockDim.x) {
            const int k = t & (half - 1);
            const int i = (t - k) * 2 + k;
            double2 w = __ldg(tw + k * stride);
            if (inv) w = cconj(w);
            const double2 u = s[i], v = cmul(s[i + half], w);
            s[i] = cadd(u, v);
            s[i + half] = csub(u, v);
        }
        __syncthreads();
    }
}

// Direct DFT of z (n points, any n) into out, both in shared memory.
__device__ void dft_smem(const double2 *z, double2 *out, int n, const double2 *__restrict__ tw, bool inv) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        int idx = 0;
        for (int x = 0; x < n; ++x) {
            double2 w = __ldg(tw + idx);
            if (inv) w = cconj(w);
            acc = cadd(acc, cmul(z[x], w));
            idx += m;
            if (idx >= n) idx -= n;
        }
        out[m] = acc;
    }
    __syncthreads();
}

// Pass A: rows y0 = 2*b+1 and y1 = y0+1 of the right-hand side -> spectra.
__global__ void __launch_bounds__(PTPB)
fwd_rows(const PoissonPlan pp, const double *__restrict__ rhs, int nxp) {
    extern __shared__ double2 sm[];
    const int nx = pp.nx;
    const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
    const bool two = j1 < pp.n;
    const double *r0 = rhs + (size_t)(j0 + 1) * nxp;
    const double *r1 = rhs + (size_t)(j1 + 1) * nxp;
    double2 *z = sm;
    if (pp.pow2) {
        const int sh = 32 - pp.log2nx;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            const int rx = pp.log2nx ? (int)(__brev((unsigned)x) >> sh) : 0;
            z[rx] = make_double2(r0[x], two ? r1[x] : 0.0);
        }
        __syncthreads();
        fft_smem(z, nx, pp.tw, false);
    } else {
        double2 *in = sm + nx;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) in[x] = make_double2(r0[x], two ? r1[x] : 0.0);
        __syncthreads();
        dft_smem(in, z, nx, pp.tw, false);
    }
    // unpack the two real-input spectra: A = (Z[m] + conj Z[-m])/2, B = (Z[m] - conj Z[-m])/(2i)
    double2 *s0 = pp.spec + (size_t)j0 * pp.mp, *s1 = pp.spec + (size_t)j1 * pp.mp;
    for (int m = threadIdx.x; m <= nx / 2; m += blockDim.x) {
        const double2 a = z[m], b = cconj(z[m == 0 ? 0 : nx - m]);
        s0[m] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        if (two) s1[m] = make_double2(0.5 * (a.y - b.y), -0.5 * (a.x - b.x));
    }
}

// Pass B: one thread per x-mode, Thomas sweep over the n interior rows.
// piv[j][m] = 1/(b_m - piv[j-1][m]) with b_m = -(2 + kx_m^2 dy^2).
__global__ void __launch_bounds__(PTPB) tridiag(const PoissonPlan pp) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m > pp.nx / 2) return;
    const size_t mp = pp.mp;
    double2 *col = pp.spec + m;
    const double *pv = pp.piv + m;
    const double dy2 = pp.dy2;
    double2 d = make_double2(0.0, 0.0);
    for (int j = 0; j < pp.n; ++j) {
        const double2 sj = col[j * mp];
        const double c = __ldg(pv + j * mp);
        d = make_double2((dy2 * sj.x - d.x) * c, (dy2 * sj.y - d.y) * c);
        col[j * mp] = d;
    }
    double2 xn = d;
    for (int j = pp.n - 2; j >= 0; --j) {
        const double2 dj = col[j * mp];
        const double c = __ldg(pv + j * mp);
        xn = make_double2(dj.x - c * xn.x, dj.y - c * xn.y);
        col[j * mp] = xn;
    }
}

// Pass C: spectra of rows (y0, y1) -> psi rows; block 0 also writes the walls.
__global__ void __launch_bounds__(PTPB)
inv_rows(const PoissonPlan pp, const Chan c, double *__restrict__ psi) {
    extern __shared__ double2 sm[];
    const int nx = pp.nx, nxp = c.nxp;
    const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
    const bool two = j1 < pp.n;
    const double2 *s0 = pp.spec + (size_t)j0 * pp.mp, *s1 = pp.spec + (size_t)j1 * pp.mp;
    double2 *z = sm;
    double2 *dst = pp.pow2 ? sm : sm + nx;
    const int sh = 32 - pp.log2nx;
    for (int m = threadIdx.x; m <= nx / 2; m += blockDim.x) {
        const double2 a = s0[m];
        const double2 b = two ? s1[m] : make_double2(0.0, 0.0);
        // Z[m] = A + iB, Z[-m] = conj(A) + i conj(B)
        const double2 zp = make_double2(a.x - b.y, a.y + b.x);
        const double2 zn = make_double2(a.x + b.y, -a.y + b.x);
        if (pp.pow2) {
            z[pp.log2nx ? (int)(__brev((unsigned)m) >> sh) : 0] = zp;
            if (m != 0 && 2 * m != nx) z[(int)(__brev((unsigned)(nx - m)) >> sh)] = zn;
        } else {
            dst[m] = zp;
            if (m != 0 && 2 * m != nx) dst[nx - m] = zn;
        }
    }
    __syncthreads();
    if (pp.pow2) fft_smem(z, nx, pp.tw, true);
    else dft_smem(dst, z, nx, pp.tw, true);
    const double inv = 1.0 / (double)nx;
    double *p0 = psi + (size_t)(j0 + 1) * nxp, *p1 = psi + (size_t)(j1 + 1) * nxp;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        p0[x] = z[x].x * inv;
        if (two) p1[x] = z[x].y * inv;
    }
    if (blockIdx.x == 0) {
        // wall rows hold the wall potential (odd_extract, poisson.cu:297-304)
        double *lo = psi, *hi = psi + (size_t)(c.ny - 1) * nxp;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            lo[x] = c.zlo[x];
            hi[x] = c.zhi[x];
        }
    }
}

}  // namespace

size_t poisson_smem_bytes_f64(int nx) {
    const bool pow2 = nx > 0 && (nx & (nx - 1)) == 0;
    return (size_t)nx * sizeof(double2) * (pow2 ? 1 : 2);
}

cudaError_t poisson_pass_f64(int pass, const PoissonPlan &pp, const Chan &c, double *fields, cudaStream_t s) {
    const size_t smem = poisson_smem_bytes_f64(pp.nx);
    const int rows2 = (pp.n + 1) / 2;
    if (pass == 0) fwd_rows<<<rows2, PTPB, smem, s>>>(pp, fields + F_RHS * c.plane, c.nxp);
    else if (pass == 1) tridiag<<<(pp.nx / 2 + 1 + PTPB - 1) / PTPB, PTPB, 0, s>>>(pp);
    else inv_rows<<<rows2, PTPB, smem, s>>>(pp, c, fields + F_PSI * c.plane);
    return cudaGetLastError();
}

cudaError_t poisson_pass_f64_at(int pass, const PoissonPlan &pp, const Chan &c, const double *rhs, double *psi,
                                cudaStream_t s) {
    const size_t smem = poisson_smem_bytes_f64(pp.nx);
    const int rows2 = (pp.n + 1) / 2;
    if (pass == 0) fwd_rows<<<rows2, PTPB, smem, s>>>(pp, rhs, c.nxp);
    else if (pass == 1) tridiag<<<(pp.nx / 2 + 1 + PTPB - 1) / PTPB, PTPB, 0, s>>>(pp);
    else inv_rows<<<rows2, PTPB, smem, s>>>(pp, c, psi);
    return cudaGetLastError();
}

cudaError_t poisson_set_smem_limits() {
    cudaError_t e = cudaFuncSetAttribute(fwd_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(inv_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

}  // namespace ek
