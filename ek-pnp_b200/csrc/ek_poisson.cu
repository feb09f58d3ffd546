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
//           complex row; register-blocked radix-16 passes for powers of two,
//           direct DFT otherwise) -> spec[j][m], m = 0..nx/2
//   pass B  per x-mode m: Thomas sweeps down the column, partitioned into row
//           segments of at most 16 rows held in registers (one thread per
//           mode for columns taller than 8192 rows)
//   pass C  per pair of rows: inverse real FFT -> psi; wall rows = zeta(x)
// The result equals the reference's to rounding (the test suite compares).
#include <cuda_runtime.h>

#include "ek_fft32.cuh"
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
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cmake(double a, double b);
template <> __device__ __forceinline__ double2 cmake<double2>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 cmake<float2>(double a, double b) { return make_float2((float)a, (float)b); }

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

// Wall rows psi[0] = zlo, psi[ny-1] = zhi (odd_extract, poisson.cu:297-304),
// spread over the nb blocks of one channel's inverse pass (lb = this block's
// index among them, bs threads a block) and issued at the start of the
// pass: one block writing both rows alone made a chain of dependent loads
// that outlasted the rest of the pass.
__device__ __forceinline__ void write_walls(double *__restrict__ psi, const double *__restrict__ zlo,
                                            const double *__restrict__ zhi, int nx, int ny, int nxp, int lb,
                                            int nb, int bs) {
    double *lo = psi, *hi = psi + (size_t)(ny - 1) * nxp;
    for (int g = lb * bs + (int)threadIdx.x; g < 2 * nx; g += nb * bs) {
        if (g < nx) lo[g] = __ldg(zlo + g);
        else hi[g - nx] = __ldg(zhi + g - nx);
    }
}

// Pass C: spectra of rows (y0, y1) -> psi rows; the walls spread over the blocks.
__global__ void __launch_bounds__(PTPB)
inv_rows(const PoissonPlan pp, const Chan c, double *__restrict__ psi) {
    extern __shared__ double2 sm[];
    const int nx = pp.nx, nxp = c.nxp;
    write_walls(psi, c.zlo, c.zhi, nx, c.ny, nxp, blockIdx.x, gridDim.x, blockDim.x);
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
}

// ---- register-blocked radix-16 row FFTs (power-of-two nx >= 16) ----------
//
// Each thread holds up to 16 complex values and runs up to four radix-2
// stages on them in registers per pass; passes exchange through shared
// memory.  The forward transform is decimation in frequency on natural-order
// input (bit-reversed output); the inverse is decimation in time on
// bit-reversed input (natural-order output).  A pass over index bits
// [b, b+RB) owns the 2^RB elements that share every other index bit; thread t
// of the T = nx/16 threads of one transform owns 16/2^RB such groups.
// Twiddle of stage st for element index i: exp(-2 pi i (i mod 2^st)/2^(st+1))
// = A * C with A = exp(-2 pi i (base mod 2^b)/2^(st+1)) from the table (one
// load per group and stage) and C = exp(-2 pi i v_low/2^(st-b+1)) a constant
// root of unity of order <= 16 for the in-register index bits v_low.
// Shared memory is addressed through swz(): the low three index bits are
// XOR-ed with bits 4..6 and with the reversed top three bits, which keeps
// both the passes and the bit-reversed unpacking free of bank conflicts.

__device__ __forceinline__ int brev(int i, int lg) { return (int)(__brev((unsigned)i) >> (32 - lg)); }
__device__ __forceinline__ int swz(int i, int k) {
    if (k < 6) return i;
    const int top = (i >> (k - 3)) & 7;
    const int rtop = ((top & 1) << 2) | (top & 2) | ((top >> 2) & 1);
    return i ^ (((i >> 4) ^ rtop) & 7);
}

// Shared-memory index of element i of a transform (the FP64 form; the FP32
// row transforms of ek_fft32.cuh have their own map).
template <typename C> __device__ __forceinline__ int sidx(int i, int k, int p);
template <> __device__ __forceinline__ int sidx<double2>(int i, int k, int) { return swz(i, k); }

// exp(-2 pi i v/2^(sl+1)) for 0 <= v < 2^sl <= 8 (compile-time arguments)
template <typename C>
__device__ __forceinline__ C root16(int sl, int v) {
    const int q = v << (3 - sl);  // angle = q * pi/8
    switch (q) {
        case 0: return cmake<C>(1.0, 0.0);
        case 1: return cmake<C>(0.92387953251128674, -0.38268343236508977);
        case 2: return cmake<C>(0.70710678118654752, -0.70710678118654752);
        case 3: return cmake<C>(0.38268343236508977, -0.92387953251128674);
        case 4: return cmake<C>(0.0, -1.0);
        case 5: return cmake<C>(-0.38268343236508977, -0.92387953251128674);
        case 6: return cmake<C>(-0.70710678118654752, -0.70710678118654752);
        default: return cmake<C>(-0.92387953251128674, -0.38268343236508977);
    }
}

template <bool INV, int RB, typename C>
__device__ __forceinline__ void reg_pass(C *s, int k, int T, int t, int b, const C *__restrict__ tw, int p) {
    constexpr int G = 16 >> RB, E = 1 << RB;
    const int ngroups = (1 << k) >> RB;
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int g = t + q * T;
        if (g >= ngroups) continue;
        const int kb = g & ((1 << b) - 1);
        const int base = kb | ((g >> b) << (b + RB));
        C r[E];
#pragma unroll
        for (int v = 0; v < E; ++v) r[v] = s[sidx<C>(base | (v << b), k, p)];
        if (!INV) {
#pragma unroll
            for (int sl = RB - 1; sl >= 0; --sl) {
                const int st = b + sl;
                const C A = __ldg(tw + (kb << (k - st - 1)));
#pragma unroll
                for (int v = 0; v < E; ++v) {
                    if (v & (1 << sl)) continue;
                    const C w = cmul(A, root16<C>(sl, v & ((1 << sl) - 1)));
                    const C u = r[v], x = r[v + (1 << sl)];
                    r[v] = cadd(u, x);
                    r[v + (1 << sl)] = cmul(csub(u, x), w);
                }
            }
        } else {
#pragma unroll
            for (int sl = 0; sl < RB; ++sl) {
                const int st = b + sl;
                const C A = cconj(__ldg(tw + (kb << (k - st - 1))));
#pragma unroll
                for (int v = 0; v < E; ++v) {
                    if (v & (1 << sl)) continue;
                    const C w = cmul(A, cconj(root16<C>(sl, v & ((1 << sl) - 1))));
                    const C u = r[v], x = cmul(r[v + (1 << sl)], w);
                    r[v] = cadd(u, x);
                    r[v + (1 << sl)] = csub(u, x);
                }
            }
        }
#pragma unroll
        for (int v = 0; v < E; ++v) s[sidx<C>(base | (v << b), k, p)] = r[v];
    }
}

template <bool INV, typename C>
__device__ __forceinline__ void reg_pass_any(C *s, int k, int T, int t, int b, int rb, const C *tw, int p) {
    switch (rb) {
        case 4: reg_pass<INV, 4, C>(s, k, T, t, b, tw, p); break;
        case 3: reg_pass<INV, 3, C>(s, k, T, t, b, tw, p); break;
        case 2: reg_pass<INV, 2, C>(s, k, T, t, b, tw, p); break;
        default: reg_pass<INV, 1, C>(s, k, T, t, b, tw, p); break;
    }
}

// Whole transform of 2^k points in s; every thread of the block calls it.
template <bool INV, typename C>
__device__ void reg_fft(C *s, int k, int T, int t, const C *__restrict__ tw, int p) {
    if (!INV) {
        for (int top = k; top > 0;) {
            const int rb = top < 4 ? top : 4;
            reg_pass_any<false, C>(s, k, T, t, top - rb, rb, tw, p);
            __syncthreads();
            top -= rb;
        }
    } else {
        for (int b = 0; b < k;) {
            const int rb = k - b < 4 ? k - b : 4;
            reg_pass_any<true, C>(s, k, T, t, b, rb, tw, p);
            __syncthreads();
            b += rb;
        }
    }
}

// Pass A, radix-16 form: row pairs (2p+1, 2p+2) of the right-hand side ->
// spectra.  One block holds BLOCK/T row pairs.
template <int BLOCK>
__device__ __forceinline__ void fwd_rows_r16_dev(const PoissonPlan &pp, const double *__restrict__ rhs, int nxp,
                                                 int pair_base, double2 *sm) {
    const int N = pp.nx, k = pp.log2nx, T = N >> 4;
    const int p = threadIdx.x / T, t = threadIdx.x - p * T;
    const int pair = pair_base + p;
    double2 *s = sm + p * N;
    const int j0 = 2 * pair, j1 = j0 + 1;
    const bool live = j0 < pp.n, two = j1 < pp.n;
    const double *r0 = rhs + (size_t)(j0 + 1) * nxp, *r1 = rhs + (size_t)(j1 + 1) * nxp;
    for (int x = t; x < N; x += T)
        s[swz(x, k)] = live ? make_double2(__ldg(r0 + x), two ? __ldg(r1 + x) : 0.0) : make_double2(0.0, 0.0);
    __syncthreads();
    reg_fft<false, double2>(s, k, T, t, pp.tw, p);
    if (!live) return;
    double2 *s0 = pp.spec + (size_t)j0 * pp.mp, *s1 = pp.spec + (size_t)j1 * pp.mp;
    for (int m = t; m <= N / 2; m += T) {
        const double2 a = s[swz(brev(m, k), k)], b = cconj(s[swz(brev((N - m) & (N - 1), k), k)]);
        s0[m] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        if (two) s1[m] = make_double2(0.5 * (a.y - b.y), -0.5 * (a.x - b.x));
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK)
fwd_rows_r16(const PoissonPlan pp, const double *__restrict__ rhs, int nxp) {
    extern __shared__ double2 sm[];
    fwd_rows_r16_dev<BLOCK>(pp, rhs, nxp, blockIdx.x * (BLOCK / (pp.nx >> 4)), sm);
}

// Pass C, radix-16 form: spectra -> psi rows and the walls.
template <int BLOCK>
__device__ __forceinline__ void inv_rows_r16_dev(const PoissonPlan &pp, int nxp, int ny, const double *zlo,
                                                 const double *zhi, double *__restrict__ psi, int pair_base,
                                                 double2 *sm) {
    const int N = pp.nx, k = pp.log2nx, T = N >> 4;
    const int p = threadIdx.x / T, t = threadIdx.x - p * T;
    const int pair = pair_base + p;
    double2 *s = sm + p * N;
    const int j0 = 2 * pair, j1 = j0 + 1;
    const bool live = j0 < pp.n, two = j1 < pp.n;
    const int per = BLOCK / T;
    write_walls(psi, zlo, zhi, N, ny, nxp, pair_base / per, ((pp.n + 1) / 2 + per - 1) / per, BLOCK);
    const double2 *s0 = pp.spec + (size_t)j0 * pp.mp, *s1 = pp.spec + (size_t)j1 * pp.mp;
    for (int m = t; m <= N / 2; m += T) {
        const double2 a = live ? s0[m] : make_double2(0.0, 0.0);
        const double2 b = two ? s1[m] : make_double2(0.0, 0.0);
        s[swz(brev(m, k), k)] = make_double2(a.x - b.y, a.y + b.x);  // A + iB
        if (m != 0 && 2 * m != N) s[swz(brev(N - m, k), k)] = make_double2(a.x + b.y, -a.y + b.x);
    }
    __syncthreads();
    reg_fft<true, double2>(s, k, T, t, pp.tw, p);
    const double inv = 1.0 / (double)N;
    if (live) {
        double *p0 = psi + (size_t)(j0 + 1) * nxp, *p1 = psi + (size_t)(j1 + 1) * nxp;
        for (int x = t; x < N; x += T) {
            const double2 z = s[swz(x, k)];
            p0[x] = z.x * inv;
            if (two) p1[x] = z.y * inv;
        }
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK)
inv_rows_r16(const PoissonPlan pp, const Chan c, double *__restrict__ psi) {
    extern __shared__ double2 sm[];
    inv_rows_r16_dev<BLOCK>(pp, c.nxp, c.ny, c.zlo, c.zhi, psi, blockIdx.x * (BLOCK / (pp.nx >> 4)), sm);
}

// ---- FP32 form of passes A and C ------------------------------------------
// The row is split into its mean (FP64: the zero mode) and the fluctuation
// about it, which is transformed in FP32.  The zero mode of every row is
// kept in column 0 of the FP64 spectrum; modes 1..nx/2 go to the FP32
// spectrum.

// Sum of v over the T threads of one transform group (T a power of two,
// groups contiguous in the block); every thread of the block calls it and
// gets the group's first lane's (or the block-level) value.
template <int BLOCK>
__device__ __forceinline__ double group_sum(double v, int T, double *red) {
    const int w = T < 32 ? T : 32;
    for (int o = w >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (T < 32) return __shfl_sync(0xffffffffu, v, (threadIdx.x & 31) & ~(T - 1));
    v = __shfl_sync(0xffffffffu, v, 0);
    if (T == 32) return v;
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int nw = T >> 5, g0 = (int)(threadIdx.x / T) * nw;
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += red[g0 + i];
    __syncthreads();
    return s;
}

// Pass A of the FP32 form for 2^K-point rows: the FP64 row sums (the zero
// mode) and the FP32 transform of the fluctuation about an offset (it only
// moves the unused FP32 zero bin; a close one keeps the rounding small).
// A row's right-hand side is rhsf plus, in FP64, the row constant: rhs_q
// (R+ - R-) of the row references and, on rows 1 and ny-2, the x-mean of the
// Dirichlet lifting -zeta/dy^2 (odd_extension, poisson.cu:228-241; its
// x-fluctuation is in rhsf).
// From the second solve on the offset is the previous solve's row mean and
// one pass over the row does both; the first solve takes two passes and the
// exact mean.  The first radix-16 pass runs on the values as loaded.
template <int BLOCK, int K>
__device__ __forceinline__ void fwd_rows_f32_k(const PoissonPlan &pp, const Chan &c, int pair_base, float2 *sm,
                                               double *red) {
    using S = fft32::Shape<K>;
    constexpr int N = S::N, T = S::T;
    const int p = threadIdx.x / T, t = threadIdx.x - p * T;
    const int pair = pair_base + p;
    float2 *s = sm + p * N;
    const int j0 = 2 * pair, j1 = j0 + 1;
    const bool live = j0 < pp.n, two = j1 < pp.n;
    const int nxp = c.nxp;
    // 32-bit offsets from the planes' base pointers (a plane is below 2^32
    // elements: one channel's planes fit device memory)
    const unsigned r0 = (unsigned)(j0 + 1) * (unsigned)nxp + (unsigned)t, r1 = r0 + (unsigned)nxp;
    const double k0 = live ? rhs_row_constant(pp, c, j0 + 1) : 0.0, k1 = two ? rhs_row_constant(pp, c, j1 + 1) : 0.0;
    const bool exact = *pp.rowmean_ok == 0;  // the same for every block of the launch
    // value - offset = rhsf + (row constant - offset)
    double d0 = (live && !exact) ? k0 - pp.rowmean[j0] : 0.0, d1 = (two && !exact) ? k1 - pp.rowmean[j1] : 0.0;
    double a0 = 0.0, a1 = 0.0;
    float2 x[16];
#pragma unroll
    for (int v = 0; v < 16; ++v) {
        const float f0 = live ? __ldg(pp.rhsf + (r0 + (unsigned)(v * T))) : 0.0f,
                    f1 = two ? __ldg(pp.rhsf + (r1 + (unsigned)(v * T))) : 0.0f;
        a0 += (double)f0;
        a1 += (double)f1;
        x[v] = make_float2((float)((double)f0 + d0), (float)((double)f1 + d1));
    }
    a0 = group_sum<BLOCK>(a0, T, red) + (double)N * k0;
    a1 = group_sum<BLOCK>(a1, T, red) + (double)N * k1;
    if (exact) {
        d0 = k0 - a0 / (double)N;
        d1 = k1 - a1 / (double)N;
#pragma unroll
        for (int v = 0; v < 16; ++v)
            x[v] = make_float2(live ? (float)((double)__ldg(pp.rhsf + (r0 + (unsigned)(v * T))) + d0) : 0.0f,
                               two ? (float)((double)__ldg(pp.rhsf + (r1 + (unsigned)(v * T))) + d1) : 0.0f);
    }
    if (t == 0 && live) {
        pp.spec[(size_t)j0 * pp.mp] = make_double2(a0, 0.0);
        pp.rowmean[j0] = a0 / (double)N;
        if (two) {
            pp.spec[(size_t)j1 * pp.mp] = make_double2(a1, 0.0);
            pp.rowmean[j1] = a1 / (double)N;
        }
    }
    fft32::fwd_pass_store<K, 1>(x, s, t, p, pp.twf);
    __syncthreads();
    fft32::fwd_rest<K, 2>(s, t, p, pp.twf);
    if (!live) return;
    const unsigned q0 = (unsigned)j0 * (unsigned)pp.mp, q1 = q0 + (unsigned)pp.mp;
    for (int m = t; m <= N / 2; m += T) {
        if (m == 0) continue;
        const float2 a = s[fft32::swz_base(brev(m, K), p)], b = cconj(s[fft32::swz_base(brev(N - m, K), p)]);
        pp.specf[q0 + (unsigned)m] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
        if (two) pp.specf[q1 + (unsigned)m] = make_float2(0.5f * (a.y - b.y), -0.5f * (a.x - b.x));
    }
}

// Wall rows of the FP32 form's psi: psim = the x-mean of the wall potential,
// psif = the potential minus it (zero for uniform walls), the FP64 plane's
// Dirichlet values too when write_f64; spread over the nb blocks of the pass.
__device__ __forceinline__ void write_walls_f32(const PoissonPlan &pp, const Chan &c, double *__restrict__ psi,
                                                bool write_f64, int lb, int nb, int bs) {
    const int nx = c.nx, ny = c.ny;
    float *flo = pp.psif, *fhi = pp.psif + (size_t)(ny - 1) * c.nxp;
    double *dlo = psi, *dhi = psi + (size_t)(ny - 1) * c.nxp;
    for (int g = lb * bs + (int)threadIdx.x; g < 2 * nx; g += nb * bs) {
        const bool low = g < nx;
        const int x = low ? g : g - nx;
        const double z = __ldg((low ? c.zlo : c.zhi) + x);
        (low ? flo : fhi)[x] = (float)(z - (low ? pp.zlo_mean : pp.zhi_mean));
        if (write_f64) (low ? dlo : dhi)[x] = z;
    }
    if (lb == 0 && threadIdx.x == 0) {
        pp.psim[0] = pp.zlo_mean;
        pp.psim[ny - 1] = pp.zhi_mean;
    }
}

// Pass C of the FP32 form: the two real rows' spectra packed as A + iB, the
// inverse transform; psif = the FP32 fluctuation / N (stored from registers by
// the last radix-16 pass), psim = the FP64 row mean, and the FP64 psi plane
// (mean + fluctuation) when write_f64.
template <int BLOCK, int K>
__device__ __forceinline__ void inv_rows_f32_k(const PoissonPlan &pp, const Chan &c, double *__restrict__ psi,
                                               bool write_f64, int pair_base, float2 *sm) {
    using S = fft32::Shape<K>;
    constexpr int N = S::N, T = S::T;
    const int p = threadIdx.x / T, t = threadIdx.x - p * T;
    const int pair = pair_base + p;
    float2 *s = sm + p * N;
    const int j0 = 2 * pair, j1 = j0 + 1;
    const bool live = j0 < pp.n, two = j1 < pp.n;
    const int nxp = c.nxp;
    constexpr int per = BLOCK / T;
    write_walls_f32(pp, c, psi, write_f64, pair_base / per, ((pp.n + 1) / 2 + per - 1) / per, BLOCK);
    // 32-bit offsets from the planes' base pointers (as in fwd_rows_f32_k)
    const unsigned q0 = (unsigned)j0 * (unsigned)pp.mp, q1 = q0 + (unsigned)pp.mp;
    // modes m = t + i T (i < 8) and, for t = 0, m = N/2: all loads first
    const float2 zero = make_float2(0.0f, 0.0f);
    float2 a[9], b[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int m = t + i * T;
        const bool in = i < 8 || t == 0;
        a[i] = (live && in && m) ? pp.specf[q0 + (unsigned)m] : zero;
        b[i] = (two && in && m) ? pp.specf[q1 + (unsigned)m] : zero;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int m = t + i * T;
        if (i == 8 && t != 0) break;
        s[fft32::swz_base(brev(m, K), p)] = make_float2(a[i].x - b[i].y, a[i].y + b[i].x);  // A + iB
        if (m != 0 && 2 * m != N)
            s[fft32::swz_base(brev(N - m, K), p)] = make_float2(a[i].x + b[i].y, -a[i].y + b[i].x);
    }
    __syncthreads();
    fft32::inv_partial<K>(s, t, p);
    fft32::inv_full<K, S::NF>(s, t, p, pp.twf);
    float2 x[16];
    fft32::inv_pass_load<K, 1>(x, s, t, p, pp.twf);
    const double inv = 1.0 / (double)N;
    const float invf = 1.0f / (float)N;  // a power of two: exact
    if (pair_base == 0 && threadIdx.x == 0) *pp.rowmean_ok = 1;
    if (live) {
        const double mean0 = pp.spec[(size_t)j0 * pp.mp].x * inv;
        const double mean1 = two ? pp.spec[(size_t)j1 * pp.mp].x * inv : 0.0;
        if (t == 0) {
            pp.psim[j0 + 1] = mean0;
            if (two) pp.psim[j1 + 1] = mean1;
        }
        const unsigned o0 = (unsigned)(j0 + 1) * (unsigned)nxp + (unsigned)t, o1 = o0 + (unsigned)nxp;
#pragma unroll
        for (int v = 0; v < 16; ++v) {
            const float y0 = x[v].x * invf, y1 = x[v].y * invf;
            const unsigned dv = (unsigned)(v * T);
            st_field_f(pp.psif + (o0 + dv), y0, pp.keep_l2);
            if (two) st_field_f(pp.psif + (o1 + dv), y1, pp.keep_l2);
            if (write_f64) {
                psi[o0 + dv] = mean0 + (double)y0;
                if (two) psi[o1 + dv] = mean1 + (double)y1;
            }
        }
    }
}

// Transform sizes a block of BLOCK threads runs: 256 threads take every
// 16 <= nx <= 4096 (several row pairs a block below 4096), 512 threads one
// row pair of nx = 8192.
template <int BLOCK, int K> __host__ __device__ constexpr bool r16f_fits() {
    return BLOCK == 256 ? (K >= 4 && K <= 12) : ((1 << K) >> 4) == BLOCK;
}

#define EK_R16F_CASES(F) F(4) F(5) F(6) F(7) F(8) F(9) F(10) F(11) F(12) F(13)

template <int BLOCK>
__device__ __forceinline__ void fwd_rows_r16f_dev(const PoissonPlan &pp, const Chan &c, int pair_base, float2 *sm,
                                                  double *red) {
    switch (pp.log2nx) {
#define EK_CASE(K)                                                                        \
    case K:                                                                               \
        if constexpr (r16f_fits<BLOCK, K>()) fwd_rows_f32_k<BLOCK, K>(pp, c, pair_base, sm, red); \
        break;
        EK_R16F_CASES(EK_CASE)
#undef EK_CASE
        default: break;
    }
}

template <int BLOCK>
__device__ __forceinline__ void inv_rows_r16f_dev(const PoissonPlan &pp, const Chan &c, double *__restrict__ psi,
                                                  bool write_f64, int pair_base, float2 *sm) {
    switch (pp.log2nx) {
#define EK_CASE(K)                                                                                    \
    case K:                                                                                           \
        if constexpr (r16f_fits<BLOCK, K>()) inv_rows_f32_k<BLOCK, K>(pp, c, psi, write_f64, pair_base, sm); \
        break;
        EK_R16F_CASES(EK_CASE)
#undef EK_CASE
        default: break;
    }
}

// 4 blocks of 256 threads per SM: the 511 row pairs of a 4096 x 1024 channel
// then run in one wave (3 blocks per SM leave a second, nearly empty wave).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
fwd_rows_r16f(const PoissonPlan pp, const Chan c) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[BLOCK / 32];
    fwd_rows_r16f_dev<BLOCK>(pp, c, blockIdx.x * (BLOCK / (pp.nx >> 4)), (float2 *)smraw, red);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
inv_rows_r16f(const PoissonPlan pp, const Chan c, double *__restrict__ psi, bool write_f64) {
    extern __shared__ __align__(16) unsigned char smraw[];
    inv_rows_r16f_dev<BLOCK>(pp, c, psi, write_f64, blockIdx.x * (BLOCK / (pp.nx >> 4)), (float2 *)smraw);
}

// ---- pass B, partitioned Thomas solve ------------------------------------
//
// A block owns M consecutive x-modes; its 512 threads are S = 512/M row
// segments x M modes, each segment at most 16 rows (M is chosen so), held in
// registers with its pivots.  The forward recurrence
// d_j = (dy^2 S_j - d_{j-1}) piv_j is linear in the value entering a segment,
// so each segment first runs with a zero entry value while accumulating the
// product of (-piv); the true entry values follow from composing the
// segments' affine maps D -> e + f D in order, a log2(S)-round scan over the
// segments of each mode in shared memory, and each segment adds its
// correction.  The backward recurrence x_j = d_j - piv_j x_{j+1} is split the
// same way.  The result is the Thomas solution, reassociated.
constexpr int TB_THREADS = 512;
constexpr int TB_L = 16;

template <typename R, typename C> struct TridiagSharedT {
    C ends[TB_THREADS];
    R mults[TB_THREADS];
};
using TridiagShared = TridiagSharedT<double, double2>;

// Value entering this thread's segment: the affine maps D -> e + f D of the
// segments of its mode (the block's threads are seg * M + mode) composed in
// order -- forward from segment 0 (FWD) or backward from segment S-1 -- by a
// Kogge-Stone scan over the S segments in shared memory (log2 S rounds); the
// first segment in that order enters with 0.  Every thread of the block
// calls it.
template <bool FWD, typename R, typename C>
__device__ __forceinline__ C seg_carry(C e, R f, int seg, int S, int M, TridiagSharedT<R, C> &sh) {
    const int tid = threadIdx.x, mode = tid - seg * M;
    for (int off = 1; off < S; off <<= 1) {
        sh.ends[tid] = e;
        sh.mults[tid] = f;
        __syncthreads();
        const int src = FWD ? seg - off : seg + off;
        if (FWD ? src >= 0 : src < S) {
            const C e2 = sh.ends[src * M + mode];
            const R f2 = sh.mults[src * M + mode];
            e = cmake<C>(e.x + f * e2.x, e.y + f * e2.y);  // this segment after the earlier ones
            f = f * f2;
        }
        __syncthreads();
    }
    sh.ends[tid] = e;
    __syncthreads();
    const int prev = FWD ? seg - 1 : seg + 1;
    const C out = (FWD ? prev >= 0 : prev < S) ? sh.ends[prev * M + mode] : cmake<C>(0.0, 0.0);
    __syncthreads();  // sh is written again by the next call
    return out;
}

// One block of the partitioned solve on a spectrum of type C (pivots R).
template <typename R, typename C>
__device__ __forceinline__ void tridiag_part_gen(const R *__restrict__ piv, C *__restrict__ spec, int n, int nx,
                                                 size_t mp, R dy2, int M, int m_base, TridiagSharedT<R, C> &sh) {
    const int mlast = nx / 2;
    const int tid = threadIdx.x, mode = tid % M, seg = tid / M, S = TB_THREADS / M;
    const int m = m_base + mode;
    const bool mvalid = m <= mlast;
    const int L = (n + S - 1) / S, ja = seg * L, cnt = max(0, min(n, ja + L) - ja);
    R c[TB_L];
    C v[TB_L];
#pragma unroll
    for (int q = 0; q < TB_L; ++q) {
        const bool on = mvalid && q < cnt;
        c[q] = on ? __ldg(piv + (size_t)(ja + q) * mp + m) : R(0);
        const C sv = on ? spec[(size_t)(ja + q) * mp + m] : cmake<C>(0.0, 0.0);
        v[q] = cmake<C>(dy2 * sv.x, dy2 * sv.y);
    }
    C d = cmake<C>(0.0, 0.0);
    R mu = R(1);
#pragma unroll
    for (int q = 0; q < TB_L; ++q) {
        if (q < cnt) {
            d = cmake<C>((v[q].x - d.x) * c[q], (v[q].y - d.y) * c[q]);
            mu = -c[q] * mu;
            v[q] = d;
        }
    }
    {
        const C D = seg_carry<true>(d, mu, seg, S, M, sh);  // true entry value of the segment
        mu = R(1);
#pragma unroll
        for (int q = 0; q < TB_L; ++q) {
            if (q < cnt) {
                mu = -c[q] * mu;
                v[q].x += mu * D.x;
                v[q].y += mu * D.y;
            }
        }
    }
    C x = cmake<C>(0.0, 0.0);
    R nu = R(1);
#pragma unroll
    for (int q = TB_L - 1; q >= 0; --q) {
        if (q < cnt) {
            x = cmake<C>(v[q].x - c[q] * x.x, v[q].y - c[q] * x.y);
            nu = -c[q] * nu;
            v[q] = x;
        }
    }
    const C X = seg_carry<false>(x, nu, seg, S, M, sh);  // true exit value of the segment (x_n = 0)
    if (!mvalid) return;
    nu = R(1);
#pragma unroll
    for (int q = TB_L - 1; q >= 0; --q) {
        if (q < cnt) {
            nu = -c[q] * nu;
            spec[(size_t)(ja + q) * mp + m] = cmake<C>(v[q].x + nu * X.x, v[q].y + nu * X.y);
        }
    }
}

__device__ __forceinline__ void tridiag_part_dev(const PoissonPlan &pp, int M, int m_base, TridiagShared &sh) {
    tridiag_part_gen<double, double2>(pp.piv, pp.spec, pp.n, pp.nx, (size_t)pp.mp, pp.dy2, M, m_base, sh);
}

__global__ void __launch_bounds__(TB_THREADS) tridiag_part(const PoissonPlan pp, int M) {
    __shared__ TridiagShared sh;
    tridiag_part_dev(pp, M, blockIdx.x * M, sh);
}

// Shared memory of the FP32 form's column kernel: the FP32 modes' segment
// ends, or the zero mode's per-warp scan totals.
union ColumnShared {
    TridiagSharedT<float, float2> f;
    double wtot[TB_THREADS / 32];
};

// Inclusive sum of v over threads 0..threadIdx.x of the block (TB_THREADS
// threads): warp shuffles, then the warp totals in shared memory.  Every
// thread of the block calls it; *total gets the block's sum.
__device__ __forceinline__ double block_scan(double v, ColumnShared &sh, double *total) {
    constexpr int NW = TB_THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += t;
    }
    if (lane == 31) sh.wtot[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = lane < NW ? sh.wtot[lane] : 0.0;
#pragma unroll
        for (int off = 1; off < NW; off <<= 1) {
            const double u = __shfl_up_sync(0xffffffffu, t, off);
            if (lane >= off) t += u;
        }
        if (lane < NW) sh.wtot[lane] = t;
    }
    __syncthreads();
    if (w > 0) v += sh.wtot[w - 1];
    *total = sh.wtot[NW - 1];
    __syncthreads();  // sh is written again by the next call
    return v;
}

// The zero mode (kx = 0) of the FP32 form's column solve in FP64, by one
// block.  Its system phi_{j-1} - 2 phi_j + phi_{j+1} = h_j, h_j = dy^2 S_j
// (S_j: the row sums in column 0 of the FP64 spectrum), phi_{-1} = phi_n = 0,
// is solved exactly by two prefix sums: with H_k = h_0 + ... + h_k,
//     phi_j = (j + 1) g_0 + (H_0 + ... + H_{j-1}),  g_0 = -(H_0 + ... + H_{n-1}) / (n + 1)
// (g_j = phi_j - phi_{j-1} steps by h_j).  Thread t owns rows [t L, t L + L),
// L = ceil(n / TB_THREADS), and reads them three times (the later reads hit
// L1), so the block holds no per-row registers and fits the FP32 kernel's
// budget; the two sums over the threads are block scans.
__device__ __forceinline__ void zero_mode_f64(const PoissonPlan &pp, ColumnShared &sh) {
    const int n = pp.n, L = (n + TB_THREADS - 1) / TB_THREADS;
    const int ja = (int)threadIdx.x * L, cnt = max(0, min(n, ja + L) - ja);
    const size_t stride = 2 * (size_t)pp.mp;  // element j of the column at col[j * stride]
    double *col = &pp.spec[0].x;
    const double dy2 = pp.dy2;
    // segment sum of h, then H at the segment's start
    double s1 = 0.0;
    for (int q = 0; q < cnt; ++q) s1 += dy2 * __ldg(col + (size_t)(ja + q) * stride);
    double tot;
    const double h0 = block_scan(s1, sh, &tot) - s1;  // H_{ja - 1}
    // segment sum of H, then the sum of H before the segment and over all rows
    double H = h0, s2 = 0.0;
    for (int q = 0; q < cnt; ++q) {
        H += dy2 * __ldg(col + (size_t)(ja + q) * stride);
        s2 += H;
    }
    double S;
    const double G0 = block_scan(s2, sh, &S) - s2;  // H_0 + ... + H_{ja - 1}
    const double g0 = -S / (double)(n + 1);
    H = h0;
    double G = G0;
    for (int q = 0; q < cnt; ++q) {
        const int j = ja + q;
        const double hj = dy2 * __ldg(col + (size_t)j * stride);
        col[(size_t)j * stride] = (double)(j + 1) * g0 + G;
        H += hj;
        G += H;
    }
}

// Pass B of the FP32 form in one kernel: block 0 solves the zero mode in
// FP64 (zero_mode_f64), blocks 1.. the modes 1..nx/2 in FP32, M per block,
// two blocks per SM.
__global__ void __launch_bounds__(TB_THREADS, 2) tridiag_modes_f32(const PoissonPlan pp, int M) {
    __shared__ ColumnShared sh;
    if (blockIdx.x == 0) {
        zero_mode_f64(pp, sh);
        return;
    }
    tridiag_part_gen<float, float2>(pp.pivf, pp.specf, pp.n, pp.nx, (size_t)pp.mp, (float)pp.dy2, M,
                                    1 + (blockIdx.x - 1) * M, sh.f);
}

// ---- batched passes: one launch for many channels -------------------------
// A block's work item names its channel and its first row pair (passes A,
// C) or first x-mode (pass B); the channel's plan comes from a device table.
// Batches run the FP32 form.
__global__ void __launch_bounds__(256, 4)
batch_fwd_rows_f32(const PoissonPlan *__restrict__ plans, const Chan *__restrict__ chans,
                   const int2 *__restrict__ items) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[256 / 32];
    const int2 it = items[blockIdx.x];
    const PoissonPlan pp = plans[it.x];
    fwd_rows_r16f_dev<256>(pp, chans[it.x], it.y, (float2 *)smraw, red);
}

__global__ void __launch_bounds__(256, 4)
batch_inv_rows_f32(const PoissonPlan *__restrict__ plans, const Chan *__restrict__ chans,
                   double *const *__restrict__ fields, const int2 *__restrict__ items, bool write_f64) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int2 it = items[blockIdx.x];
    const PoissonPlan pp = plans[it.x];
    const Chan &c = chans[it.x];
    inv_rows_r16f_dev<256>(pp, c, fields[it.x] + F_PSI * c.plane, write_f64, it.y, (float2 *)smraw);
}

// items {channel, first mode, modes per block}: FP32 mode blocks, and for
// modes per block == 0 the channel's FP64 zero mode (zero_mode_f64)
__global__ void __launch_bounds__(TB_THREADS, 2)
batch_tridiag_modes_f32(const PoissonPlan *__restrict__ plans, const int3 *__restrict__ items) {
    __shared__ ColumnShared sh;
    const int3 it = items[blockIdx.x];
    const PoissonPlan pp = plans[it.x];
    if (it.z == 0) {
        zero_mode_f64(pp, sh);
        return;
    }
    tridiag_part_gen<float, float2>(pp.pivf, pp.specf, pp.n, pp.nx, (size_t)pp.mp, (float)pp.dy2, it.z, it.y,
                                    sh.f);
}

// Modes per block of tridiag_part for n rows, so that every segment has at
// most TB_L rows (0: too tall, use the one-thread-per-mode `tridiag`).
int tridiag_modes(int n) {
    for (int M = 8; M >= 1; M >>= 1)
        if ((n + TB_THREADS / M - 1) / (TB_THREADS / M) <= TB_L) return M;
    return 0;
}

bool use_r16(const PoissonPlan &pp) { return pp.pow2 && pp.nx >= 16; }

// Threads per block and row pairs per block of the radix-16 row kernels.
void r16_shape(int nx, int *threads, int *per) {
    const int T = nx >> 4;
    *threads = T >= 256 ? T : 256;
    *per = *threads / T;
}

size_t r16_smem(int nx, int per) { return (size_t)per * nx * sizeof(double2); }

}  // namespace

size_t poisson_smem_bytes_f64(int nx) {
    const bool pow2 = nx > 0 && (nx & (nx - 1)) == 0;
    return (size_t)nx * sizeof(double2) * (pow2 ? 1 : 2);
}

cudaError_t poisson_pass_f64(int pass, const PoissonPlan &pp, const Chan &c, double *fields, cudaStream_t s) {
    return poisson_pass_f64_at(pass, pp, c, fields + F_RHS * c.plane, fields + F_PSI * c.plane, s);
}

cudaError_t poisson_pass_f64_at(int pass, const PoissonPlan &pp, const Chan &c, const double *rhs, double *psi,
                                cudaStream_t s) {
    const int rows2 = (pp.n + 1) / 2;
    if (pass == 1) {
        const int M = tridiag_modes(pp.n);
        if (M > 0) tridiag_part<<<(pp.nx / 2 + M) / M, TB_THREADS, 0, s>>>(pp, M);
        else tridiag<<<(pp.nx / 2 + 1 + PTPB - 1) / PTPB, PTPB, 0, s>>>(pp);
        return cudaGetLastError();
    }
    if (use_r16(pp)) {
        int threads, per;
        r16_shape(pp.nx, &threads, &per);
        const size_t smem = r16_smem(pp.nx, per);
        const int blocks = (rows2 + per - 1) / per;
        if (threads == 256) {
            if (pass == 0) fwd_rows_r16<256><<<blocks, 256, smem, s>>>(pp, rhs, c.nxp);
            else inv_rows_r16<256><<<blocks, 256, smem, s>>>(pp, c, psi);
        } else {
            if (pass == 0) fwd_rows_r16<512><<<blocks, 512, smem, s>>>(pp, rhs, c.nxp);
            else inv_rows_r16<512><<<blocks, 512, smem, s>>>(pp, c, psi);
        }
        return cudaGetLastError();
    }
    const size_t smem = poisson_smem_bytes_f64(pp.nx);
    if (pass == 0) fwd_rows<<<rows2, PTPB, smem, s>>>(pp, rhs, c.nxp);
    else inv_rows<<<rows2, PTPB, smem, s>>>(pp, c, psi);
    return cudaGetLastError();
}

int poisson_tridiag_modes(int n) { return tridiag_modes(n); }

bool poisson_f32_supported(const PoissonPlan &pp) {
    return use_r16(pp) && tridiag_modes(pp.n) > 0 && pp.twf && pp.pivf && pp.specf && pp.rowmean && pp.rowmean_ok;
}

cudaError_t poisson_tridiag_f32(const PoissonPlan &pp, cudaStream_t s) {
    if (!poisson_f32_supported(pp)) return cudaErrorInvalidValue;
    const int M = tridiag_modes(pp.n);
    tridiag_modes_f32<<<1 + (pp.nx / 2 + M - 1) / M, TB_THREADS, 0, s>>>(pp, M);
    return cudaGetLastError();
}

cudaError_t poisson_pass_f32(int pass, const PoissonPlan &pp, const Chan &c, double *psi, bool write_f64,
                             cudaStream_t s) {
    // pass B of this form runs through poisson_tridiag_f32
    if (!poisson_f32_supported(pp) || pass == 1) return cudaErrorInvalidValue;
    int threads, per;
    r16_shape(pp.nx, &threads, &per);
    const size_t smem = (size_t)per * pp.nx * sizeof(float2);
    const int blocks = ((pp.n + 1) / 2 + per - 1) / per;
    if (threads == 256) {
        if (pass == 0) return launch_pdl(fwd_rows_r16f<256>, dim3(blocks), dim3(256), smem, s, pp, c);
        inv_rows_r16f<256><<<blocks, 256, smem, s>>>(pp, c, psi, write_f64);
    } else {
        if (pass == 0) return launch_pdl(fwd_rows_r16f<512>, dim3(blocks), dim3(512), smem, s, pp, c);
        inv_rows_r16f<512><<<blocks, 512, smem, s>>>(pp, c, psi, write_f64);
    }
    return cudaGetLastError();
}

cudaError_t batch_poisson(int pass, const PoissonPlan *plans, const Chan *chans, double *const *fields,
                          const void *items, int nitems, bool write_f64, cudaStream_t s) {
    if (nitems <= 0) return cudaSuccess;
    if (pass == 1) return cudaErrorInvalidValue;  // runs through batch_tridiag_f32
    if (pass == 0)
        batch_fwd_rows_f32<<<nitems, 256, 32768, s>>>(plans, chans, (const int2 *)items);
    else
        batch_inv_rows_f32<<<nitems, 256, 32768, s>>>(plans, chans, fields, (const int2 *)items, write_f64);
    return cudaGetLastError();
}

cudaError_t batch_tridiag_f32(const PoissonPlan *plans, const void *items, int nitems, cudaStream_t s) {
    if (nitems > 0) batch_tridiag_modes_f32<<<nitems, TB_THREADS, 0, s>>>(plans, (const int3 *)items);
    return cudaGetLastError();
}

cudaError_t poisson_set_smem_limits() {
    const void *fns[] = {(const void *)fwd_rows, (const void *)inv_rows, (const void *)fwd_rows_r16<256>,
                         (const void *)inv_rows_r16<256>, (const void *)fwd_rows_r16<512>,
                         (const void *)inv_rows_r16<512>, (const void *)fwd_rows_r16f<256>,
                         (const void *)inv_rows_r16f<256>, (const void *)fwd_rows_r16f<512>,
                         (const void *)inv_rows_r16f<512>, (const void *)batch_fwd_rows_f32,
                         (const void *)batch_inv_rows_f32};
    for (const void *f : fns) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace ek
