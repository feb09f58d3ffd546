/*
 * ek_oracle.cpp -- CPU oracle of the EK-PNP coupled step.  TEST INFRASTRUCTURE
 * ONLY: the checker used by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py.  The product (libekpnp.so) never links or calls it.
 *
 * A plain FP64 C++/OpenMP restatement of the reference's update rules, in the
 * reference's own push form and memory layout so that each phase can be read
 * against the CUDA kernel it restates:
 *
 *   collide   gpu_collide_save      LBM.cu:331-804
 *   walls     gpu_boundary          LBM.cu:806-860
 *   stream    gpu_stream            LBM.cu:862-906
 *   ion walls gpu_bc_charge         LBM.cu:908-1024
 *   poisson   fast_Poisson + odd_extension/gpu_derivative/odd_extract
 *             poisson.cu:180-306, wavenumbers main.cu:119-137
 *   E field   gpu_efield + gpu_bc   poisson.cu:145-174
 *   init      gpu_init_equilibrium  LBM.cu:195-305
 *
 * Deliberate choices (each also stated where it is made):
 *   - The lower-wall velocity mirror reads the PRE-collision populations of
 *     row 1.  The reference reads them while another block may already have
 *     overwritten the rest populations in place (LBM.cu:403-405 vs 775-777);
 *     pre-collision is the order the code intends.
 *   - cuFFT (a closed library) is replaced by this file's own complex FFT
 *     (iterative radix-2 for powers of two, Bluestein's chirp-z algorithm for
 *     other lengths) applied to the same odd-extended array, forward sign -1
 *     and unnormalised inverse, as cufftExecZ2Z computes.
 *   - No FMA contraction (built with -ffp-contract=off): results differ from
 *     the GPU builds by rounding only.
 *
 * Parity pin: the reference has no tests or golden data.  This oracle is
 * pinned against dumps of the patched reference build itself (recipe in
 * oracle/ref_build.py), committed as fixtures under tests/golden/.
 */
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/ekpnp.h"

namespace {

typedef std::complex<double> cplx;

const double W0 = 4.0 / 9.0, WS = 1.0 / 9.0, WD = 1.0 / 36.0;  // LBM.h:105-107
// D2Q9 numbering of the reference (LBM.cu:831-834):  6 2 5 / 3 0 1 / 7 4 8
const int CX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
const int CY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
const int OPP[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

// ---------------------------------------------------------------- FFT ----
bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

// In-place iterative radix-2 transform, exponent sign `sgn`, no scaling.
void fft_pow2(cplx *a, size_t n, int sgn) {
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len >> 1;
        for (size_t k = 0; k < half; ++k) {
            const double ang = sgn * 2.0 * M_PI * (double)k / (double)len;
            const cplx w(std::cos(ang), std::sin(ang));
            for (size_t i = k; i < n; i += len) {
                const cplx u = a[i], v = a[i + half] * w;
                a[i] = u + v;
                a[i + half] = u - v;
            }
        }
    }
}

// Transform of any length: radix-2 or Bluestein (chirp-z) through a
// power-of-two circular convolution.
struct Fft1d {
    size_t n = 0, m = 0;
    int sgn = -1;
    std::vector<cplx> chirp, bhat;
    void plan(size_t n_, int sgn_) {
        n = n_;
        sgn = sgn_;
        if (is_pow2(n)) return;
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
        chirp.resize(n);
        for (size_t k = 0; k < n; ++k) {
            // angle pi*k^2/n, with k^2 reduced mod 2n to keep the argument small
            const unsigned long long k2 = ((unsigned long long)k * k) % (2ull * n);
            const double ang = sgn * M_PI * (double)k2 / (double)n;
            chirp[k] = cplx(std::cos(ang), std::sin(ang));
        }
        bhat.assign(m, cplx(0, 0));
        bhat[0] = std::conj(chirp[0]);
        for (size_t k = 1; k < n; ++k) bhat[k] = bhat[m - k] = std::conj(chirp[k]);
        fft_pow2(bhat.data(), m, -1);
    }
    void run(cplx *a, std::vector<cplx> &work) const {
        if (is_pow2(n)) { fft_pow2(a, n, sgn); return; }
        work.assign(m, cplx(0, 0));
        for (size_t k = 0; k < n; ++k) work[k] = a[k] * chirp[k];
        fft_pow2(work.data(), m, -1);
        for (size_t k = 0; k < m; ++k) work[k] *= bhat[k];
        fft_pow2(work.data(), m, +1);
        const double inv = 1.0 / (double)m;
        for (size_t k = 0; k < n; ++k) a[k] = work[k] * inv * chirp[k];
    }
};

// 2D transform of a rows x cols row-major array: every row, then every column.
void fft2d(cplx *a, size_t rows, size_t cols, const Fft1d &frow, const Fft1d &fcol) {
#pragma omp parallel
    {
        std::vector<cplx> work, col(rows);
#pragma omp for schedule(static)
        for (long r = 0; r < (long)rows; ++r) frow.run(a + (size_t)r * cols, work);
#pragma omp for schedule(static)
        for (long c = 0; c < (long)cols; ++c) {
            for (size_t r = 0; r < rows; ++r) col[r] = a[r * cols + c];
            fcol.run(col.data(), work);
            for (size_t r = 0; r < rows; ++r) a[r * cols + c] = col[r];
        }
    }
}

// ------------------------------------------------------- equilibria ----
// w * dens * (omusq + cu*(1 + cu/2)), the form of LBM.cu:468-552, with the
// direction's cu = (c_i . u)/cs2/cfl built as the reference builds it.
inline double feq_term(double wdens, double omusq, double cu) {
    return wdens * (omusq + cu * (1.0 + 0.5 * cu));
}

void equilibria(double dens, double tux, double tuy, double omusq, double omusq_rest,
                double e[9]) {
    const double w0d = W0 * dens, wsd = WS * dens, wdd = WD * dens;
    e[0] = w0d * omusq_rest;
    e[1] = feq_term(wsd, omusq, tux);
    e[2] = feq_term(wsd, omusq, tuy);
    e[3] = feq_term(wsd, omusq, -tux);
    e[4] = feq_term(wsd, omusq, -tuy);
    e[5] = feq_term(wdd, omusq, tux + tuy);
    e[6] = feq_term(wdd, omusq, tuy - tux);
    e[7] = feq_term(wdd, omusq, -(tux + tuy));
    e[8] = feq_term(wdd, omusq, tux - tuy);
}

// Guo force populations, LBM.cu:556-572 (e_i = c_i/cfl).
void guo_pops(double ux, double uy, double fx, double fy, double cs2, double cfl, double s[9]) {
    const double coe0 = W0 / cs2, coes = WS / cs2, coed = WD / cs2;
    const double ci = 1.0 / cfl;
    const double ci2 = ci * ci / cs2;
    const double axx = (ci * ux) * ci / cs2;  // (e.u) e_x / cs2 for the x axis
    const double ayy = (ci * uy) * ci / cs2;
    s[0] = coe0 * (-ux * fx - uy * fy);
    s[1] = coes * (((ci - ux) + axx) * fx - uy * fy);
    s[2] = coes * (-ux * fx + ((ci - uy) + ayy) * fy);
    s[3] = coes * (((-ci - ux) + axx) * fx - uy * fy);
    s[4] = coes * (-ux * fx + ((-ci - uy) + ayy) * fy);
    s[5] = coed * (((ci - ux) + (ux + uy) * ci2) * fx + ((ci - uy) + (ux + uy) * ci2) * fy);
    s[6] = coed * (((-ci - ux) + (ux - uy) * ci2) * fx + ((ci - uy) + (-ux + uy) * ci2) * fy);
    s[7] = coed * (((-ci - ux) + (ux + uy) * ci2) * fx + ((-ci - uy) + (ux + uy) * ci2) * fy);
    s[8] = coed * (((ci - ux) + (ux - uy) * ci2) * fx + ((-ci - uy) + (-ux + uy) * ci2) * fy);
}

// TRT relaxation with symmetric/antisymmetric split (LBM.cu:574-803).
// wp, wm: omega_plus*dt, omega_minus*dt; src may be null (ions).
void trt(const double t[9], const double e[9], const double *src, double dt, double wp,
         double wm, double out[9]) {
    const double r0 = t[0] - (wp * (t[0] - e[0]) + wm * (0.0 - 0.0));
    out[0] = src ? r0 + dt * src[0] : r0;
    const int first[4] = {1, 2, 5, 6};
    for (int k = 0; k < 4; ++k) {
        const int a = first[k], b = OPP[a];
        const double p = 0.5 * (t[a] + t[b]), m = 0.5 * (t[a] - t[b]);
        const double ep = 0.5 * (e[a] + e[b]), em = 0.5 * (e[a] - e[b]);
        const double ra = t[a] - (wp * (p - ep) + wm * (m - em));
        const double rb = t[b] - (wp * (p - ep) + wm * (-m - -em));
        out[a] = src ? ra + dt * src[a] : ra;
        out[b] = src ? rb + dt * src[b] : rb;
    }
}

}  // namespace

// ------------------------------------------------------------- state ----
struct ekor {
    ek_params p;
    size_t nx, ny, nn, ne;
    // populations in the reference layout: rest [y][x], moving [d-1][y][x]
    std::vector<double> f0, f1, f2, h0, h1, h2, t0, t1, t2, f0bc;
    // fields
    std::vector<double> rho, ux, uy, cp, cn, psi, ex, ey;
    // wall profiles along x
    std::vector<double> zlo, zhi, cplo, cphi, cnlo, cnhi;
    std::vector<double> kx, ky;
    std::vector<cplx> ext;
    Fft1d fx_fwd, fx_inv, fy_fwd, fy_inv;
    int64_t steps = 0;
    size_t fi(size_t x, size_t y, int d) const { return nx * (ny * (size_t)(d - 1) + y) + x; }
    size_t si(size_t x, size_t y) const { return nx * y + x; }
};

namespace {

struct Rates { double wp, wm, wcp, wcm, wtp, wtm, sp, sm; };

// LBM.cu:336-341 and 745-746, 766-771
Rates rates(const ek_params &p) {
    Rates r;
    const double om_p = 1.0 / (p.nu / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double om_m = 1.0 / (p.magic_f / (p.nu / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    const double oc_m = 1.0 / (p.diff_p / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double oc_p = 1.0 / (p.magic_p / (p.diff_p / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    const double ot_m = 1.0 / (p.diff_n / p.cs2 / p.dt + 1.0 / 2.0) / p.dt;
    const double ot_p = 1.0 / (p.magic_n / (p.diff_n / p.cs2 / p.dt) + 1.0 / 2.0) / p.dt;
    r.wp = om_p * p.dt;
    r.wm = om_m * p.dt;
    r.wcp = oc_p * p.dt;
    r.wcm = oc_m * p.dt;
    r.wtp = ot_p * p.dt;
    r.wtm = ot_m * p.dt;
    r.sp = 1.0 - 0.5 * p.dt * om_p;
    r.sm = 1.0 - 0.5 * p.dt * om_m;
    return r;
}

void load9(const ekor &s, const std::vector<double> &a0, const std::vector<double> &a1, size_t x,
           size_t y, double t[9]) {
    t[0] = a0[s.si(x, y)];
    for (int d = 1; d < 9; ++d) t[d] = a1[s.fi(x, y, d)];
}

double sum9(const double t[9]) {
    return t[0] + t[1] + t[2] + t[3] + t[4] + t[5] + t[6] + t[7] + t[8];
}

// gpu_collide_save, LBM.cu:331-804.  Rest populations are written to new
// arrays so every node (and the lower-wall mirror) reads pre-collision values.
void collide(ekor &s) {
    const ek_params &p = s.p;
    const Rates r = rates(p);
    const bool force_on = (p.flags & EK_FLAG_FORCE) != 0;
    const bool quirk = (p.flags & EK_FLAG_REST_QUIRK) != 0;
    std::vector<double> nf0(s.nn), nh0(s.nn), nt0(s.nn);
    for (size_t x = 0; x < s.nx; ++x) {
        s.f0bc[x] = s.f0[s.si(x, 0)];
        s.f0bc[s.nx + x] = s.f0[s.si(x, s.ny - 1)];
    }
#pragma omp parallel for schedule(static)
    for (long yl = 0; yl < (long)s.ny; ++yl) {
        const size_t y = (size_t)yl;
        for (size_t x = 0; x < s.nx; ++x) {
            double ft[9], ht[9], tt[9];
            load9(s, s.f0, s.f1, x, y, ft);
            load9(s, s.h0, s.h1, x, y, ht);
            load9(s, s.t0, s.t1, x, y, tt);
            const double rho = sum9(ft);
            const double rhoinv = 1.0 / rho;
            const double charge = sum9(ht);
            const double temp = sum9(tt);
            const size_t k = s.si(x, y);
            const double Ex = s.ex[k], Ey = s.ey[k];
            double fx = 0.0, fy = 0.0;
            if (force_on) {  // the expression commented out at LBM.cu:388-389
                fx = p.f_charge * (charge - temp) * (Ex + p.ext_x) + p.exf;
                fy = p.f_charge * (charge - temp) * Ey;
            }
            double ux = rhoinv * ((ft[1] + ft[5] + ft[8] - (ft[3] + ft[6] + ft[7])) / p.cfl + fx * p.dt * 0.5);
            double uy = rhoinv * ((ft[2] + ft[5] + ft[6] - (ft[4] + ft[7] + ft[8])) / p.cfl + fy * p.dt * 0.5);
            if (y == 0) {
                // lower wall: minus the velocity of row 1 (LBM.cu:402-443), with the
                // wall node's own force as in the commented expression at 438-439
                double fm[9];
                load9(s, s.f0, s.f1, x, 1, fm);
                const double rhoinvm = 1.0 / sum9(fm);
                ux = -rhoinvm * ((fm[1] + fm[5] + fm[8] - (fm[3] + fm[6] + fm[7])) / p.cfl + fx * p.dt * 0.5);
                uy = -rhoinvm * ((fm[2] + fm[5] + fm[6] - (fm[4] + fm[7] + fm[8])) / p.cfl + fy * p.dt * 0.5);
            }
            s.rho[k] = rho;
            s.ux[k] = ux;
            s.uy[k] = uy;
            s.cp[k] = charge;
            s.cn[k] = temp;

            const double upx = ux + p.mob_p * Ex, upy = uy + p.mob_p * Ey;
            const double unx = ux + p.mob_n * Ex, uny = uy + p.mob_n * Ey;
            const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy) / p.cs2;
            const double omusq_c = 1.0 - 0.5 * (upx * upx + upy * upy) / p.cs2;
            const double omusq_cn = 1.0 - 0.5 * (unx * unx + uny * uny) / p.cs2;
            double fe[9], he[9], te[9];
            equilibria(rho, ux / p.cs2 / p.cfl, uy / p.cs2 / p.cfl, omusq, omusq, fe);
            equilibria(charge, upx / p.cs2 / p.cfl, upy / p.cs2 / p.cfl, omusq_c, omusq_c, he);
            equilibria(temp, unx / p.cs2 / p.cfl, uny / p.cs2 / p.cfl, omusq_cn,
                       quirk ? omusq : omusq_cn, te);

            double fpop[9], src[9];
            guo_pops(ux, uy, fx, fy, p.cs2, p.cfl, fpop);
            src[0] = r.sp * fpop[0];
            const int first[4] = {1, 2, 5, 6};
            for (int q = 0; q < 4; ++q) {
                const int a = first[q], b = OPP[a];
                const double fp = 0.5 * (fpop[a] + fpop[b]), fm = 0.5 * (fpop[a] - fpop[b]);
                src[a] = r.sp * fp + r.sm * fm;
                src[b] = r.sp * fp + r.sm * -fm;
            }
            double fo[9], ho[9], to[9];
            trt(ft, fe, src, p.dt, r.wp, r.wm, fo);
            trt(ht, he, nullptr, p.dt, r.wcp, r.wcm, ho);
            trt(tt, te, nullptr, p.dt, r.wtp, r.wtm, to);
            nf0[k] = fo[0];
            nh0[k] = ho[0];
            nt0[k] = to[0];
            for (int d = 1; d < 9; ++d) {
                const size_t j = s.fi(x, y, d);
                s.f2[j] = fo[d];
                s.h2[j] = ho[d];
                s.t2[j] = to[d];
            }
        }
    }
    s.f0.swap(nf0);
    s.h0.swap(nh0);
    s.t0.swap(nt0);
}

// gpu_boundary, LBM.cu:806-860: full-way bounce-back of the pre-collision
// populations at both walls, moving top wall through uw.
void fluid_walls(ekor &s) {
    const ek_params &p = s.p;
    const double ms = 2.0 * p.rho0 * p.uw / p.cs2 * WS / p.cfl;
    const double md = 2.0 * p.rho0 * p.uw / p.cs2 * WD / p.cfl;
    const size_t top = s.ny - 1;
    for (size_t x = 0; x < s.nx; ++x) {
        s.f0[s.si(x, 0)] = s.f0bc[x];
        for (int d = 1; d < 9; ++d) s.f2[s.fi(x, 0, OPP[d])] = s.f1[s.fi(x, 0, d)];
        s.f0[s.si(x, top)] = s.f0bc[s.nx + x];
        const double add[9] = {0, -ms, 0, +ms, 0, -md, +md, +md, -md};
        for (int d = 1; d < 9; ++d) s.f2[s.fi(x, top, OPP[d])] = s.f1[s.fi(x, top, d)] + add[d];
    }
}

// gpu_stream, LBM.cu:862-906: push streaming, periodic in x and y.
void stream(ekor &s) {
#pragma omp parallel for schedule(static)
    for (long yl = 0; yl < (long)s.ny; ++yl) {
        const size_t y = (size_t)yl;
        for (int d = 1; d < 9; ++d) {
            const size_t ys = (y + s.ny - CY[d]) % s.ny;
            for (size_t x = 0; x < s.nx; ++x) {
                const size_t xs = (x + s.nx - CX[d]) % s.nx;
                const size_t dst = s.fi(x, y, d), src = s.fi(xs, ys, d);
                s.f1[dst] = s.f2[src];
                s.h1[dst] = s.h2[src];
                s.t1[dst] = s.t2[src];
            }
        }
    }
}

// gpu_bc_charge, LBM.cu:908-1024: anti-bounce-back with Dirichlet wall
// concentrations, all nine populations of each wall node.
void ion_walls(ekor &s) {
    const size_t rows[2] = {0, s.ny - 1};
    for (int w = 0; w < 2; ++w) {
        const size_t y = rows[w];
        for (size_t x = 0; x < s.nx; ++x) {
            const double cw = w == 0 ? s.cplo[x] : s.cphi[x];
            const double nw = w == 0 ? s.cnlo[x] : s.cnhi[x];
            const double wc[3] = {2.0 * cw * W0, 2.0 * cw * WS, 2.0 * cw * WD};
            const double wt[3] = {2.0 * nw * W0, 2.0 * nw * WS, 2.0 * nw * WD};
            const size_t k = s.si(x, y);
            s.h0[k] = -s.h0[k] + wc[0];
            s.t0[k] = -s.t0[k] + wt[0];
            for (int d = 1; d < 9; ++d) {
                const int cls = d < 5 ? 1 : 2;
                s.h1[s.fi(x, y, OPP[d])] = -s.h2[s.fi(x, y, d)] + wc[cls];
                s.t1[s.fi(x, y, OPP[d])] = -s.t2[s.fi(x, y, d)] + wt[cls];
            }
        }
    }
}

// fast_Poisson, poisson.cu:180-306, and efield/gpu_bc, poisson.cu:132-174.
void poisson(ekor &s) {
    const ek_params &p = s.p;
    const size_t nx = s.nx, ny = s.ny, ne = s.ne;
    std::vector<cplx> &a = s.ext;
    // odd_extension (poisson.cu:220-263): rows 1..ny-2 carry the source with the
    // Dirichlet lifting at rows 1 and ny-2; rows ne-y carry its negative.
    for (size_t x = 0; x < nx; ++x) {
        a[x] = 0.0;
        a[(ny - 1) * nx + x] = 0.0;
    }
    for (size_t y = 1; y + 1 < ny; ++y) {
        for (size_t x = 0; x < nx; ++x) {
            double v = -p.f_charge * (s.cp[s.si(x, y)] - s.cn[s.si(x, y)]) / p.eps;
            if (y == 1) v = v - s.zlo[x] / p.dy / p.dy;
            if (y == ny - 2) v = v - s.zhi[x] / p.dy / p.dy;
            a[y * nx + x] = cplx(v, 0.0);
            a[(ne - y) * nx + x] = cplx(-v, 0.0);
        }
    }
    fft2d(a.data(), ne, nx, s.fx_fwd, s.fy_fwd);
    // gpu_derivative (poisson.cu:274-283)
    for (size_t y = 0; y < ne; ++y) {
        const double J = s.ky[y];
        for (size_t x = 0; x < nx; ++x) {
            const double I = s.kx[x];
            double mu = (4.0 / p.dy / p.dy) * (std::sin(J * p.dy * 0.5) * std::sin(J * p.dy * 0.5)) + I * I;
            if (y == 0 && x == 0) mu = 1.0;
            cplx &c = a[y * nx + x];
            c = cplx(-c.real() / mu, -c.imag() / mu);
        }
    }
    fft2d(a.data(), ne, nx, s.fx_inv, s.fy_inv);
    // odd_extract (poisson.cu:294-306)
    const double size = (double)(nx * ne);
    for (size_t y = 0; y < ny; ++y)
        for (size_t x = 0; x < nx; ++x) {
            double v = a[y * nx + x].real() / size;
            if (y == 0) v = s.zlo[x];
            if (y == ny - 1) v = s.zhi[x];
            s.psi[s.si(x, y)] = v;
        }
    // gpu_efield + gpu_bc
    for (size_t y = 0; y < ny; ++y)
        for (size_t x = 0; x < nx; ++x) {
            const size_t xp = (x + 1) % nx, xm = (x + nx - 1) % nx;
            const size_t yp = (y + 1) % ny, ym = (y + ny - 1) % ny;
            s.ex[s.si(x, y)] = 0.5 * (s.psi[s.si(xm, y)] - s.psi[s.si(xp, y)]) / p.dx;
            s.ey[s.si(x, y)] = 0.5 * (s.psi[s.si(x, ym)] - s.psi[s.si(x, yp)]) / p.dy;
        }
    for (size_t x = 0; x < nx; ++x) {
        s.ey[s.si(x, 0)] = s.ey[s.si(x, 1)];
        s.ey[s.si(x, ny - 1)] = s.ey[s.si(x, ny - 2)];
    }
}

// gpu_init_equilibrium, LBM.cu:195-305 (rest population of c- uses its own
// drift velocity there, LBM.cu:242).
void init_equilibrium(ekor &s) {
    const ek_params &p = s.p;
#pragma omp parallel for schedule(static)
    for (long yl = 0; yl < (long)s.ny; ++yl) {
        const size_t y = (size_t)yl;
        for (size_t x = 0; x < s.nx; ++x) {
            const size_t k = s.si(x, y);
            const double ux = s.ux[k], uy = s.uy[k], Ex = s.ex[k], Ey = s.ey[k];
            const double upx = ux + p.mob_p * Ex, upy = uy + p.mob_p * Ey;
            const double unx = ux + p.mob_n * Ex, uny = uy + p.mob_n * Ey;
            const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy) / p.cs2;
            const double omusq_c = 1.0 - 0.5 * (upx * upx + upy * upy) / p.cs2;
            const double omusq_cn = 1.0 - 0.5 * (unx * unx + uny * uny) / p.cs2;
            double fe[9], he[9], te[9];
            equilibria(s.rho[k], ux / p.cs2 / p.cfl, uy / p.cs2 / p.cfl, omusq, omusq, fe);
            equilibria(s.cp[k], upx / p.cs2 / p.cfl, upy / p.cs2 / p.cfl, omusq_c, omusq_c, he);
            equilibria(s.cn[k], unx / p.cs2 / p.cfl, uny / p.cs2 / p.cfl, omusq_cn, omusq_cn, te);
            s.f0[k] = fe[0];
            s.h0[k] = he[0];
            s.t0[k] = te[0];
            for (int d = 1; d < 9; ++d) {
                const size_t j = s.fi(x, y, d);
                s.f1[j] = fe[d];
                s.h1[j] = he[d];
                s.t1[j] = te[d];
            }
        }
    }
}

}  // namespace

// ------------------------------------------------------------ C ABI ----
extern "C" {

int ekor_create(const ek_params *p, ekor **out) {
    if (!p || !out || p->nx < 1 || p->ny < 4) return EK_ERR_INVALID;
    ekor *s = new ekor();
    s->p = *p;
    s->nx = (size_t)p->nx;
    s->ny = (size_t)p->ny;
    s->nn = s->nx * s->ny;
    s->ne = 2 * (s->ny - 1);
    const size_t nn = s->nn, n8 = 8 * nn;
    for (auto *v : {&s->f0, &s->h0, &s->t0}) v->assign(nn, 0.0);
    for (auto *v : {&s->f1, &s->f2, &s->h1, &s->h2, &s->t1, &s->t2}) v->assign(n8, 0.0);
    for (auto *v : {&s->rho, &s->ux, &s->uy, &s->cp, &s->cn, &s->psi, &s->ex, &s->ey}) v->assign(nn, 0.0);
    s->f0bc.assign(2 * s->nx, 0.0);
    s->zlo.assign(s->nx, p->zeta_lo);
    s->zhi.assign(s->nx, p->zeta_hi);
    s->cplo.assign(s->nx, p->cp_lo);
    s->cphi.assign(s->nx, p->cp_hi);
    s->cnlo.assign(s->nx, p->cn_lo);
    s->cnhi.assign(s->nx, p->cn_hi);
    // wavenumbers, main.cu:119-137
    s->kx.resize(s->nx);
    s->ky.resize(s->ne);
    for (size_t i = 0; i < s->nx; ++i) {
        const double m = i <= s->nx / 2 ? (double)i : (double)i - (double)s->nx;
        s->kx[i] = m * 2.0 * M_PI / p->lx;
    }
    for (size_t i = 0; i < s->ne; ++i) {
        const double m = i <= s->ne / 2 ? (double)i : (double)i - (double)s->ne;
        s->ky[i] = m * 2.0 * M_PI / ((double)s->ne * p->dy);
    }
    s->ext.assign(s->ne * s->nx, cplx(0, 0));
    s->fx_fwd.plan(s->nx, -1);
    s->fx_inv.plan(s->nx, +1);
    s->fy_fwd.plan(s->ne, -1);
    s->fy_inv.plan(s->ne, +1);
    *out = s;
    return EK_OK;
}

void ekor_destroy(ekor *s) { delete s; }

int ekor_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int ekor_set_fields(ekor *s, const double *rho, const double *ux, const double *uy,
                    const double *cp, const double *cn, const double *psi, const double *ex,
                    const double *ey) {
    if (!s) return EK_ERR_INVALID;
    const size_t b = s->nn * sizeof(double);
    if (rho) std::memcpy(s->rho.data(), rho, b);
    if (ux) std::memcpy(s->ux.data(), ux, b);
    if (uy) std::memcpy(s->uy.data(), uy, b);
    if (cp) std::memcpy(s->cp.data(), cp, b);
    if (cn) std::memcpy(s->cn.data(), cn, b);
    if (psi) std::memcpy(s->psi.data(), psi, b);
    if (ex) std::memcpy(s->ex.data(), ex, b);
    if (ey) std::memcpy(s->ey.data(), ey, b);
    return EK_OK;
}

int ekor_set_wall_profile(ekor *s, const double *zlo, const double *zhi, const double *cplo,
                          const double *cphi, const double *cnlo, const double *cnhi) {
    if (!s) return EK_ERR_INVALID;
    const size_t b = s->nx * sizeof(double);
    if (zlo) std::memcpy(s->zlo.data(), zlo, b);
    if (zhi) std::memcpy(s->zhi.data(), zhi, b);
    if (cplo) std::memcpy(s->cplo.data(), cplo, b);
    if (cphi) std::memcpy(s->cphi.data(), cphi, b);
    if (cnlo) std::memcpy(s->cnlo.data(), cnlo, b);
    if (cnhi) std::memcpy(s->cnhi.data(), cnhi, b);
    return EK_OK;
}

// Poisson-Boltzmann start, LBM.cu:95-145: fields of gpu_initialization
// (rho0, u = 0, psi = voltage everywhere, E = 0), then `iters` rounds of
// {c+- = c0 exp(-+ e_kt psi) (gpu_PBE), fast_Poisson, psi = omega psi +
// (1 - omega) psi_old (gpu_PBE_phi)}.  E keeps the last Poisson result.
int ekor_init_pb(ekor *s, int iters, double omega, double e_kt) {
    if (!s || iters < 0) return EK_ERR_INVALID;
    const size_t nn = s->nn;
    for (size_t k = 0; k < nn; ++k) {
        s->rho[k] = s->p.rho0;
        s->ux[k] = s->uy[k] = 0.0;
        s->psi[k] = s->zlo[k % s->nx];
        s->ex[k] = s->ey[k] = 0.0;
    }
    std::vector<double> old(s->psi);
    for (int it = 0; it < iters; ++it) {
        for (size_t k = 0; k < nn; ++k) {
            s->cp[k] = s->p.c0 * std::exp(-e_kt * s->psi[k]);
            s->cn[k] = s->p.c0 * std::exp(e_kt * s->psi[k]);
        }
        poisson(*s);
        for (size_t k = 0; k < nn; ++k) {
            s->psi[k] = omega * s->psi[k] + (1.0 - omega) * old[k];
            old[k] = s->psi[k];
        }
    }
    return EK_OK;
}

int ekor_init_equilibrium(ekor *s) {
    if (!s) return EK_ERR_INVALID;
    init_equilibrium(*s);
    s->steps = 0;
    return EK_OK;
}

// One step of the reference loop body (main.cu:194-199).
int ekor_step(ekor *s, int n) {
    if (!s || n < 0) return EK_ERR_INVALID;
    for (int i = 0; i < n; ++i) {
        collide(*s);
        fluid_walls(*s);
        stream(*s);
        ion_walls(*s);
        poisson(*s);
        ++s->steps;
    }
    return EK_OK;
}

int ekor_poisson(ekor *s) {
    if (!s) return EK_ERR_INVALID;
    poisson(*s);
    return EK_OK;
}

int ekor_get_fields(ekor *s, double *rho, double *ux, double *uy, double *cp, double *cn,
                    double *psi, double *ex, double *ey) {
    if (!s) return EK_ERR_INVALID;
    const size_t b = s->nn * sizeof(double);
    if (rho) std::memcpy(rho, s->rho.data(), b);
    if (ux) std::memcpy(ux, s->ux.data(), b);
    if (uy) std::memcpy(uy, s->uy.data(), b);
    if (cp) std::memcpy(cp, s->cp.data(), b);
    if (cn) std::memcpy(cn, s->cn.data(), b);
    if (psi) std::memcpy(psi, s->psi.data(), b);
    if (ex) std::memcpy(ex, s->ex.data(), b);
    if (ey) std::memcpy(ey, s->ey.data(), b);
    return EK_OK;
}

// Pre-collision populations in the reference layout (9*nx*ny per species:
// rest then directions 1..8), for layout-level checks.
int ekor_get_populations(ekor *s, double *f, double *h, double *t) {
    if (!s) return EK_ERR_INVALID;
    const size_t nn = s->nn;
    auto put = [&](double *o, const std::vector<double> &a0, const std::vector<double> &a1) {
        if (!o) return;
        std::memcpy(o, a0.data(), nn * sizeof(double));
        std::memcpy(o + nn, a1.data(), 8 * nn * sizeof(double));
    };
    put(f, s->f0, s->f1);
    put(h, s->h0, s->h1);
    put(t, s->t0, s->t1);
    return EK_OK;
}

}  // extern "C"
