// ek_io.cu -- the reference's file formats and diagnostics, on host arrays
// (host code only; no device work).
//
//   restart   data_end.dat: one line per node, y-major, x fastest, nine
//             "%10.6f" columns time ux uy rho c+ phi Ex Ey c-
//             (save_data_end LBM.cu:1272-1312, read_data LBM.cu:1350-1392)
//   Tecplot   VARIABLES header on the first zone, one POINT zone per call with
//             derived fields: charge gradient, vorticity, its Laplacian, the
//             curl of the electric force (save_data_tecplot LBM.cu:1100-1270)
//   DMD       c+ column of the DMD snapshots (save_data_dmd LBM.cu:1314-1348)
//   current   I = K dy sum_x c+(x, top) Ey(x, top) after the reference's
//             linear extrapolation of the wall rows (current LBM.cu:1394-1417)
//   umax      the maximum of u_y after extrapolating the top row, as the
//             reference computes it (record_umax LBM.cu:1419-1451)
// The reference extrapolates wall rows of its host copies in place; these
// functions work on copies and leave the caller's arrays unchanged.
#include <cstdio>
#include <string>
#include <vector>

#include "ek_ctx.h"

namespace {

inline size_t at(int nx, int x, int y) { return (size_t)nx * y + x; }

// v[row] = 2 v[row+d] - v[row+2d] along x (wall-row extrapolation)
void extrapolate(std::vector<double> &v, int nx, int row, int d) {
    for (int x = 0; x < nx; ++x) v[at(nx, x, row)] = 2.0 * v[at(nx, x, row + d)] - v[at(nx, x, row + 2 * d)];
}

int bad(const char *msg) { return ek::ctx_fail(EK_ERR_INVALID, msg); }

}  // namespace

extern "C" {

int ek_write_restart(const char *path, int32_t nx, int32_t ny, double time, const double *ux, const double *uy,
                     const double *rho, const double *cp, const double *psi, const double *ex, const double *ey,
                     const double *cn) {
    if (!path || nx <= 0 || ny <= 0 || !ux || !uy || !rho || !cp || !psi || !ex || !ey || !cn)
        return bad("bad restart arguments");
    FILE *f = std::fopen(path, "w");
    if (!f) return bad((std::string("cannot open ") + path).c_str());
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(nx, x, y);
            std::fprintf(f, "%10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f\n", time, ux[i], uy[i],
                         rho[i], cp[i], psi[i], ex[i], ey[i], cn[i]);
        }
    const bool ok = std::fclose(f) == 0;
    return ok ? EK_OK : bad("write error");
}

int ek_read_restart(const char *path, int32_t nx, int32_t ny, double *time, double *ux, double *uy, double *rho,
                    double *cp, double *psi, double *ex, double *ey, double *cn) {
    if (!path || nx <= 0 || ny <= 0 || !time || !ux || !uy || !rho || !cp || !psi || !ex || !ey || !cn)
        return bad("bad restart arguments");
    FILE *f = std::fopen(path, "r");
    if (!f) return bad((std::string("cannot open ") + path).c_str());
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(nx, x, y);
            if (std::fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf %lf", time, &ux[i], &uy[i], &rho[i], &cp[i], &psi[i],
                            &ex[i], &ey[i], &cn[i]) != 9) {
                std::fclose(f);
                return bad("restart file shorter than nx*ny lines of nine numbers");
            }
        }
    std::fclose(f);
    return EK_OK;
}

int ek_write_tecplot(const char *path, int32_t first, double time, int32_t nx, int32_t ny, double dx, double dy,
                     const double *ux_in, const double *uy_in, const double *rho_in, const double *cp_in,
                     const double *psi, const double *ex, const double *ey, const double *cn_in) {
    if (!path || nx < 3 || ny < 6 || !ux_in || !uy_in || !rho_in || !cp_in || !psi || !ex || !ey || !cn_in)
        return bad("bad Tecplot arguments (nx >= 3, ny >= 6)");
    const size_t n = (size_t)nx * ny;
    std::vector<double> ux(ux_in, ux_in + n), uy(uy_in, uy_in + n), rho(rho_in, rho_in + n), cp(cp_in, cp_in + n),
        cn(cn_in, cn_in + n), rdx(n, 0.0), rdy(n, 0.0), vor(n, 0.0), vdf(n, 0.0), curl(n);
    // the constants of the reference's writer (LBM.cu:1119-1121)
    const double X = 1000.0, Re = 170.07 / 100.0, extu = 0.25;
    for (int y = 1; y < ny - 1; ++y)
        for (int x = 0; x < nx; ++x) {
            const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;  // periodic ends as LBM.cu:1145-1151
            rdx[at(nx, x, y)] = (cp[at(nx, xp, y)] - cp[at(nx, xm, y)]) / dx / 2;
            rdy[at(nx, x, y)] = (cp[at(nx, x, y + 1)] - cp[at(nx, x, y - 1)]) / dy / 2;
            vor[at(nx, x, y)] = (uy[at(nx, xp, y)] - uy[at(nx, xm, y)]) / dx / 2 -
                                (ux[at(nx, x, y + 1)] - ux[at(nx, x, y - 1)]) / dy / 2;
        }
    for (int y = 2; y < ny - 4; ++y)
        for (int x = 1; x < nx - 1; ++x)
            vdf[at(nx, x, y)] = (vor[at(nx, x + 1, y)] + vor[at(nx, x, y + 1)] + vor[at(nx, x - 1, y)] +
                                 vor[at(nx, x, y - 1)] - 4 * vor[at(nx, x, y)]) / (dy * dy);
    for (int y = 1; y < ny - 2; ++y) {  // periodic end columns (LBM.cu:1175-1179)
        const int a = 0, b = nx - 1;
        vdf[at(nx, a, y)] = (vor[at(nx, 1, y)] + vor[at(nx, a, y + 1)] + vor[at(nx, b, y)] + vor[at(nx, a, y - 1)] -
                             4 * vor[at(nx, a, y)]) / (dy * dy);
        vdf[at(nx, b, y)] = (vor[at(nx, a, y)] + vor[at(nx, b, y + 1)] + vor[at(nx, b - 1, y)] +
                             vor[at(nx, b, y - 1)] - 4 * vor[at(nx, b, y)]) / (dy * dy);
    }
    for (std::vector<double> *v : {&rho, &cp, &cn, &ux, &uy, &rdx, &rdy, &vor}) {
        extrapolate(*v, nx, 0, 1);
        extrapolate(*v, nx, ny - 1, -1);
    }
    for (int x = 0; x < nx; ++x) {  // copies of the nearest computed row (LBM.cu:1189-1210)
        vdf[at(nx, x, 1)] = vdf[at(nx, x, 2)];
        vdf[at(nx, x, 0)] = vdf[at(nx, x, 1)];
        vdf[at(nx, x, ny - 4)] = vdf[at(nx, x, ny - 5)];
        vdf[at(nx, x, ny - 3)] = vdf[at(nx, x, ny - 4)];
        vdf[at(nx, x, ny - 2)] = vdf[at(nx, x, ny - 3)];
        vdf[at(nx, x, ny - 1)] = vdf[at(nx, x, ny - 2)];
    }
    for (size_t i = 0; i < n; ++i) {
        curl[i] = (rdx[i] * ey[i] - rdy[i] * ex[i]) / 1e5;
        vor[i] = vor[i] / extu;
        vdf[i] = vdf[i] / extu;
    }
    FILE *f = std::fopen(path, first ? "w" : "a");
    if (!f) return bad((std::string("cannot open ") + path).c_str());
    if (first)
        std::fprintf(f, "%s\n",
                     "VARIABLES=\"x\",\"y\",\"u\",\"v\",\"p\",\"Positive charge\",\"phi\",\"Ex\",\"Ey\",\"vorticity\","
                     "\"curlForce\",\"vorticity_diff\",\"XcurlForce\",\"Negative charge\"");
    std::fprintf(f, "\n");
    std::fprintf(f, "ZONE T=\"t=%g\", F=POINT, I = %d, J = %d\n", time, nx, ny);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(nx, x, y);
            std::fprintf(f,
                         "%g %g %10.12f %10.12f %10.12f %10.12f %10.12f %10.12f %10.12f %10.12f %10.12f %10.12f "
                         "%10.12f %10.12f\n",
                         dx * x, dy * y, ux[i], uy[i], rho[i], cp[i], psi[i], ex[i], ey[i], vor[i], curl[i],
                         1 / Re * vdf[i], X * curl[i], cn[i]);
        }
    return std::fclose(f) == 0 ? EK_OK : bad("write error");
}

int ek_write_dmd(const char *path, int32_t append, int32_t nx, int32_t ny, const double *cp_in) {
    if (!path || nx <= 0 || ny < 3 || !cp_in) return bad("bad DMD arguments");
    std::vector<double> cp(cp_in, cp_in + (size_t)nx * ny);
    extrapolate(cp, nx, ny - 1, -1);
    FILE *f = std::fopen(path, append ? "a" : "w");
    if (!f) return bad((std::string("cannot open ") + path).c_str());
    for (size_t i = 0; i < cp.size(); ++i) std::fprintf(f, "%10.6f \n", cp[i]);
    return std::fclose(f) == 0 ? EK_OK : bad("write error");
}

int ek_diag_current(int32_t nx, int32_t ny, const double *cp_in, const double *ey, double mob_p, double dy,
                    double *out) {
    if (nx <= 0 || ny < 3 || !cp_in || !ey || !out) return bad("bad current arguments");
    std::vector<double> cp(cp_in, cp_in + (size_t)nx * ny);
    extrapolate(cp, nx, 0, 1);
    extrapolate(cp, nx, ny - 1, -1);
    double I = 0.0;
    for (int x = 0; x < nx; ++x) I += cp[at(nx, x, ny - 1)] * ey[at(nx, x, ny - 1)];
    *out = I * mob_p * dy;
    return EK_OK;
}

int ek_diag_umax(int32_t nx, int32_t ny, const double *uy_in, double *out) {
    if (nx <= 0 || ny < 3 || !uy_in || !out) return bad("bad umax arguments");
    std::vector<double> uy(uy_in, uy_in + (size_t)nx * ny);
    extrapolate(uy, nx, ny - 1, -1);
    double m = 0.0;  // the reference starts from 0 (LBM.cu:1424)
    for (double v : uy) m = v > m ? v : m;
    *out = m;
    return EK_OK;
}

// A context's fields to / from the restart format (LBM.cu:1272-1312,
// 1350-1392): save_data_end and read_data of one channel.
int ek_save_restart(ek_ctx *c, const char *path, double time) {
    if (!c || !path) return bad("null argument");
    const size_t n = (size_t)c->p.nx * c->p.ny;
    std::vector<double> f(8 * n);
    double *rho = &f[0], *ux = &f[n], *uy = &f[2 * n], *cp = &f[3 * n], *cn = &f[4 * n], *psi = &f[5 * n],
           *ex = &f[6 * n], *ey = &f[7 * n];
    int rc = ek_get_fields(c, rho, ux, uy, cp, cn, psi, ex, ey);
    if (rc != EK_OK) return rc;
    return ek_write_restart(path, c->p.nx, c->p.ny, time, ux, uy, rho, cp, psi, ex, ey, cn);
}

int ek_load_restart(ek_ctx *c, const char *path, double *time) {
    if (!c || !path || !time) return bad("null argument");
    const size_t n = (size_t)c->p.nx * c->p.ny;
    std::vector<double> f(8 * n);
    double *rho = &f[0], *ux = &f[n], *uy = &f[2 * n], *cp = &f[3 * n], *cn = &f[4 * n], *psi = &f[5 * n],
           *ex = &f[6 * n], *ey = &f[7 * n];
    int rc = ek_read_restart(path, c->p.nx, c->p.ny, time, ux, uy, rho, cp, psi, ex, ey, cn);
    if (rc != EK_OK) return rc;
    return ek_set_fields(c, rho, ux, uy, cp, cn, psi, ex, ey);
}

}  // extern "C"
