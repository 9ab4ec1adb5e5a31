// Non-uniform grids (host code, no GPU).
//
// lica_grid_section restates one section of the reference's grid generator (grid.f:118-128
// with UNIFORM grid.f:326-345, GEOPRO 348-380, HYPTAN 383-420) in double precision, as the
// solver is built (-fdefault-real-8).  lica_grid_metrics is GEOMETRIC (1d.f:4808-4882) for
// one wall-bounded direction.  lica_mg_stretched_system writes a pressure system on a
// wall-normal grid stretched in y in the form the uniform-grid multigrid solves.
#include <cmath>
#include <string>

#include "lica_gpu.h"

void lica_set_last_error(const char* what, const char* msg, const char* file, int line);

namespace {

int bad(const char* what, const std::string& msg, int line) {
    lica_set_last_error(what, msg.c_str(), __FILE__, line);
    return LICA_BAD_ARG;
}

}  // namespace

extern "C" {

int lica_grid_section(int32_t iopt, double xyzi, double xyzf, int32_t ngi, int32_t ngf, double fac1, double fac2,
                      double* xyz) {
    if (!xyz || ngi < 1 || ngf <= ngi) return bad("lica_grid_section", "need 1 <= ngi < ngf and an array", __LINE__);
    double* X = xyz - 1;  // X[N] = XYZ(N), N = ngi..ngf
    if (iopt == 1) {
        // UNIFORM
        const double dc = (xyzf - xyzi) / (ngf - ngi);
        for (int n = ngi; n <= ngf; ++n) X[n] = xyzi + (n - ngi) * dc;
    } else if (iopt == 2) {
        // GEOPRO: ER = fac1 (the expansion ratio; its inverse when YESEXP = fac2 /= 1)
        double er = fac1;
        if (er == 1.0) return bad("lica_grid_section", "Expansion Ratio is 1 (grid.f:358-361)", __LINE__);
        if (fac2 != 1.0) er = 1.0 / er;
        const double dsi = (xyzf - xyzi) * (1.0 - er) / (1.0 - std::pow(er, ngf - ngi));
        for (int n = ngi + 1; n <= ngf - 1; ++n) X[n] = xyzi + dsi * (1.0 - std::pow(er, n - ngi)) / (1.0 - er);
        X[ngi] = xyzi;
        X[ngf] = xyzf;
    } else if (iopt == 3) {
        // HYPTAN: GAM = fac1, XSI = fac2 (1 flat plate, 0.5 channel, 0 the compressed form)
        const double gam = fac1;
        if (fac2 != 0.0) {
            const double xsi = fac2;
            for (int n = ngi; n <= ngf; ++n) {
                const double seg = (double)(n - ngi) / (double)(ngf - ngi);
                X[n] = xyzi + (xyzf - xyzi) * xsi * (1.0 - std::tanh(gam * (xsi - seg)) / std::tanh(gam * xsi));
            }
        } else {
            const double xsi = 1.0;
            for (int n = ngi; n <= ngf; ++n) {
                const double seg = (double)(n - ngi) / (double)(ngf - ngi);
                X[n] = xyzi + (xyzf - xyzi) * xsi * std::tanh(gam * seg) / std::tanh(gam * xsi);
            }
        }
    } else {
        // grid.f:126-130 calls HYPTAN for any IOPT other than 1 and 2
        return lica_grid_section(3, xyzi, xyzf, ngi, ngf, fac1, fac2, xyz);
    }
    return LICA_OK;
}

int lica_grid_metrics(int32_t n, const double* z, double* sdz, double* vdz, double* ssdz, double* vvdz, double* zp) {
    if (n < 2 || !z || !sdz || !vdz || !ssdz || !vvdz || !zp)
        return bad("lica_grid_metrics", "need n >= 2 faces and every array", __LINE__);
    const int nm = n - 1;
    for (int k = 0; k <= n; ++k) sdz[k] = vdz[k] = ssdz[k] = vvdz[k] = zp[k] = 0.0;
    if (nm == 1) {
        // one cell: ZL = 1 (1d.f:4846-4851)
        sdz[1] = 1.0 / nm;
        ssdz[1] = 1.0 / sdz[1];
        vdz[1] = sdz[1];
        vvdz[1] = ssdz[1];
    } else {
        for (int k = 1; k <= nm; ++k) sdz[k] = z[k + 1] - z[k];
        for (int k = 2; k <= nm; ++k) vdz[k] = 0.5 * (sdz[k] + sdz[k - 1]);
        vdz[1] = 0.5 * sdz[1];
        vdz[n] = 0.5 * sdz[nm];
        for (int k = 1; k <= nm; ++k) {
            if (!(sdz[k] > 0.0)) return bad("lica_grid_metrics", "faces must increase", __LINE__);
            ssdz[k] = 1.0 / sdz[k];
        }
        for (int k = 1; k <= n; ++k) vvdz[k] = 1.0 / vdz[k];
    }
    sdz[0] = 0.0;
    for (int k = 1; k <= nm; ++k) zp[k] = z[k] + 0.5 * sdz[k];
    zp[n] = z[n];
    zp[0] = z[1];
    return LICA_OK;
}

// The stretched operator (a cell of height dy_j = y_{j+1} - y_j, centre distances
// vd_j = (dy_j + dy_{j-1}) / 2, vd_ny = dy_{ny-1} / 2 to the top face where p = 0):
//   (1/hx^2) [bx_{i+1}(p_e - p) - bx_i(p - p_w)] + (1/dy_j) [by_{j+1}/vd_{j+1} (p_n - p)
//   - by_j/vd_j (p - p_s)] = f,
// the 2-D form of POISSON's AK / CK = VVDZ SSDZ DENF_ZI (1d.f:3535-3541) with x uniform.
// Multiplied by dy_j it is symmetric and is the multigrid's operator with hy = 1:
// bx' = bx dy_j, by'_j = by_j / vd_j (the top row by / dy_{ny-1}, which the multigrid
// doubles), f' = f dy_j.  Row 0 of by is the Neumann wall and is copied.
int lica_mg_stretched_system(int32_t nx, int32_t ny, const double* yface, const double* bx, const double* by,
                             const double* f, double* bx_out, double* by_out, double* f_out) {
    if (nx < 1 || ny < 2 || !yface || !bx || !by || !f || !bx_out || !by_out || !f_out)
        return bad("lica_mg_stretched_system", "need nx >= 1, ny >= 2 and every array", __LINE__);
    for (int j = 0; j < ny; ++j)
        if (!(yface[j + 1] > yface[j])) return bad("lica_mg_stretched_system", "faces must increase", __LINE__);
    const size_t NX = (size_t)nx;
    for (int j = 0; j < ny; ++j) {
        const double dy = yface[j + 1] - yface[j];
        for (size_t i = 0; i < NX; ++i) {
            bx_out[j * NX + i] = bx[j * NX + i] * dy;
            f_out[j * NX + i] = f[j * NX + i] * dy;
        }
    }
    for (size_t i = 0; i < NX; ++i) by_out[i] = by[i];
    for (int j = 1; j <= ny; ++j) {
        const double dyb = yface[j] - yface[j - 1];
        const double vd = (j < ny) ? 0.5 * ((yface[j + 1] - yface[j]) + dyb) : dyb;
        for (size_t i = 0; i < NX; ++i) by_out[j * NX + i] = by[j * NX + i] / vd;
    }
    return LICA_OK;
}

}  // extern "C"
