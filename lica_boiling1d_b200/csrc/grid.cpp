// Non-uniform grids (host code, no GPU).
//
// lica_grid_section restates one section of the reference's grid generator (grid.f:118-128
// with UNIFORM grid.f:326-345, GEOPRO 348-380, HYPTAN 383-420) in double precision, as the
// solver is built (-fdefault-real-8).  lica_grid_metrics is GEOMETRIC (1d.f:4808-4882) for
// one wall-bounded direction.  lica_mg_stretched_system writes a pressure system on a
// wall-normal grid stretched in y in the form the uniform-grid multigrid solves.
// lica_grid_coupling_z is GEOM_COUPLING's z tables (1d.f:5037-5370) between a flow grid of
// any spacing and the uniform level-set grid.
#include <cmath>
#include <string>
#include <vector>

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

namespace {

// The first refined face at or above x (GEOM_COUPLING's face search): (KF-1, KF) when
// ZF(KF) = x within 1e-10, (KF-1, KF-1) when ZF(KF) is the first face above x.
bool face_pair(double x, int n3f, const double* zf, int32_t& a, int32_t& b) {
    for (int kf = 1; kf <= n3f; ++kf) {
        if (std::fabs(zf[kf] - x) <= 1e-10) {
            a = kf - 1;
            b = kf;
            return true;
        } else if (zf[kf] > x) {
            a = kf - 1;
            b = kf - 1;
            return true;
        }
    }
    return false;
}

// KCOU_VEL / KCOUMP_VEL: the flow centre at or below zz, by the reference's test order.
int centre_below(double zz, int n3m, const double* zp) {
    for (int kk = 1; kk <= n3m; ++kk) {
        if (std::fabs(zz - zp[kk]) <= 1e-10) return kk;
        if (zp[1] > zz) return 1;
        if (zp[kk] > zz) return kk - 1;
        if (zp[n3m] < zz) return n3m;
    }
    return -1;
}

}  // namespace

int lica_grid_coupling_z(int32_t n3, const double* z, int32_t n3f, const double* zf, int32_t* kcou1, int32_t* kcou2,
                         int32_t* kcoump1, int32_t* kcoump2, int32_t* kcou_vel, int32_t* kcoump_vel) {
    if (n3 < 4 || n3f < 3 || !z || !zf || !kcou1 || !kcou2 || !kcoump1 || !kcoump2 || !kcou_vel || !kcoump_vel)
        return bad("lica_grid_coupling_z", "need n3 >= 4 flow faces, n3f >= 3 refined faces and every array",
                   __LINE__);
    const int n3m = n3 - 1;
    // GEOMETRIC's ZP (1d.f:4873-4876) and GEOMETRIC_LVS's ZPF (1d.f:4928-4938)
    std::vector<double> zp(n3 + 1), zpf(n3f + 1);
    for (int k = 1; k <= n3m; ++k) zp[k] = z[k] + 0.5 * (z[k + 1] - z[k]);
    zp[n3] = z[n3];
    zp[0] = z[1];
    const double sdzf = zf[2] - zf[1];
    for (int k = 1; k <= n3f; ++k) zpf[k] = zf[k] + 0.5 * sdzf;
    auto K1 = [&](int k) -> int32_t& { return kcou1[k + 1]; };
    auto K2 = [&](int k) -> int32_t& { return kcou2[k + 1]; };
    auto M1 = [&](int k) -> int32_t& { return kcoump1[k + 1]; };
    auto M2 = [&](int k) -> int32_t& { return kcoump2[k + 1]; };
    // KCOU_VEL / KCOUMP_VEL (1d.f:5142-5190)
    for (int k = 1; k <= n3f; ++k) {
        const int a = centre_below(zf[k], n3m, zp.data()), b = centre_below(zpf[k], n3m, zp.data());
        if (a < 0 || b < 0) return bad("lica_grid_coupling_z", "Z-DIR FLOW_SOLVER->REFINED COUPLING PROBLEM", __LINE__);
        kcou_vel[k] = a;
        kcoump_vel[k] = b;
    }
    kcou_vel[0] = kcoump_vel[0] = 0;
    // KCOU1 / KCOU2 of the faces and KCOUMP1 / KCOUMP2 of the centres (1d.f:5308-5363)
    for (int k = 1; k <= n3; ++k)
        if (!face_pair(z[k], n3f, zf, K1(k), K2(k)))
            return bad("lica_grid_coupling_z", "CAL KCOU HAVE PROBLEM: a flow face above the refined grid", __LINE__);
    K1(0) = K1(1) - (K1(n3m) - K1(n3m - 1));
    K1(-1) = K1(0) - (K1(n3m - 1) - K1(n3m - 2));
    K1(n3 + 1) = K1(n3) + (K1(2) - K1(1));
    K1(n3 + 2) = K1(n3 + 1) + (K1(3) - K1(2));
    K2(0) = K2(1) - (K2(n3m) - K2(n3m - 1));
    K2(-1) = K2(0) - (K2(n3m - 1) - K2(n3m - 2));
    K2(n3 + 1) = K2(n3) + (K2(2) - K2(1));
    K2(n3 + 2) = K2(n3 + 1) + (K2(3) - K2(2));
    for (int k = 1; k <= n3m; ++k)
        if (!face_pair(zp[k], n3f, zf, M1(k), M2(k)))
            return bad("lica_grid_coupling_z", "CAL KCOUMP HAVE PROBLEM: a flow centre above the refined grid",
                       __LINE__);
    M1(0) = M1(1) - (M1(n3m) - M1(n3m - 1));
    M1(-1) = M1(0) - (M1(n3m - 1) - M1(n3m - 2));
    M1(n3) = M1(n3m) + (M1(n3m) - M1(n3m - 1));
    M1(n3 + 1) = M1(n3) + (M1(2) - M1(1));
    M2(0) = M2(1) - (M2(n3m) - M2(n3m - 1));
    M2(-1) = M2(0) - (M2(n3m - 1) - M2(n3m - 2));
    M2(n3) = M2(n3m) + (M2(n3m) - M2(n3m - 1));
    M2(n3 + 1) = M2(n3) + (M2(2) - M2(1));
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
