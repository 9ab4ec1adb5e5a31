// One RK3 time step of the 2-D film-boiling model on a B200: a MAC flow grid of nx x ny
// cells (x periodic, y the reference's wall-normal z with a heated no-slip wall at the bottom
// and an outflow top with p = 0 on the face) and the level set on the 2x refined grid.
//
// The step generalises the reference's 1-D hot-path rows to 2-D:
//   RK3COEF substeps (1d.f:1310-1322) with stored right-hand sides; properties linear in the
//   liquid fraction psi (1d.f:437-489) with psi from a smoothed Heaviside of the refined level
//   set (GRID_COUPLING / CAL_PSIF's role, two_phase.f:2503-5538); explicit momentum with
//   central convection, the full variable-viscosity stress and the buoyancy of the modified
//   pressure p + rho_l g y (RHSZ / LHSW's role, 1d.f:1603-1809); the incremental projection
//   (predictor with -alpha dt beta grad p, div(beta grad dp) = (div u* - S) / (alpha dt)
//   solved from zero by the 2-D multigrid (mg.cu), u -= alpha dt beta grad dp, p += dp:
//   PRESSURE_CORRECTION's role); the phase-change mass flux mdot = Ja/(Re Pr) k max(0, -grad theta .
//   grad psi) with the volume source S = mdot (1/rho_v - 1/rho_l) (TEMP_GRAD / TF_GRAD /
//   VOL_TOT_MFDOT / CAL_CONTINUITY2's role); the energy update with theta = 0 in the liquid
//   (PASSIVE_SCALAR / TEMPASSIGN's role); TRANSPORT_RK3 with the reference's HJWENO in x and y
//   (two_phase.f:1133-1495, 2477-2500); REINITIALIZATION's SSP-RK3 pseudo-time iterations with
//   GODUNOV and Peng's smoothed sign (two_phase.f:2033-2474).
// Surface tension is CAL_CUR's SURF CUR dpsi/dx / rho_f on the faces where psi jumps, with
// CAL_CUR / CAL_CUR_INTEGRAL / INTER_CUR (two_phase.f:3317-4432) restated in 2-D below.
// Simplifications: no interface recession term, explicit viscous terms.
//
// Every kernel is one thread per output cell, 32 x 8 thread blocks (coalesced rows), and
// evaluates each expression in a fixed order; the library is compiled without FMA
// contraction, so every field equals the CPU restatement bit for bit except through the
// iterative pressure solve.
//
// Layout (row-major, x fastest): u (ny, nx) on the face west of cell i; v (ny + 1, nx) on the
// face below cell row j (v[0] = 0, v[ny] the top); p, theta (ny, nx); phi (2 ny, 2 nx).
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

#include "common.cuh"
#include "lica_gpu.h"

extern "C" void lica_count_launches(int64_t n);

namespace lica {
namespace film2d {

constexpr double kGamma[4] = {0.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
constexpr double kRo[4] = {0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0};

// Constants of the step (the CPU restatement computes the same expressions).
struct Const {
    int nx, ny, nxf, nyf;
    double h, hf, ih, ih2, inv2h, ihsq, ihf, eps_h, inv2e, hf2, redtl, band, ih2f, ihfsq, q4;
    double denm, den_diff, vism, vis_diff, denscm, densc_diff, tcm, tc_diff, pei, cmd, cvol, gravity, denp, surf;
};

Const make_const(int nx, int ny, const lica_film2d_props& P) {
    Const c{};
    c.nx = nx;
    c.ny = ny;
    c.nxf = 2 * nx;
    c.nyf = 2 * ny;
    c.h = 1.0 / nx;
    c.hf = 0.5 * c.h;
    c.ih = 1.0 / c.h;
    c.ih2 = 2.0 / c.h;
    c.inv2h = 0.5 / c.h;
    c.ihsq = 1.0 / (c.h * c.h);
    c.ihf = 1.0 / c.hf;
    c.eps_h = c.h;
    c.inv2e = 1.0 / (2.0 * c.eps_h);
    c.hf2 = c.hf * c.hf;
    c.redtl = 0.5 * c.hf;
    c.band = 8.0 * c.hf;
    c.denm = 1.0;
    c.den_diff = P.denr - 1.0;
    c.vism = 1.0 / P.re;
    c.vis_diff = P.visr / P.re - 1.0 / P.re;
    c.denscm = 1.0;
    c.densc_diff = P.denr * P.scr - 1.0;
    c.tcm = 1.0;
    c.tc_diff = P.tcr - 1.0;
    c.pei = 1.0 / (P.re * P.prm);
    c.cmd = P.jakob * c.pei;
    c.cvol = 1.0 / 1.0 - 1.0 / P.denr;
    c.gravity = (P.fr == 0.0) ? 0.0 : 1.0 / (P.fr * P.fr);
    c.denp = P.denr;
    c.surf = (P.we == 0.0) ? 0.0 : 1.0 / P.we;
    c.ih2f = 0.5 / c.hf;
    c.ihfsq = 1.0 / (c.hf * c.hf);
    c.q4 = 0.25 * c.ihfsq;
    return c;
}

__device__ __forceinline__ int east(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int west(int i, int n) { return i == 0 ? n - 1 : i - 1; }

__device__ __forceinline__ double heaviside(double x, const Const& c) {
    if (x <= -c.eps_h) return 0.0;
    if (x >= c.eps_h) return 1.0;
    const double s = (x + c.eps_h) * c.inv2e;
    return s * s * s * (10.0 + s * (-15.0 + 6.0 * s));
}

// ---------------------------------------------------------------- flow-grid kernels
// psi, den, vis, densc, tc per cell.
__global__ void k_props(const double* __restrict__ phi, double* __restrict__ psi, double* __restrict__ den,
                        double* __restrict__ vis, double* __restrict__ densc, double* __restrict__ tc, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const double* r0 = phi + (size_t)(2 * j) * c.nxf;
    const double* r1 = r0 + c.nxf;
    const double q = (heaviside(r0[2 * i], c) + heaviside(r0[2 * i + 1], c)) +
                     (heaviside(r1[2 * i], c) + heaviside(r1[2 * i + 1], c));
    const double ps = 0.25 * q;
    const size_t k = (size_t)j * c.nx + i;
    psi[k] = ps;
    den[k] = c.denm + c.den_diff * ps;
    vis[k] = c.vism + c.vis_diff * ps;
    densc[k] = c.denscm + c.densc_diff * ps;
    tc[k] = c.tcm + c.tc_diff * ps;
}

// ---------------------------------------------------------------- CAL_CUR in 2-D
// CAL_CUR(N_CUR = 4) (two_phase.f:2792, 3317-4432) on the refined grid, x periodic, y indices
// clamped: (1) CURF_TMP, the curvature -(GXX GZ^2 + GZZ GX^2 - 2 GXZ GX GZ) / |grad phi|^3 by
// central differences on band layers 1..N_CUR+1 (:3362-3397; the reference's y terms vanish
// exactly for a field constant in y; |g|^3 = g2 sqrt(g2)); (2) CURF, CURF_TMP interpolated to
// the foot of each cell of layers 1..N_CUR on the interface (:3405-3458, the trilinear form
// with YD = 0); (3) per flow face where psi jumps, INTER_CUR's mean of CURF over the face box's
// refined cells cut by the interface (0 < psi_f < 1, CURF /= 0), or over the box twice as wide
// if it holds none (CAL_CUR_INTEGRAL, :3654-3795).  On the uniform 2x refinement the boxes
// are whole refined cells.  A band layer m is |phi| < m hf.
constexpr int kNCur = 4;

__global__ void k_cur_tmp(const double* __restrict__ phi, double* __restrict__ kt, const Const c) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= c.nxf || J >= c.nyf) return;
    const int nxf = c.nxf, nyf = c.nyf;
    const double* row = phi + (size_t)J * nxf;
    const double C = row[I];
    double out = 0.0;
    if (fabs(C) < (kNCur + 1) * c.hf) {
        const int Ie = (I + 1 == nxf) ? 0 : I + 1, Iw = (I == 0) ? nxf - 1 : I - 1;
        const double* up = phi + (size_t)(J + 1 < nyf ? J + 1 : nyf - 1) * nxf;
        const double* dn = phi + (size_t)(J > 0 ? J - 1 : 0) * nxf;
        const double E = row[Ie], W = row[Iw], N = up[I], S = dn[I];
        const double gx = 0.5 * (E - W) * c.ihf;
        const double gz = 0.5 * (N - S) * c.ihf;
        const double gxx = ((E - 2.0 * C) + W) * c.ihf * c.ihf;
        const double gzz = ((N - 2.0 * C) + S) * c.ihf * c.ihf;
        const double gxz = 0.25 * ((up[Ie] - up[Iw]) - (dn[Ie] - dn[Iw])) * c.ihf * c.ihf;
        const double g2 = gx * gx + gz * gz;
        if (g2 > 0.0) {
            const double num = (gxx * (gz * gz) + gzz * (gx * gx)) - 2.0 * (gxz * gx * gz);
            out = -num / (g2 * sqrt(g2));
        }
    }
    kt[(size_t)J * nxf + I] = out;
}

__global__ void k_cur_foot(const double* __restrict__ phi, const double* __restrict__ kt, double* __restrict__ cf,
                           const Const c) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= c.nxf || J >= c.nyf) return;
    const int nxf = c.nxf, nyf = c.nyf;
    const double C = phi[(size_t)J * nxf + I];
    double out = 0.0;
    if (fabs(C) < kNCur * c.hf) {
        const int Ie = (I + 1 == nxf) ? 0 : I + 1, Iw = (I == 0) ? nxf - 1 : I - 1;
        const int Jn = J + 1 < nyf ? J + 1 : nyf - 1, Js = J > 0 ? J - 1 : 0;
        const double dpx = 0.5 * (phi[(size_t)J * nxf + Ie] - phi[(size_t)J * nxf + Iw]) * c.ihf;
        const double dpz = 0.5 * (phi[(size_t)Jn * nxf + I] - phi[(size_t)Js * nxf + I]) * c.ihf;
        const double g2 = dpx * dpx + dpz * dpz;
        if (g2 > 0.0) {
            const double amdpi = 1.0 / sqrt(g2);
            const double dis = C * amdpi;
            const double xp = (I + 0.5) * c.hf, zp = (J + 0.5) * c.hf;
            const double xb = xp - dis * (dpx * amdpi), zb = zp - dis * (dpz * amdpi);
            int i1, i2, j1, j2;
            double xd, zd;
            if (xb >= xp) {
                xd = (xb - xp) * c.ihf;
                i1 = I;
                i2 = Ie;
            } else {
                xd = (xb - (xp - c.hf)) * c.ihf;
                i1 = Iw;
                i2 = I;
            }
            if (zb >= zp) {
                zd = (zb - zp) * c.ihf;
                j1 = J;
                j2 = Jn;
            } else {
                zd = (zb - (zp - c.hf)) * c.ihf;
                j1 = Js;
                j2 = J;
            }
            const double c00 = kt[(size_t)j1 * nxf + i1] * (1.0 - xd) + kt[(size_t)j1 * nxf + i2] * xd;
            const double c01 = kt[(size_t)j2 * nxf + i1] * (1.0 - xd) + kt[(size_t)j2 * nxf + i2] * xd;
            out = c00 * (1.0 - zd) + c01 * zd;
        }
    }
    cf[(size_t)J * nxf + I] = out;
}

// INTER_CUR over refined columns c0..c0+nc-1 (x periodic) and rows r0..r0+nr-1, column by
// column; returns the cut-cell count (VOLF) and leaves the mean in cur when it is not 0.
__device__ __forceinline__ double inter_cur(const double* __restrict__ phi, const double* __restrict__ cf, int c0,
                                            int nc, int r0, int nr, const Const& c, double& cur) {
    const int nxf = c.nxf;
    double sum = 0.0, volf = 0.0;
    for (int a = 0; a < nc; ++a) {
        int II = c0 + a;
        II = II < 0 ? II + nxf : (II >= nxf ? II - nxf : II);
        for (int b = 0; b < nr; ++b) {
            const size_t q = (size_t)(r0 + b) * nxf + II;
            const double hh = heaviside(phi[q], c);
            const double v = cf[q];
            if (hh > 0.0 && hh < 1.0 && v != 0.0) {
                sum = sum + v;
                volf = volf + 1.0;
            }
        }
    }
    if (volf != 0.0) cur = sum / volf;
    return volf;
}

// Face curvatures: cx on the face west of cell (i, j), cy on the face below it (row 0, the
// wall: 0).
__global__ void k_face_cur(const double* __restrict__ phi, const double* __restrict__ cf,
                           const double* __restrict__ psi, double* __restrict__ cx, double* __restrict__ cy,
                           const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx;
    const size_t k = (size_t)j * nx + i;
    double vx = 0.0, vy = 0.0;
    if ((psi[k] - psi[(size_t)j * nx + west(i, nx)]) != 0.0) {
        if (inter_cur(phi, cf, 2 * i - 1, 2, 2 * j, 2, c, vx) == 0.0) inter_cur(phi, cf, 2 * i - 2, 4, 2 * j, 2, c, vx);
    }
    if (j >= 1 && (psi[k] - psi[k - nx]) != 0.0) {
        if (inter_cur(phi, cf, 2 * i, 2, 2 * j - 1, 2, c, vy) == 0.0) inter_cur(phi, cf, 2 * i, 2, 2 * j - 2, 4, c, vy);
    }
    cx[k] = vx;
    cy[k] = vy;
}

// Face coefficients beta = 1/rho: bx by harmonic mean (x periodic), by on rows 0..ny.
__global__ void k_beta(const double* __restrict__ den, double* __restrict__ bx, double* __restrict__ by, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx, ny = c.ny;
    const double d = den[(size_t)j * nx + i];
    bx[(size_t)j * nx + i] = 2.0 / (den[(size_t)j * nx + west(i, nx)] + d);
    by[(size_t)j * nx + i] = (j == 0) ? 1.0 / d : 2.0 / (den[(size_t)(j - 1) * nx + i] + d);
    if (j == ny - 1) by[(size_t)ny * nx + i] = 1.0 / d;
}

// Momentum predictor with the current pressure gradient: u* at the face west of cell (i, j)
// and v* at the face above it (j + 1 = 1..ny); the right-hand sides are stored for the next
// substep.
__global__ void k_momentum(const double* __restrict__ u, const double* __restrict__ v,
                           const double* __restrict__ den, const double* __restrict__ vis,
                           const double* __restrict__ psi, const double* __restrict__ cx,
                           const double* __restrict__ cy, const double* __restrict__ p, const double* __restrict__ bx,
                           const double* __restrict__ by, double* __restrict__ us, double* __restrict__ vs,
                           double* __restrict__ ru, double* __restrict__ rv, double dt, double gam, double ro,
                           double adt, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx, ny = c.ny, ie = east(i, nx), iw = west(i, nx);
    const double ih = c.ih;
    const size_t k = (size_t)j * nx + i;
    const double* urow = u + (size_t)j * nx;
    const double* urn = (j + 1 < ny) ? urow + nx : u + (size_t)(ny - 1) * nx;  // row j+1 (top: copy)
    const double* vrow = v + (size_t)j * nx;                                    // face below cell j
    const double* vrn = vrow + nx;                                              // face above cell j
    const double* mrow = vis + (size_t)j * nx;
    const double* mrn = (j + 1 < ny) ? mrow + nx : vis + (size_t)(ny - 1) * nx;
    const double* mrs = (j > 0) ? mrow - nx : vis;
    {
        // u at the face west of cell (i, j)
        const double uc = urow[i], ue = urow[ie], uw = urow[iw];
        const double un = urn[i];
        const double usv = (j > 0) ? urow[i - nx] : -u[i];
        const double vn = 0.5 * (vrn[iw] + vrn[i]);
        const double vsv = 0.5 * (vrow[iw] + vrow[i]);
        const double uci = 0.5 * (uc + ue);
        const double ucm = 0.5 * (uw + uc);
        const double conv = (uci * uci - ucm * ucm) * ih + (0.5 * (uc + un) * vn - 0.5 * (usv + uc) * vsv) * ih;
        const double mc = mrow[i], mw = mrow[iw];
        const double txe = 2.0 * mc * (ue - uc) * ih;
        const double txw = 2.0 * mw * (uc - uw) * ih;
        const double mun = 0.25 * ((mw + mc) + (mrn[iw] + mrn[i]));
        const double mus = 0.25 * ((mrs[iw] + mrs[i]) + (mw + mc));
        const double tyn = mun * ((un - uc) * ih + (vrn[i] - vrn[iw]) * ih);
        const double tys = mus * ((uc - usv) * ih + (vrow[i] - vrow[iw]) * ih);
        const double rho = 0.5 * (den[(size_t)j * nx + iw] + den[k]);
        const double visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho;
        // surface tension SURF CUR dpsi/dx on the face (CAL_CUR's SUR_X, two_phase.f:3547-3556)
        const double nu = visc - conv + (c.surf * cx[k]) * ((psi[k] - psi[(size_t)j * nx + iw]) * ih) / rho;
        us[k] = uc + dt * (gam * nu + ro * ru[k]) - adt * (bx[k] * ((p[k] - p[(size_t)j * nx + iw]) * ih));
        ru[k] = nu;
    }
    {
        // v at the face above cell (i, j): face row jf = j + 1
        const int jf = j + 1;
        const double vc = vrn[i], vsv = vrow[i];
        const double vnv = (jf + 1 <= ny) ? vrn[i + nx] : vrn[i];
        const double ve = vrn[ie], vw = vrn[iw];
        const double ulo = urow[i], uhi = urn[i], ulo_e = urow[ie], uhi_e = urn[ie];
        const double vcj = 0.5 * (vc + vnv);
        const double vcm = 0.5 * (vsv + vc);
        const double conv = ((0.5 * (ulo_e + uhi_e)) * (0.5 * (vc + ve)) - (0.5 * (ulo + uhi)) * (0.5 * (vw + vc))) * ih +
                            (vcj * vcj - vcm * vcm) * ih;
        const double mulo = mrow[i], muhi = mrn[i];
        const double tyn = 2.0 * muhi * (vnv - vc) * ih;
        const double tys = 2.0 * mulo * (vc - vsv) * ih;
        const double mue = 0.25 * ((mulo + mrow[ie]) + (muhi + mrn[ie]));
        const double muw = 0.25 * ((mrow[iw] + mulo) + (mrn[iw] + muhi));
        const double txe = mue * ((ve - vc) * ih + (uhi_e - ulo_e) * ih);
        const double txw = muw * ((vc - vw) * ih + (uhi - ulo) * ih);
        const double dlo = den[k], dhi = (j + 1 < ny) ? den[k + nx] : den[(size_t)(ny - 1) * nx + i];
        const double rho = 0.5 * (dlo + dhi);
        const double visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho;
        const size_t khi = (j + 1 < ny) ? k + nx : (size_t)(ny - 1) * nx + i;
        const double cur = (j + 1 < ny) ? cy[k + nx] : 0.0;   // the face above row j (top face: 0)
        const double nv = visc - conv + c.gravity * (c.denp / rho - 1.0) +
                          (c.surf * cur) * ((psi[khi] - psi[k]) * ih) / rho;
        const size_t kf = (size_t)jf * nx + i;
        const double gp = (jf < ny) ? (p[kf] - p[k]) * ih : (0.0 - p[k]) * c.ih2;  // p = 0 on the top face
        vs[kf] = vc + dt * (gam * nv + ro * rv[k]) - adt * (by[kf] * gp);
        rv[k] = nv;
    }
}

// Phase-change volume source and the projection's right-hand side f = (div u* - S) iadt.
__global__ void k_source_rhs(const double* __restrict__ th, const double* __restrict__ psi,
                             const double* __restrict__ tc, const double* __restrict__ us,
                             const double* __restrict__ vs, double* __restrict__ f, double* __restrict__ mdot,
                             double iadt, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx, ny = c.ny, ie = east(i, nx), iw = west(i, nx);
    const size_t k = (size_t)j * nx + i;
    const double tn = (j + 1 < ny) ? th[k + nx] : th[k];
    const double ts = (j > 0) ? th[k - nx] : 2.0 - th[i];
    const double pn = (j + 1 < ny) ? psi[k + nx] : psi[k];
    const double ps = (j > 0) ? psi[k - nx] : psi[i];
    const double gtx = (th[(size_t)j * nx + ie] - th[(size_t)j * nx + iw]) * c.inv2h;
    const double gty = (tn - ts) * c.inv2h;
    const double gpx = (psi[(size_t)j * nx + ie] - psi[(size_t)j * nx + iw]) * c.inv2h;
    const double gpy = (pn - ps) * c.inv2h;
    const double q = -(gtx * gpx + gty * gpy);
    const double md = (c.cmd * tc[k]) * fmax(q, 0.0);
    const double S = md * c.cvol;
    mdot[k] = md;
    const double div = (us[(size_t)j * nx + ie] - us[k]) * c.ih + (vs[k + nx] - vs[k]) * c.ih;
    f[k] = (div - S) * iadt;
}

// u = u* - alpha dt beta grad dp (dp = 0 on the top face), p += dp.
__global__ void k_correct(const double* __restrict__ us, const double* __restrict__ vs, const double* __restrict__ dp,
                          const double* __restrict__ bx, const double* __restrict__ by, double* __restrict__ u,
                          double* __restrict__ v, double* __restrict__ p, double adt, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx, ny = c.ny, iw = west(i, nx);
    const size_t k = (size_t)j * nx + i;
    u[k] = us[k] - adt * (bx[k] * ((dp[k] - dp[(size_t)j * nx + iw]) * c.ih));
    v[k] = (j == 0) ? vs[k] : vs[k] - adt * (by[k] * ((dp[k] - dp[k - nx]) * c.ih));
    if (j == ny - 1) {
        const size_t t = (size_t)ny * nx + i;
        v[t] = vs[t] - adt * (by[t] * ((0.0 - dp[k]) * c.ih2));
    }
    p[k] = p[k] + dp[k];
}

// theta += dt (gam E + ro E_old), E = pei div(k grad theta) / densc - u . grad theta;
// theta = 0 where psi > 1/2.
__global__ void k_energy(const double* __restrict__ th, const double* __restrict__ u, const double* __restrict__ v,
                         const double* __restrict__ densc, const double* __restrict__ tc,
                         const double* __restrict__ psi, double* __restrict__ th_out, double* __restrict__ rth,
                         double dt, double gam, double ro, const Const c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.nx || j >= c.ny) return;
    const int nx = c.nx, ny = c.ny, ie = east(i, nx), iw = west(i, nx);
    const size_t k = (size_t)j * nx + i;
    const double t = th[k];
    const double te = th[(size_t)j * nx + ie], tw = th[(size_t)j * nx + iw];
    const double tn = (j + 1 < ny) ? th[k + nx] : t;
    const double ts = (j > 0) ? th[k - nx] : 2.0 - th[i];
    const double uc = 0.5 * (u[k] + u[(size_t)j * nx + ie]);
    const double vc = 0.5 * (v[k] + v[k + nx]);
    const double adv = uc * ((te - tw) * c.inv2h) + vc * ((tn - ts) * c.inv2h);
    const double kc = tc[k];
    const double ke = 0.5 * (kc + tc[(size_t)j * nx + ie]);
    const double kw = 0.5 * (tc[(size_t)j * nx + iw] + kc);
    const double kn = 0.5 * (kc + ((j + 1 < ny) ? tc[k + nx] : kc));
    const double ks = 0.5 * (((j > 0) ? tc[k - nx] : tc[i]) + kc);
    const double dif = ((ke * (te - t) - kw * (t - tw)) + (kn * (tn - t) - ks * (t - ts))) * c.ihsq;
    const double e = (c.pei * dif) / densc[k] - adv;
    const double thn = t + dt * (gam * e + ro * rth[k]);
    rth[k] = e;
    th_out[k] = (psi[k] > 0.5) ? 0.0 : thn;
}

// ---------------------------------------------------------------- refined-grid kernels
// HJWENO, two_phase.f:2477-2500 (the expression order of lvs_device.cuh).
__device__ __forceinline__ double hjweno(double a, double b, double cc, double dd) {
    const double eps = 1e-6;
    const double s1 = 13.0 * (a - b) * (a - b) + 3.0 * (a - 3.0 * b) * (a - 3.0 * b);
    const double s2 = 13.0 * (b - cc) * (b - cc) + 3.0 * (b + cc) * (b + cc);
    const double s3 = 13.0 * (cc - dd) * (cc - dd) + 3.0 * (3.0 * cc - dd) * (3.0 * cc - dd);
    const double a1 = 1.0 / ((eps + s1) * (eps + s1));
    const double a2 = 6.0 / ((eps + s2) * (eps + s2));
    const double a3 = 3.0 / ((eps + s3) * (eps + s3));
    const double w1 = a1 / (a1 + a2 + a3);
    const double w3 = a3 / (a1 + a2 + a3);
    return 1.0 / 3.0 * w1 * (a - 2.0 * b + cc) + 1.0 / 6.0 * (w3 - 0.5) * (b - 2.0 * cc + dd);
}

// One-sided WENO5 derivatives from the six face differences d[0..5] = dp(c-3 .. c+2).
__device__ __forceinline__ void weno_pair(const double* d, double& dm, double& dpl) {
    {
        const double v1 = d[0], v2 = d[1], v3 = d[2], v4 = d[3], v5 = d[4];
        dm = 1.0 / 12.0 * (-v2 + 7.0 * v3 + 7.0 * v4 - v5) - hjweno(v2 - v1, v3 - v2, v4 - v3, v5 - v4);
    }
    {
        const double q1 = d[5], q2 = d[4], q3 = d[3], q4 = d[2], q5 = d[1];
        dpl = 1.0 / 12.0 * (-q5 + 7.0 * q4 + 7.0 * q3 - q2) + hjweno(q1 - q2, q2 - q3, q3 - q4, q4 - q5);
    }
}

// Face differences around refined cell (I, J): dx[m] = dpx(I - 3 + m) (x periodic) and
// dy[m] = dpy(clamp(J - 3 + m, 0, nyf - 2)), m = 0..5.
__device__ __forceinline__ void face_diffs(const double* __restrict__ phi, int I, int J, const Const& c, double* dx,
                                           double* dy) {
    const int nxf = c.nxf, nyf = c.nyf;
    const double* row = phi + (size_t)J * nxf;
    double f[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        int x = I - 3 + m;
        x = x < 0 ? x + nxf : (x >= nxf ? x - nxf : x);
        f[m] = row[x];
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) dx[m] = (f[m + 1] - f[m]) * c.ihf;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        int y = J - 3 + m;
        y = y < 0 ? 0 : (y > nyf - 2 ? nyf - 2 : y);
        dy[m] = (phi[(size_t)(y + 1) * nxf + I] - phi[(size_t)y * nxf + I]) * c.ihf;
    }
}

// Level-set transport substep on the band |phi| < band (BAND_GENERATION's role): phi_out =
// phi + dt (gam L + ro L_old), L = -(u phi_x + v phi_y) with upwinded WENO5 derivatives and
// the MAC velocity interpolated to the refined centre; cells outside keep phi and store L = 0.
__global__ void k_ls_transport(const double* __restrict__ phi, const double* __restrict__ u,
                               const double* __restrict__ v, double* __restrict__ phi_out,
                               double* __restrict__ rphi, double dt, double gam, double ro, const Const c) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= c.nxf || J >= c.nyf) return;
    const size_t k = (size_t)J * c.nxf + I;
    const double ph0 = phi[k];
    if (!(fabs(ph0) < c.band)) {
        // outside the band: unchanged, no stored right-hand side
        phi_out[k] = ph0;
        rphi[k] = 0.0;
        return;
    }
    const int nx = c.nx, ny = c.ny;
    const int m = I >> 1, a = I & 1, jp = J >> 1, b = J & 1;
    double uf, vf;
    {
        // u: rows r0 = jp - 1 + b and r0 + 1 (row -1: -u[0], row ny: u[ny-1]); faces m, m + 1
        const int r0 = jp - 1 + b, r1 = r0 + 1;
        const int c0 = m, c1 = (m + 1 == nx) ? 0 : m + 1;
        const double wx = a == 0 ? 0.25 : 0.75, wy = b == 0 ? 0.75 : 0.25;
        auto U = [&](int r, int cc) {
            if (r < 0) return -u[cc];
            if (r >= ny) return u[(size_t)(ny - 1) * nx + cc];
            return u[(size_t)r * nx + cc];
        };
        const double a00 = U(r0, c0), a10 = U(r0, c1), a01 = U(r1, c0), a11 = U(r1, c1);
        uf = (1.0 - wy) * ((1.0 - wx) * a00 + wx * a10) + wy * ((1.0 - wx) * a01 + wx * a11);
    }
    {
        // v: columns m - 1 + a and m + a (periodic); face rows jp, jp + 1
        int c0 = m - 1 + a, c1 = m + a;
        c0 = c0 < 0 ? c0 + nx : c0;
        c1 = c1 >= nx ? c1 - nx : c1;
        const double wx = a == 0 ? 0.75 : 0.25, wy = b == 0 ? 0.25 : 0.75;
        const double* r0 = v + (size_t)jp * nx;
        const double* r1 = r0 + nx;
        vf = (1.0 - wy) * ((1.0 - wx) * r0[c0] + wx * r0[c1]) + wy * ((1.0 - wx) * r1[c0] + wx * r1[c1]);
    }
    double dx[6], dy[6];
    face_diffs(phi, I, J, c, dx, dy);
    double dmx, dplx, dmy, dply;
    weno_pair(dx, dmx, dplx);
    weno_pair(dy, dmy, dply);
    const double px = (uf >= 0.0) ? dmx : dplx;
    const double py = (vf >= 0.0) ? dmy : dply;
    const double L = -(uf * px + vf * py);
    phi_out[k] = ph0 + dt * (gam * L + ro * rphi[k]);
    rphi[k] = L;
}

// GODUNOV, two_phase.f:2448-2474.
__device__ __forceinline__ double godunov(double sg, double ap, double am) {
    const double aplus = sg * ap, aminus = sg * am;
    if (aplus >= 0.0 && aminus >= 0.0) return am;
    if (aplus <= 0.0 && aminus <= 0.0) return ap;
    if (aplus > 0.0 && aminus < 0.0) return 0.0;
    if (aplus + aminus > 0.0) return am;
    return ap;
}

// One reinitialisation stage s = phi + redtl sg (1 - |grad phi|_Godunov) on the band
// |a0| < band, written as out = s, 0.75 rk + 0.25 s or rk / 3 + 2 s / 3 (combine 0, 1, 2);
// cells outside the band keep phi.
__global__ void k_reinit_stage(const double* __restrict__ phi, const double* __restrict__ a0v,
                               const double* __restrict__ rk, double* __restrict__ out, int combine, const Const c) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= c.nxf || J >= c.nyf) return;
    const size_t k = (size_t)J * c.nxf + I;
    const double a0 = a0v[k];
    if (!(fabs(a0) < c.band)) {
        out[k] = phi[k];  // outside the band: unchanged (and not combined)
        return;
    }
    double dx[6], dy[6];
    face_diffs(phi, I, J, c, dx, dy);
    double dmx, dplx, dmy, dply;
    weno_pair(dx, dmx, dplx);
    weno_pair(dy, dmy, dply);
    const double gx = 0.5 * (dx[2] + dx[3]);
    const double gz = 0.5 * (dy[2] + dy[3]);
    const double dal = gx * gx + gz * gz;
    const double sg = a0 / sqrt(a0 * a0 + dal * c.hf2);
    const double ax = godunov(sg, dplx, dmx);
    const double az = godunov(sg, dply, dmy);
    const double drhs = sg * (1.0 - sqrt(ax * ax + az * az));
    const double s = phi[k] + c.redtl * drhs;
    if (combine == 1) out[k] = 0.75 * rk[k] + 0.25 * s;
    else if (combine == 2) out[k] = 1.0 / 3.0 * rk[k] + 2.0 / 3.0 * s;
    else out[k] = s;
}

}  // namespace film2d
}  // namespace lica

using namespace lica;
using namespace lica::film2d;

struct lica_film2d {
    int nx = 0, ny = 0, nlevels = 0;
    lica_film2d_props props{};
    Const c{};
    lica_mg* mg = nullptr;
    // flow-grid scratch
    double *psi = nullptr, *den = nullptr, *vis = nullptr, *densc = nullptr, *tc = nullptr, *bx = nullptr,
           *by = nullptr, *us = nullptr, *vs = nullptr, *ru = nullptr, *rv = nullptr, *rth = nullptr, *f = nullptr,
           *mdot = nullptr, *th2 = nullptr, *dp = nullptr, *cx = nullptr, *cy = nullptr;
    // refined-grid scratch (kt, cf: CAL_CUR's CURF_TMP and CURF)
    double *rphi = nullptr, *ph[3] = {nullptr, nullptr, nullptr}, *kt = nullptr, *cf = nullptr;
    // optional learned initial guess of the pressure solves, and the training-pair capture
    lica_unet* guess = nullptr;
    double* capture = nullptr;
    // optional warm start: each substep's increment kept for the same substep of the next step
    bool warm = false;
    bool have_prev[3] = {false, false, false};
    double* dp_prev[3] = {nullptr, nullptr, nullptr};
};

namespace {

int dalloc(double** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(double));
    if (e != cudaSuccess) {
        lica_set_last_error("cudaMalloc", cudaGetErrorString(e), __FILE__, __LINE__);
        return LICA_ERR_NOMEM;
    }
    return cudaMemset(*p, 0, n * sizeof(double)) == cudaSuccess ? LICA_OK : LICA_ERR_CUDA;
}

void free_all(lica_film2d* F) {
    if (F->mg) lica_mg_destroy(F->mg);
    for (double*& d : F->dp_prev) {
        cudaFree(d);
        d = nullptr;
    }
    double* ptrs[] = {F->psi, F->den, F->vis, F->densc, F->tc, F->bx, F->by, F->us, F->vs, F->ru, F->rv, F->rth, F->f,
                      F->mdot, F->th2, F->dp, F->cx, F->cy, F->rphi, F->ph[0], F->ph[1], F->ph[2], F->kt, F->cf};
    for (double* p : ptrs)
        if (p) cudaFree(p);
}

}  // namespace

extern "C" {

int lica_film2d_create(lica_film2d** out, int32_t nx, int32_t ny, const lica_film2d_props* props,
                       int32_t nlevels, int32_t precision) {
    if (!out || !props) return LICA_BAD_ARG;
    *out = nullptr;
    if (nx < 32 || ny < 32 || nx % 32 || ny % 32 || nlevels < 2 || !(props->re > 0) || !(props->prm > 0) ||
        !(props->denr > 0) || props->nreinit < 0 || (precision != 0 && precision != 1)) {
        lica_set_last_error("lica_film2d_create", "bad sizes or properties", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    lica_film2d* F = new lica_film2d();
    F->nx = nx;
    F->ny = ny;
    F->nlevels = nlevels;
    F->props = *props;
    F->c = make_const(nx, ny, *props);
    lica_mg_options o{};
    o.nlevels = nlevels;
    o.nu1 = 2;
    o.nu2 = 2;
    o.ncoarse = 2;
    o.precision = precision;
    o.use_graph = 1;
    int st = lica_mg_create(&F->mg, nx, ny, F->c.h, F->c.h, &o);
    if (st) {
        F->mg = nullptr;
        delete F;
        return st;
    }
    const size_t n = (size_t)nx * ny, nv = n + nx, nf = 4 * n;
    double** flow[] = {&F->psi, &F->den, &F->vis, &F->densc, &F->tc, &F->bx, &F->us, &F->ru, &F->rv, &F->rth,
                       &F->f, &F->mdot, &F->th2, &F->dp, &F->cx, &F->cy};
    for (double** p : flow)
        if ((st = dalloc(p, n))) break;
    if (!st) st = dalloc(&F->by, nv);
    if (!st) st = dalloc(&F->vs, nv);
    if (!st) st = dalloc(&F->rphi, nf);
    if (!st) st = dalloc(&F->kt, nf);
    if (!st) st = dalloc(&F->cf, nf);
    for (int b = 0; b < 3 && !st; ++b) st = dalloc(&F->ph[b], nf);
    if (st) {
        free_all(F);
        delete F;
        return st;
    }
    *out = F;
    return LICA_OK;
}

int lica_film2d_destroy(lica_film2d* F) {
    if (!F) return LICA_OK;
    free_all(F);
    delete F;
    return LICA_OK;
}

int lica_film2d_step_device(lica_film2d* F, double* u, double* v, double* p, double* th, double* phi, double dt,
                            lica_film2d_stats* stats, void* stream) {
    if (!F || !u || !v || !p || !th || !phi || !(dt > 0)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Const& c = F->c;
    const dim3 blk(32, 8);
    const dim3 gflow((c.nx + 31) / 32, (c.ny + 7) / 8), gref((c.nxf + 31) / 32, (c.nyf + 7) / 8);
    const size_t n = (size_t)c.nx * c.ny, nfr = 4 * n;
    double* thc = th;      // current theta
    double* thn = F->th2;  // next theta
    double* phc = phi;     // current phi
    double* phn = F->ph[0];
    int launches = 0;
    lica_film2d_stats local{};
    for (int k = 1; k <= 3; ++k) {
        const double gam = kGamma[k], ro = kRo[k], alpha = gam + ro;
        const double adt = alpha * dt, iadt = 1.0 / (alpha * dt);
        k_props<<<gflow, blk, 0, s>>>(phc, F->psi, F->den, F->vis, F->densc, F->tc, c);
        k_beta<<<gflow, blk, 0, s>>>(F->den, F->bx, F->by, c);
        k_cur_tmp<<<gref, blk, 0, s>>>(phc, F->kt, c);
        k_cur_foot<<<gref, blk, 0, s>>>(phc, F->kt, F->cf, c);
        k_face_cur<<<gflow, blk, 0, s>>>(phc, F->cf, F->psi, F->cx, F->cy, c);
        k_momentum<<<gflow, blk, 0, s>>>(u, v, F->den, F->vis, F->psi, F->cx, F->cy, p, F->bx, F->by, F->us, F->vs,
                                         F->ru, F->rv, dt, gam, ro, adt, c);
        k_source_rhs<<<gflow, blk, 0, s>>>(thc, F->psi, F->tc, F->us, F->vs, F->f, F->mdot, iadt, c);
        LICA_CUDA_TRY(cudaGetLastError());
        launches += 7;
        // the pressure increment, from the learned guess (zero if it is no better) or zero
        local.guess_rel[k - 1] = 1.0;
        if (F->guess) {
            double rel0 = 1.0;
            const int gs = lica_unet_guess_checked_device(F->guess, F->den, F->f, F->bx, F->by, c.h, c.h, F->dp,
                                                          &rel0, s);
            if (gs != LICA_OK) return gs;
            local.guess_rel[k - 1] = rel0 < 1.0 ? rel0 : 1.0;
        } else if (F->warm && F->have_prev[k - 1]) {
            LICA_CUDA_TRY(cudaMemcpyAsync(F->dp, F->dp_prev[k - 1], n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        } else {
            LICA_CUDA_TRY(cudaMemsetAsync(F->dp, 0, n * sizeof(double), s));
        }
        lica_mg_result r{};
        const int st =
            lica_mg_solve_device(F->mg, F->dp, F->f, F->bx, F->by, F->props.rtol, F->props.max_iters, &r, s);
        local.iterations[k - 1] = r.iterations;
        local.rel_residual[k - 1] = r.rel_residual;
        local.status[k - 1] = r.status;
        if (st != LICA_OK && st != LICA_NOT_CONVERGED && st != LICA_STALLED) return st;
        if (F->warm) {
            LICA_CUDA_TRY(cudaMemcpyAsync(F->dp_prev[k - 1], F->dp, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            F->have_prev[k - 1] = true;
        }
        if (F->capture) {
            double* q = F->capture + (size_t)(k - 1) * (4 * n + (size_t)(F->ny + 1) * F->nx);
            const size_t nb = (size_t)(F->ny + 1) * F->nx;
            LICA_CUDA_TRY(cudaMemcpyAsync(q, F->den, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            LICA_CUDA_TRY(cudaMemcpyAsync(q + n, F->f, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            LICA_CUDA_TRY(cudaMemcpyAsync(q + 2 * n, F->bx, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            LICA_CUDA_TRY(cudaMemcpyAsync(q + 3 * n, F->by, nb * sizeof(double), cudaMemcpyDeviceToDevice, s));
            LICA_CUDA_TRY(cudaMemcpyAsync(q + 3 * n + nb, F->dp, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
        k_correct<<<gflow, blk, 0, s>>>(F->us, F->vs, F->dp, F->bx, F->by, u, v, p, adt, c);
        k_energy<<<gflow, blk, 0, s>>>(thc, u, v, F->densc, F->tc, F->psi, thn, F->rth, dt, gam, ro, c);
        k_ls_transport<<<gref, blk, 0, s>>>(phc, u, v, phn, F->rphi, dt, gam, ro, c);
        LICA_CUDA_TRY(cudaGetLastError());
        launches += 3;
        std::swap(thc, thn);
        // phi ping-pongs between the caller's array and ph[0]
        std::swap(phc, phn);
    }
    // reinitialisation: a0 = phc (kept), three rotating buffers among {phi, ph[0], ph[1],
    // ph[2]} \ {a0}
    double* a0 = phc;
    double* pool[3];
    {
        int m = 0;
        double* all[4] = {phi, F->ph[0], F->ph[1], F->ph[2]};
        for (double* b : all)
            if (b != a0) pool[m++] = b;
    }
    double* cur = a0;
    for (int it = 0; it < F->props.nreinit; ++it) {
        double* fr[2];
        int m = 0;
        for (double* b : pool)
            if (b != cur && m < 2) fr[m++] = b;
        k_reinit_stage<<<gref, blk, 0, s>>>(cur, a0, cur, fr[0], 0, c);
        k_reinit_stage<<<gref, blk, 0, s>>>(fr[0], a0, cur, fr[1], 1, c);
        k_reinit_stage<<<gref, blk, 0, s>>>(fr[1], a0, cur, fr[0], 2, c);
        LICA_CUDA_TRY(cudaGetLastError());
        launches += 3;
        cur = fr[0];
    }
    if (cur != phi) LICA_CUDA_TRY(cudaMemcpyAsync(phi, cur, nfr * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (thc != th) LICA_CUDA_TRY(cudaMemcpyAsync(th, thc, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    lica_count_launches(launches);
    if (stats) *stats = local;
    for (int k = 0; k < 3; ++k)
        if (local.status[k] != LICA_OK) return local.status[k];
    return LICA_OK;
}

int lica_film2d_set_guess(lica_film2d* F, lica_unet* net) {
    if (!F) return LICA_BAD_ARG;
    F->guess = net;
    return LICA_OK;
}

int lica_film2d_set_warm_start(lica_film2d* F, int32_t on) {
    if (!F || (on != 0 && on != 1)) return LICA_BAD_ARG;
    const size_t n = (size_t)F->nx * F->ny;
    if (on) {
        for (double*& d : F->dp_prev)
            if (!d) {
                const int rc = dalloc(&d, n);
                if (rc != LICA_OK) return rc;
            }
    }
    F->warm = on != 0;
    for (bool& h : F->have_prev) h = false;
    return LICA_OK;
}

int lica_film2d_capture_device(lica_film2d* F, double* systems) {
    if (!F) return LICA_BAD_ARG;
    F->capture = systems;
    return LICA_OK;
}

int lica_film2d_mdot_device(lica_film2d* F, double* out, void* stream) {
    if (!F || !out) return LICA_BAD_ARG;
    LICA_CUDA_TRY(cudaMemcpyAsync(out, F->mdot, (size_t)F->nx * F->ny * sizeof(double), cudaMemcpyDeviceToDevice,
                                  (cudaStream_t)stream));
    return LICA_OK;
}

}  // extern "C"
