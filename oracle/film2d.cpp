// ORACLE (test infrastructure only) -- C++/OpenMP restatement of one RK3 step of the 2-D
// film-boiling model, statement for statement the numpy restatement in film2d.py (the readable
// specification) and so the same expressions, in the same order, as the CUDA kernels in
// lica_boiling1d_b200/csrc/film2d.cu.  Compiled without FMA contraction; every cell is computed
// independently, so the OpenMP row loops give the same bits on any thread count, and the
// pressure solves are the oracle's multigrid (orc_mg_solve, mg2d.cpp).  See film2d.py for the
// model, the reference rows it generalises and its documented simplifications.
//
// Layout (row-major, x fastest): u (ny, nx) on the face west of cell i; v (ny + 1, nx) on the
// face below cell row j; p, th (ny, nx); phi (2 ny, 2 nx).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" int orc_mg_solve(int nx, int ny, double hx, double hy, int nlevels, int nu1, int nu2, int ncoarse, int sym,
                            int method, int mixed, const double* f, const double* bx, const double* by, double* p,
                            double rtol, int max_cycles, int* cycles, double* rel, double* hist);

namespace {

const double GAMMA[4] = {0.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double RO[4] = {0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0};

using Vec = std::vector<double>;

// the constants of film2d.py's Derived
struct D2 {
    int nx, ny, nxf, nyf;
    double h, hf, ih, ih2, inv2h, ihsq, ihf, eps_h, inv2e, denm, den_diff, vism, vis_diff, denscm, densc_diff, tcm,
        tc_diff, pei, cmd, cvol, gravity, denp, surf, ih2f, ihfsq, q4, band;
    int nreinit;
    D2(int nx_, int ny_, const double* P, int nreinit_) {
        const double re = P[0], visr = P[1], denr = P[2], prm = P[3], scr = P[4], tcr = P[5], jakob = P[6], fr = P[7],
                     we = P[8];
        nx = nx_;
        ny = ny_;
        nxf = 2 * nx;
        nyf = 2 * ny;
        h = 1.0 / nx;
        hf = 0.5 * h;
        ih = 1.0 / h;
        ih2 = 2.0 / h;
        inv2h = 0.5 / h;
        ihsq = 1.0 / (h * h);
        ihf = 1.0 / hf;
        eps_h = h;
        inv2e = 1.0 / (2.0 * eps_h);
        denm = 1.0;
        den_diff = denr - 1.0;
        vism = 1.0 / re;
        vis_diff = visr / re - 1.0 / re;
        denscm = 1.0;
        densc_diff = denr * scr - 1.0;
        tcm = 1.0;
        tc_diff = tcr - 1.0;
        pei = 1.0 / (re * prm);
        cmd = jakob * pei;
        cvol = 1.0 / 1.0 - 1.0 / denr;
        gravity = (fr == 0.0) ? 0.0 : 1.0 / (fr * fr);
        denp = denr;
        surf = (we == 0.0) ? 0.0 : 1.0 / we;
        ih2f = 0.5 / hf;
        ihfsq = 1.0 / (hf * hf);
        q4 = 0.25 * ihfsq;
        nreinit = nreinit_;
        band = 8.0 * hf;
    }
};

inline int E_(int i, int n) { return i + 1 == n ? 0 : i + 1; }
inline int W_(int i, int n) { return i == 0 ? n - 1 : i - 1; }

double heaviside(double x, const D2& d) {
    const double s = (x + d.eps_h) * d.inv2e;
    const double poly = s * s * s * (10.0 + s * (-15.0 + 6.0 * s));
    return (x <= -d.eps_h) ? 0.0 : ((x >= d.eps_h) ? 1.0 : poly);
}

struct Props {
    Vec psi, den, vis, densc, tc, bx, by, cx, cy;
};

void properties(const Vec& phi, const D2& d, Props& P) {
    const int nx = d.nx, ny = d.ny, nxf = d.nxf;
    const size_t n = (size_t)nx * ny;
    P.psi.assign(n, 0.0);
    P.den.assign(n, 0.0);
    P.vis.assign(n, 0.0);
    P.densc.assign(n, 0.0);
    P.tc.assign(n, 0.0);
    P.bx.assign(n, 0.0);
    P.by.assign(n + nx, 0.0);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double* r0 = &phi[(size_t)(2 * j) * nxf];
            const double* r1 = r0 + nxf;
            const double ps = 0.25 * ((heaviside(r0[2 * i], d) + heaviside(r0[2 * i + 1], d)) +
                                      (heaviside(r1[2 * i], d) + heaviside(r1[2 * i + 1], d)));
            const size_t k = (size_t)j * nx + i;
            P.psi[k] = ps;
            P.den[k] = d.denm + d.den_diff * ps;
            P.vis[k] = d.vism + d.vis_diff * ps;
            P.densc[k] = d.denscm + d.densc_diff * ps;
            P.tc[k] = d.tcm + d.tc_diff * ps;
        }
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            P.bx[k] = 2.0 / (P.den[(size_t)j * nx + W_(i, nx)] + P.den[k]);
            P.by[k] = (j == 0) ? 1.0 / P.den[k] : 2.0 / (P.den[k - nx] + P.den[k]);
        }
    for (int i = 0; i < nx; ++i) P.by[(size_t)ny * nx + i] = 1.0 / P.den[(size_t)(ny - 1) * nx + i];
}

// CAL_CUR (two_phase.f:3317-4432) in 2-D, as film2d.py's curvature_refined,
// curvature_interface and face_curvature state it: CURF_TMP on band layers 1..N_CUR+1,
// CURF at the interface foot of layers 1..N_CUR, and per face INTER_CUR's mean over the
// interface cells of the face's box (the box twice as wide where it holds none).
constexpr int N_CUR = 4;

void curvature_refined(const Vec& phi, const D2& d, Vec& kt) {
    const int nxf = d.nxf, nyf = d.nyf;
    kt.assign((size_t)nxf * nyf, 0.0);
#pragma omp parallel for
    for (int J = 0; J < nyf; ++J)
        for (int I = 0; I < nxf; ++I) {
            const double* row = &phi[(size_t)J * nxf];
            const double* up = &phi[(size_t)std::min(J + 1, nyf - 1) * nxf];
            const double* dn = &phi[(size_t)std::max(J - 1, 0) * nxf];
            const int Ie = E_(I, nxf), Iw = W_(I, nxf);
            const double C = row[I], E = row[Ie], W = row[Iw], N = up[I], S = dn[I];
            if (!(std::fabs(C) < (N_CUR + 1) * d.hf)) continue;
            const double gx = 0.5 * (E - W) * d.ihf;
            const double gz = 0.5 * (N - S) * d.ihf;
            const double gxx = ((E - 2.0 * C) + W) * d.ihf * d.ihf;
            const double gzz = ((N - 2.0 * C) + S) * d.ihf * d.ihf;
            const double gxz = 0.25 * ((up[Ie] - up[Iw]) - (dn[Ie] - dn[Iw])) * d.ihf * d.ihf;
            const double g2 = gx * gx + gz * gz;
            if (!(g2 > 0.0)) continue;
            const double num = (gxx * (gz * gz) + gzz * (gx * gx)) - 2.0 * (gxz * gx * gz);
            kt[(size_t)J * nxf + I] = -num / (g2 * std::sqrt(g2));
        }
}

void curvature_interface(const Vec& phi, const Vec& kt, const D2& d, Vec& cf) {
    const int nxf = d.nxf, nyf = d.nyf;
    cf.assign((size_t)nxf * nyf, 0.0);
#pragma omp parallel for
    for (int J = 0; J < nyf; ++J)
        for (int I = 0; I < nxf; ++I) {
            const int Jn = std::min(J + 1, nyf - 1), Js = std::max(J - 1, 0);
            const int Ie = E_(I, nxf), Iw = W_(I, nxf);
            const double C = phi[(size_t)J * nxf + I];
            if (!(std::fabs(C) < N_CUR * d.hf)) continue;
            const double dpx = 0.5 * (phi[(size_t)J * nxf + Ie] - phi[(size_t)J * nxf + Iw]) * d.ihf;
            const double dpz = 0.5 * (phi[(size_t)Jn * nxf + I] - phi[(size_t)Js * nxf + I]) * d.ihf;
            const double g2 = dpx * dpx + dpz * dpz;
            if (!(g2 > 0.0)) continue;
            const double amdpi = 1.0 / std::sqrt(g2);
            const double dis = C * amdpi;
            const double xp = (I + 0.5) * d.hf, zp = (J + 0.5) * d.hf;
            const double xb = xp - dis * (dpx * amdpi), zb = zp - dis * (dpz * amdpi);
            int i1, i2, j1, j2;
            double xd, zd;
            if (xb >= xp) {
                xd = (xb - xp) * d.ihf;
                i1 = I;
                i2 = Ie;
            } else {
                xd = (xb - (xp - d.hf)) * d.ihf;
                i1 = Iw;
                i2 = I;
            }
            if (zb >= zp) {
                zd = (zb - zp) * d.ihf;
                j1 = J;
                j2 = Jn;
            } else {
                zd = (zb - (zp - d.hf)) * d.ihf;
                j1 = Js;
                j2 = J;
            }
            const double c00 = kt[(size_t)j1 * nxf + i1] * (1.0 - xd) + kt[(size_t)j1 * nxf + i2] * xd;
            const double c01 = kt[(size_t)j2 * nxf + i1] * (1.0 - xd) + kt[(size_t)j2 * nxf + i2] * xd;
            cf[(size_t)J * nxf + I] = c00 * (1.0 - zd) + c01 * zd;
        }
}

// INTER_CUR over refined columns c0..c0+nc-1 (x periodic) and rows r0..r0+nr-1, column by
// column: the mean of CURF over the cells cut by the interface (0 < psi_f < 1, CURF /= 0).
static bool inter_cur(const Vec& phi, const Vec& cf, int c0, int nc, int r0, int nr, const D2& d, double& cur) {
    const int nxf = d.nxf;
    double sum = 0.0, volf = 0.0;
    for (int a = 0; a < nc; ++a) {
        const int II = ((c0 + a) % nxf + nxf) % nxf;
        for (int b = 0; b < nr; ++b) {
            const size_t q = (size_t)(r0 + b) * nxf + II;
            const double hh = heaviside(phi[q], d);
            if (hh > 0.0 && hh < 1.0 && cf[q] != 0.0) {
                sum = sum + cf[q];
                volf = volf + 1.0;
            }
        }
    }
    if (volf != 0.0) cur = sum / volf;
    return volf != 0.0;
}

void face_curvature(const Vec& phi, const Vec& cf, const D2& d, Props& P) {
    const int nx = d.nx, ny = d.ny;
    P.cx.assign((size_t)nx * ny, 0.0);
    P.cy.assign((size_t)nx * ny, 0.0);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            if ((P.psi[k] - P.psi[(size_t)j * nx + W_(i, nx)]) != 0.0) {
                double cur = 0.0;
                if (!inter_cur(phi, cf, 2 * i - 1, 2, 2 * j, 2, d, cur)) inter_cur(phi, cf, 2 * i - 2, 4, 2 * j, 2, d, cur);
                P.cx[k] = cur;
            }
            if (j >= 1 && (P.psi[k] - P.psi[k - nx]) != 0.0) {
                double cur = 0.0;
                if (!inter_cur(phi, cf, 2 * i, 2, 2 * j - 1, 2, d, cur)) inter_cur(phi, cf, 2 * i, 2, 2 * j - 2, 4, d, cur);
                P.cy[k] = cur;
            }
        }
}

void curvature(const Vec& phi, const D2& d, Props& P) {
    Vec kt, cf;
    curvature_refined(phi, d, kt);
    curvature_interface(phi, kt, d, cf);
    face_curvature(phi, cf, d, P);
}

// volume source S and mdot (mass_source)
void mass_source(const Vec& th, const Props& P, const D2& d, Vec& S, Vec& md) {
    const int nx = d.nx, ny = d.ny;
    S.assign((size_t)nx * ny, 0.0);
    md.assign((size_t)nx * ny, 0.0);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            const int ie = E_(i, nx), iw = W_(i, nx);
            const double ts = (j > 0) ? th[k - nx] : 2.0 - th[i];
            const double tn = (j + 1 < ny) ? th[k + nx] : th[k];
            const double ps = (j > 0) ? P.psi[k - nx] : P.psi[i];
            const double pn = (j + 1 < ny) ? P.psi[k + nx] : P.psi[k];
            const double gtx = (th[(size_t)j * nx + ie] - th[(size_t)j * nx + iw]) * d.inv2h;
            const double gty = (tn - ts) * d.inv2h;
            const double gpx = (P.psi[(size_t)j * nx + ie] - P.psi[(size_t)j * nx + iw]) * d.inv2h;
            const double gpy = (pn - ps) * d.inv2h;
            const double q = -(gtx * gpx + gty * gpy);
            const double m = (d.cmd * P.tc[k]) * std::max(q, 0.0);
            md[k] = m;
            S[k] = m * d.cvol;
        }
}

// momentum right-hand sides: nu on the u faces, nv on the v faces 1..ny (ny rows)
void momentum(const Vec& u, const Vec& v, const Props& P, const D2& d, Vec& nu, Vec& nv) {
    const int nx = d.nx, ny = d.ny;
    const double ih = d.ih;
    nu.assign((size_t)nx * ny, 0.0);
    nv.assign((size_t)nx * ny, 0.0);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            const int ie = E_(i, nx), iw = W_(i, nx);
            const size_t kw = (size_t)j * nx + iw, ke = (size_t)j * nx + ie;
            const size_t rn = (j + 1 < ny) ? (size_t)(j + 1) * nx : (size_t)(ny - 1) * nx;  // row j + 1 (top: copy)
            const size_t rs = (j > 0) ? (size_t)(j - 1) * nx : 0;                         // row j - 1 (bottom: row 0)
            const size_t vrow = (size_t)j * nx, vrn = (size_t)(j + 1) * nx;
            {
                const double uc = u[k], ue = u[ke], uw = u[kw];
                const double un = u[rn + i];
                const double us = (j > 0) ? u[rs + i] : -u[i];
                const double vn = 0.5 * (v[vrn + iw] + v[vrn + i]);
                const double vs = 0.5 * (v[vrow + iw] + v[vrow + i]);
                const double uci = 0.5 * (uc + ue);
                const double ucm = 0.5 * (uw + uc);
                const double conv = (uci * uci - ucm * ucm) * ih + (0.5 * (uc + un) * vn - 0.5 * (us + uc) * vs) * ih;
                const double mc = P.vis[k], mw = P.vis[kw];
                const double txe = 2.0 * mc * (ue - uc) * ih;
                const double txw = 2.0 * mw * (uc - uw) * ih;
                const double mun = 0.25 * ((mw + mc) + (P.vis[rn + iw] + P.vis[rn + i]));
                const double mus = 0.25 * ((P.vis[rs + iw] + P.vis[rs + i]) + (mw + mc));
                const double tyn = mun * ((un - uc) * ih + (v[vrn + i] - v[vrn + iw]) * ih);
                const double tys = mus * ((uc - us) * ih + (v[vrow + i] - v[vrow + iw]) * ih);
                const double rho = 0.5 * (P.den[kw] + P.den[k]);
                const double visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho;
                nu[k] = visc - conv + (d.surf * P.cx[k]) * ((P.psi[k] - P.psi[kw]) * ih) / rho;
            }
            {
                // face j + 1
                const size_t vc_r = vrn, vs_r = vrow;
                const size_t vn_r = (j + 1 < ny) ? (size_t)(j + 2) * nx : vrn;
                const double vc = v[vc_r + i], vsv = v[vs_r + i], vnv = v[vn_r + i];
                const double ve = v[vc_r + ie], vw = v[vc_r + iw];
                const double ulo = u[k], uhi = u[rn + i], ulo_e = u[ke], uhi_e = u[rn + ie];
                const double vcj = 0.5 * (vc + vnv);
                const double vcm = 0.5 * (vsv + vc);
                const double conv =
                    ((0.5 * (ulo_e + uhi_e)) * (0.5 * (vc + ve)) - (0.5 * (ulo + uhi)) * (0.5 * (vw + vc))) * ih +
                    (vcj * vcj - vcm * vcm) * ih;
                const double mulo = P.vis[k], muhi = P.vis[rn + i];
                const double tyn = 2.0 * muhi * (vnv - vc) * ih;
                const double tys = 2.0 * mulo * (vc - vsv) * ih;
                const double mue = 0.25 * ((mulo + P.vis[ke]) + (muhi + P.vis[rn + ie]));
                const double muw = 0.25 * ((P.vis[kw] + mulo) + (P.vis[rn + iw] + muhi));
                const double txe = mue * ((ve - vc) * ih + (uhi_e - ulo_e) * ih);
                const double txw = muw * ((vc - vw) * ih + (uhi - ulo) * ih);
                const double dlo = P.den[k], dhi = P.den[rn + i];
                const double rho = 0.5 * (dlo + dhi);
                const double visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho;
                const double cf = (j + 1 < ny) ? P.cy[k + nx] : 0.0;   // the face above row j
                nv[k] = visc - conv + d.gravity * (d.denp / rho - 1.0) +
                        (d.surf * cf) * ((P.psi[rn + i] - P.psi[k]) * ih) / rho;
            }
        }
}

void energy_rhs(const Vec& th, const Vec& u, const Vec& v, const Props& P, const D2& d, Vec& e) {
    const int nx = d.nx, ny = d.ny;
    e.assign((size_t)nx * ny, 0.0);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            const int ie = E_(i, nx), iw = W_(i, nx);
            const double t = th[k];
            const double te = th[(size_t)j * nx + ie], tw = th[(size_t)j * nx + iw];
            const double tn = (j + 1 < ny) ? th[k + nx] : t;
            const double ts = (j > 0) ? th[k - nx] : 2.0 - th[i];
            const double uc = 0.5 * (u[k] + u[(size_t)j * nx + ie]);
            const double vc = 0.5 * (v[k] + v[k + nx]);
            const double adv = uc * ((te - tw) * d.inv2h) + vc * ((tn - ts) * d.inv2h);
            const double kc = P.tc[k];
            const double ke = 0.5 * (kc + P.tc[(size_t)j * nx + ie]);
            const double kw = 0.5 * (P.tc[(size_t)j * nx + iw] + kc);
            const double kn = 0.5 * (kc + ((j + 1 < ny) ? P.tc[k + nx] : kc));
            const double ks = 0.5 * (((j > 0) ? P.tc[k - nx] : P.tc[i]) + kc);
            const double dif = ((ke * (te - t) - kw * (t - tw)) + (kn * (tn - t) - ks * (t - ts))) * d.ihsq;
            e[k] = (d.pei * dif) / P.densc[k] - adv;
        }
}

double hjweno(double a, double b, double cc, double dd) {
    const double eps = 1e-6;
    const double s1 = 13.0 * (a - b) * (a - b) + 3.0 * (a - 3.0 * b) * (a - 3.0 * b);
    const double s2 = 13.0 * (b - cc) * (b - cc) + 3.0 * (b + cc) * (b + cc);
    const double s3 = 13.0 * (cc - dd) * (cc - dd) + 3.0 * (3.0 * cc - dd) * (3.0 * cc - dd);
    const double a1 = 1.0 / ((eps + s1) * (eps + s1));
    const double a2 = 6.0 / ((eps + s2) * (eps + s2));
    const double a3 = 3.0 / ((eps + s3) * (eps + s3));
    const double w1 = a1 / (a1 + a2 + a3);
    const double w3 = a3 / (a1 + a2 + a3);
    return (1.0 / 3.0) * w1 * (a - 2.0 * b + cc) + (1.0 / 6.0) * (w3 - 0.5) * (b - 2.0 * cc + dd);
}

// one-sided WENO5 derivatives from the six face differences dp(c-3 .. c+2)
void weno_pair(const double* q, double& dm, double& dpl) {
    const double v1 = q[0], v2 = q[1], v3 = q[2], v4 = q[3], v5 = q[4];
    dm = (1.0 / 12.0) * (-v2 + 7.0 * v3 + 7.0 * v4 - v5) - hjweno(v2 - v1, v3 - v2, v4 - v3, v5 - v4);
    const double q1 = q[5], q2 = q[4], q3 = q[3], q4 = q[2], q5 = q[1];
    dpl = (1.0 / 12.0) * (-q5 + 7.0 * q4 + 7.0 * q3 - q2) + hjweno(q1 - q2, q2 - q3, q3 - q4, q4 - q5);
}

void face_diffs(const Vec& phi, int I, int J, const D2& d, double* dx, double* dy) {
    const int nxf = d.nxf, nyf = d.nyf;
    const double* row = &phi[(size_t)J * nxf];
    for (int m = 0; m < 6; ++m) {
        int x0 = I - 3 + m, x1 = x0 + 1;
        x0 = (x0 % nxf + nxf) % nxf;
        x1 = (x1 % nxf + nxf) % nxf;
        dx[m] = (row[x1] - row[x0]) * d.ihf;
        int y = std::min(std::max(J - 3 + m, 0), nyf - 2);
        dy[m] = (phi[(size_t)(y + 1) * nxf + I] - phi[(size_t)y * nxf + I]) * d.ihf;
    }
}

void refined_velocity(const Vec& u, const Vec& v, const D2& d, int I, int J, double& uf, double& vf) {
    const int nx = d.nx, ny = d.ny;
    const int m = I >> 1, a = I & 1, jp = J >> 1, b = J & 1;
    auto U = [&](int r, int c) {
        if (r < 0) return -u[c];
        if (r >= ny) return u[(size_t)(ny - 1) * nx + c];
        return u[(size_t)r * nx + c];
    };
    {
        const int r0 = jp - 1 + b, r1 = r0 + 1, c0 = m, c1 = (m + 1) % nx;
        const double wx = a == 0 ? 0.25 : 0.75, wy = b == 0 ? 0.75 : 0.25;
        uf = (1.0 - wy) * ((1.0 - wx) * U(r0, c0) + wx * U(r0, c1)) + wy * ((1.0 - wx) * U(r1, c0) + wx * U(r1, c1));
    }
    {
        const int c0 = ((m - 1 + a) % nx + nx) % nx, c1 = (m + a) % nx;
        const double wx = a == 0 ? 0.75 : 0.25, wy = b == 0 ? 0.25 : 0.75;
        const double* r0 = &v[(size_t)jp * nx];
        const double* r1 = r0 + nx;
        vf = (1.0 - wy) * ((1.0 - wx) * r0[c0] + wx * r0[c1]) + wy * ((1.0 - wx) * r1[c0] + wx * r1[c1]);
    }
}

double godunov(double sg, double ap, double am) {
    const double aplus = sg * ap, aminus = sg * am;
    if (aplus >= 0.0 && aminus >= 0.0) return am;
    if (aplus <= 0.0 && aminus <= 0.0) return ap;
    if (aplus > 0.0 && aminus < 0.0) return 0.0;
    if (aplus + aminus > 0.0) return am;
    return ap;
}

// one reinitialisation stage on the band |a0| < band; cells outside keep phi
void reinit_stage(const Vec& phi, const Vec& a0, const D2& d, Vec& out) {
    const int nxf = d.nxf, nyf = d.nyf;
    out.resize(phi.size());
#pragma omp parallel for
    for (int J = 0; J < nyf; ++J)
        for (int I = 0; I < nxf; ++I) {
            const size_t k = (size_t)J * nxf + I;
            double dx[6], dy[6], dmx, dplx, dmy, dply;
            face_diffs(phi, I, J, d, dx, dy);
            weno_pair(dx, dmx, dplx);
            weno_pair(dy, dmy, dply);
            const double gx = 0.5 * (dx[2] + dx[3]);
            const double gz = 0.5 * (dy[2] + dy[3]);
            const double dal = gx * gx + gz * gz;
            const double sg = a0[k] / std::sqrt(a0[k] * a0[k] + dal * (d.hf * d.hf));
            const double ax = godunov(sg, dplx, dmx);
            const double az = godunov(sg, dply, dmy);
            const double drhs = sg * (1.0 - std::sqrt(ax * ax + az * az));
            out[k] = (std::fabs(a0[k]) < d.band) ? phi[k] + (0.5 * d.hf) * drhs : phi[k];
        }
}

}  // namespace

extern "C" {

// One RK3 step of film2d.py's step() in place on u, v, p, th, phi.  props = [re, visr, denr,
// prm, scr, tcr, jakob, fr, we].  iters / rels / stats: the three pressure solves.  S_out and
// md_out (ny x nx, may be null): the last substep's volume source and mass flux.  Returns the
// first non-zero solve status, or 0.
int orc_film2d_step(int nx, int ny, const double* props, double rtol, int nreinit, int nlevels, double dt, double* u,
                    double* v, double* p, double* th, double* phi, int* iters, double* rels, int* stats, double* S_out,
                    double* md_out) {
    if (nx < 8 || ny < 8 || !props || !u || !v || !p || !th || !phi) return 4;
    const D2 d(nx, ny, props, nreinit);
    const size_t n = (size_t)nx * ny, nv = n + nx, nfr = 4 * n;
    Vec U(u, u + n), V(v, v + nv), Pp(p, p + n), T(th, th + n), PH(phi, phi + nfr);
    Vec ru(n, 0.0), rv(n, 0.0), rth(n, 0.0), rphi(nfr, 0.0);
    Props P;
    Vec S, md, nu, nvv, e, f(n), dp(n), us(n), vs(nv), hist(201);
    int worst = 0;
    for (int k = 1; k <= 3; ++k) {
        const double gam = GAMMA[k], ro = RO[k], alpha = gam + ro;
        const double adt = alpha * dt, iadt = 1.0 / (alpha * dt);
        properties(PH, d, P);
        mass_source(T, P, d, S, md);
        curvature(PH, d, P);
        momentum(U, V, P, d, nu, nvv);
#pragma omp parallel for
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t q = (size_t)j * nx + i;
                us[q] = U[q] + dt * (gam * nu[q] + ro * ru[q]) -
                        adt * (P.bx[q] * ((Pp[q] - Pp[(size_t)j * nx + W_(i, nx)]) * d.ih));
                const size_t qf = q + nx;  // face j + 1
                const double gp = (j + 1 < ny) ? (Pp[qf] - Pp[q]) * d.ih : (0.0 - Pp[q]) * d.ih2;
                vs[qf] = V[qf] + dt * (gam * nvv[q] + ro * rv[q]) - adt * (P.by[qf] * gp);
            }
        for (int i = 0; i < nx; ++i) vs[i] = 0.0;
        ru = nu;
        rv = nvv;
#pragma omp parallel for
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t q = (size_t)j * nx + i;
                f[q] = ((us[(size_t)j * nx + E_(i, nx)] - us[q]) * d.ih + (vs[q + nx] - vs[q]) * d.ih - S[q]) * iadt;
            }
        std::fill(dp.begin(), dp.end(), 0.0);
        int cyc = 0;
        double rel = 0.0;
        // V(2,2), 2 coarse cycles, flags 5 = symmetric smoothing + piecewise-constant
        // prolongation (the GPU multigrid's cycle), PCG
        const int st = orc_mg_solve(nx, ny, d.h, d.h, nlevels, 2, 2, 2, 5, 2, 0, f.data(), P.bx.data(), P.by.data(),
                                    dp.data(), rtol, 200, &cyc, &rel, hist.data());
        if (iters) iters[k - 1] = cyc;
        if (rels) rels[k - 1] = rel;
        if (stats) stats[k - 1] = st;
        if (st && !worst) worst = st;
#pragma omp parallel for
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t q = (size_t)j * nx + i;
                U[q] = us[q] - adt * (P.bx[q] * ((dp[q] - dp[(size_t)j * nx + W_(i, nx)]) * d.ih));
                if (j > 0) V[q] = vs[q] - adt * (P.by[q] * ((dp[q] - dp[q - nx]) * d.ih));
                else V[q] = vs[q];
            }
        for (int i = 0; i < nx; ++i) {
            const size_t t = (size_t)ny * nx + i;
            V[t] = vs[t] - adt * (P.by[t] * ((0.0 - dp[(size_t)(ny - 1) * nx + i]) * d.ih2));
        }
        for (size_t q = 0; q < n; ++q) Pp[q] = Pp[q] + dp[q];
        energy_rhs(T, U, V, P, d, e);
#pragma omp parallel for
        for (int q = 0; q < (int)n; ++q) {
            const double thn = T[q] + dt * (gam * e[q] + ro * rth[q]);
            T[q] = (P.psi[q] > 0.5) ? 0.0 : thn;
        }
        rth = e;
        // level-set transport on the band |phi| < band
        Vec L(nfr, 0.0), PHn(nfr);
#pragma omp parallel for
        for (int J = 0; J < d.nyf; ++J)
            for (int I = 0; I < d.nxf; ++I) {
                const size_t q = (size_t)J * d.nxf + I;
                if (!(std::fabs(PH[q]) < d.band)) {
                    PHn[q] = PH[q];
                    continue;
                }
                double uf, vf, dx[6], dy[6], dmx, dplx, dmy, dply;
                refined_velocity(U, V, d, I, J, uf, vf);
                face_diffs(PH, I, J, d, dx, dy);
                weno_pair(dx, dmx, dplx);
                weno_pair(dy, dmy, dply);
                const double px = (uf >= 0.0) ? dmx : dplx;
                const double py = (vf >= 0.0) ? dmy : dply;
                L[q] = -(uf * px + vf * py);
                PHn[q] = PH[q] + dt * (gam * L[q] + ro * rphi[q]);
            }
        PH.swap(PHn);
        rphi.swap(L);
        if (k == 3) {
            if (S_out) std::memcpy(S_out, S.data(), n * sizeof(double));
            if (md_out) std::memcpy(md_out, md.data(), n * sizeof(double));
        }
    }
    // reinitialisation (band |a0| < band)
    {
        const Vec a0 = PH;
        Vec s1, s2;
        for (int it = 0; it < d.nreinit; ++it) {
            const Vec rk = PH;
            reinit_stage(PH, a0, d, s1);
            reinit_stage(s1, a0, d, s2);
            for (size_t q = 0; q < nfr; ++q)
                PH[q] = (std::fabs(a0[q]) < d.band) ? 0.75 * rk[q] + 0.25 * s2[q] : s2[q];
            reinit_stage(PH, a0, d, s1);
            for (size_t q = 0; q < nfr; ++q)
                PH[q] = (std::fabs(a0[q]) < d.band) ? (1.0 / 3.0) * rk[q] + (2.0 / 3.0) * s1[q] : s1[q];
        }
    }
    std::memcpy(u, U.data(), n * sizeof(double));
    std::memcpy(v, V.data(), nv * sizeof(double));
    std::memcpy(p, Pp.data(), n * sizeof(double));
    std::memcpy(th, T.data(), n * sizeof(double));
    std::memcpy(phi, PH.data(), nfr * sizeof(double));
    return worst;
}

}  // extern "C"
