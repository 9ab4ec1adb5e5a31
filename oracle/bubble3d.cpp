// ORACLE (test infrastructure only) -- C++ restatement of BUBBLE_TRACKING (two_phase.f:
// 6321-6555), BUBBLE_EIGENV (6558-6705) and Jacobi_bub (two_phase.f:19-97): per level set,
// the gas volume, volume-weighted centroid and velocity over the cells with PSI_TMP != 1,
// then, in a second sweep, the second moment of the gas volume about that centroid, its
// eigenvalues and eigenvectors by cyclic Jacobi rotations, the aspect ratio and the two
// angles of the smallest eigenvalue's axis.  Loops in the reference's order (K, J, I), one
// thread, so the sums are the reference's sums in a fixed order.  Compiled without FMA
// contraction.
//
// Layout: fields (0:N1, 0:N2, 0:N3) column-major, (i, j, k) at i + (n1m+2)(j + (n2m+2)k);
// sdx, xp n1m+2 entries (index = Fortran index), likewise y and z.  The record has the
// layout of lica_bub_record.
#include <cmath>
#include <cstdint>

namespace {

struct Record {
    double time;
    int64_t llvs;
    double col[9];
    double vel[3];
    double vol;
    double ami[3];
    int64_t iz_periodic;
};

// Jacobi_bub: a[r][c] = A(r+1, c+1); x receives the eigenvectors as columns.
void jacobi(double a[3][3], double x[3][3], double abserr) {
    const int n = 3;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) x[i][j] = (i == j) ? 1.0 : 0.0;
    double b2 = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) b2 = b2 + a[i][j] * a[i][j];
    if (b2 <= abserr) return;
    double bar = 0.5 * b2 / double(n * n);
    for (int iter = 1; iter <= 500; ++iter) {
        for (int i = 0; i < n - 1; ++i) {
            for (int j = i + 1; j < n; ++j) {
                if (a[j][i] * a[j][i] <= bar) continue;
                b2 = b2 - 2.0 * a[j][i] * a[j][i];
                bar = 0.5 * b2 / double(n * n);
                double beta = (a[j][j] - a[i][i]) / (2.0 * a[j][i]);
                double coeff = 0.5 * beta / std::sqrt(1.0 + beta * beta);
                double s = std::sqrt(std::fmax(0.5 + coeff, 0.0));
                double c = std::sqrt(std::fmax(0.5 - coeff, 0.0));
                for (int k = 0; k < n; ++k) {
                    double cs = c * a[i][k] + s * a[j][k];
                    double sc = -s * a[i][k] + c * a[j][k];
                    a[i][k] = cs;
                    a[j][k] = sc;
                }
                for (int k = 0; k < n; ++k) {
                    double cs = c * a[k][i] + s * a[k][j];
                    double sc = -s * a[k][i] + c * a[k][j];
                    a[k][i] = cs;
                    a[k][j] = sc;
                    cs = c * x[k][i] + s * x[k][j];
                    sc = -s * x[k][i] + c * x[k][j];
                    x[k][i] = cs;
                    x[k][j] = sc;
                }
            }
        }
        if (b2 <= abserr) return;
    }
}

struct Grid {
    int n1m, n2m, n3m, ipx, ipy, ipz;
    double zl;
    const double *sdx, *sdy, *sdz, *xp, *yp, *zp;
    long long idx(int i, int j, int k) const { return i + (long long)(n1m + 2) * (j + (long long)(n2m + 2) * k); }
    int ipv(int i) const { return (i == n1m) ? (ipx ? 1 : n1m + 1) : i + 1; }
    int jpv(int j) const { return (j == n2m) ? (ipy ? 1 : n2m + 1) : j + 1; }
    int kpv(int k) const { return (k == n3m) ? (ipz ? 1 : n3m + 1) : k + 1; }
};

void tracking(const Grid& g, const double* psi, const double* u, const double* v, const double* w, double time,
              int llvs, int icacy, Record* out) {
    const double pi = std::acos(-1.0);
    int iz_periodic = 0;
    for (int j = 1; j <= g.n2m; ++j)
        for (int i = 1; i <= g.n1m; ++i)
            if (psi[g.idx(i, j, g.n3m)] != 1.0) iz_periodic = 1;
    const bool shift = g.ipz == 1 && iz_periodic == 1;
    double xx = 0.0, yy = 0.0, zz = 0.0, uu = 0.0, vv = 0.0, ww = 0.0, vol = 0.0;
    for (int k = 1; k <= g.n3m; ++k)
        for (int j = 1; j <= g.n2m; ++j)
            for (int i = 1; i <= g.n1m; ++i) {
                const long long c = g.idx(i, j, k);
                if (psi[c] == 1.0) continue;
                const double volf = (1.0 - psi[c]) * g.sdx[i] * g.sdy[j] * g.sdz[k];
                xx = xx + g.xp[i] * volf;
                yy = yy + g.yp[j] * volf;
                if (shift && g.zp[k] <= 0.5 * g.zl)
                    zz = zz + (g.zp[k] + g.zl) * volf;
                else
                    zz = zz + g.zp[k] * volf;
                uu = uu + 0.5 * (u[c] + u[g.idx(g.ipv(i), j, k)]) * volf;
                vv = vv + 0.5 * (v[c] + v[g.idx(i, g.jpv(j), k)]) * volf;
                ww = ww + 0.5 * (w[c] + w[g.idx(i, j, g.kpv(k))]) * volf;
                vol = vol + volf;
            }
    if (vol != 0.0) {
        const double voli = 1.0 / vol;
        xx = xx * voli;
        yy = yy * voli;
        zz = zz * voli;
        uu = uu * voli;
        vv = vv * voli;
        ww = ww * voli;
    }
    Record r;
    r.time = time;
    r.llvs = llvs;
    double xc, yc, zc;
    if (icacy == 2) {
        const double rr = std::sqrt(xx * xx + yy * yy);
        double tt = std::atan(yy / xx);
        if (xx <= 0.0 && yy >= 0.0)
            tt = tt + pi;
        else if (xx <= 0.0 && yy <= 0.0)
            tt = tt + pi;
        else if (xx >= 0.0 && yy <= 0.0)
            tt = tt + 2.0 * pi;
        const double ur = uu * std::cos(tt) + vv * std::sin(tt);
        const double ut = -uu * std::sin(tt) + vv * std::cos(tt);
        xc = rr * std::cos(tt);
        yc = rr * std::sin(tt);
        zc = zz;
        r.col[0] = rr;
        r.col[1] = tt;
        r.col[2] = zz;
        r.col[3] = ur;
        r.col[4] = ut;
    } else {
        xc = xx;
        yc = yy;
        zc = zz;
        r.col[0] = xx;
        r.col[1] = yy;
        r.col[2] = zz;
        r.col[3] = uu;
        r.col[4] = vv;
    }
    r.col[5] = ww;
    // BUBBLE_EIGENV: second moment about (xc, yc, zc)
    double axx = 0.0, ayy = 0.0, azz = 0.0, axy = 0.0, ayz = 0.0, azx = 0.0;
    for (int k = 1; k <= g.n3m; ++k)
        for (int j = 1; j <= g.n2m; ++j)
            for (int i = 1; i <= g.n1m; ++i) {
                const long long c = g.idx(i, j, k);
                if (psi[c] == 1.0) continue;
                const double volf = (1.0 - psi[c]) * g.sdx[i] * g.sdy[j] * g.sdz[k];
                const double dx = g.xp[i] - xc;
                const double dy = g.yp[j] - yc;
                const double dz = (shift && g.zp[k] <= 0.5 * g.zl) ? (g.zp[k] + g.zl) - zc : g.zp[k] - zc;
                axx = axx + dx * dx * volf;
                ayy = ayy + dy * dy * volf;
                azz = azz + dz * dz * volf;
                axy = axy + dx * dy * volf;
                ayz = ayz + dy * dz * volf;
                azx = azx + dz * dx * volf;
            }
    // the reference leaves AMI unset for VOL = 0; zero here
    double a[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    if (vol != 0.0) {
        const double voli = 1.0 / vol;
        a[0][0] = axx * voli;
        a[1][1] = ayy * voli;
        a[2][2] = azz * voli;
        a[0][1] = axy * voli;
        a[1][2] = ayz * voli;
        a[2][0] = azx * voli;
    }
    a[1][0] = a[0][1];
    a[2][1] = a[1][2];
    a[0][2] = a[2][0];
    double e[3][3];
    jacobi(a, e, 1.0e-12);
    double ar;
    int ismall;
    if (a[0][0] >= a[1][1]) {
        if (a[0][0] >= a[2][2]) {
            if (a[1][1] >= a[2][2]) {
                ar = std::sqrt(a[0][0] / a[2][2]);
                ismall = 3;
            } else {
                ar = std::sqrt(a[0][0] / a[1][1]);
                ismall = 2;
            }
        } else {
            ar = std::sqrt(a[2][2] / a[1][1]);
            ismall = 2;
        }
    } else {
        if (a[1][1] >= a[2][2]) {
            if (a[0][0] >= a[2][2]) {
                ar = std::sqrt(a[1][1] / a[2][2]);
                ismall = 3;
            } else {
                ar = std::sqrt(a[1][1] / a[0][0]);
                ismall = 1;
            }
        } else {
            ar = std::sqrt(a[2][2] / a[0][0]);
            ismall = 1;
        }
    }
    const int s = ismall - 1;
    const double denom = 1.0 / std::sqrt(e[0][s] * e[0][s] + e[1][s] * e[1][s] + e[2][s] * e[2][s]);
    double ang1 = std::acos(e[0][s] * denom) * 57.295779513082321;
    double ang2 = std::acos(e[2][s] * denom) * 57.295779513082321;
    if (ang1 >= 90.0) ang1 = 180.0 - ang1;
    if (ang2 >= 90.0) ang2 = 180.0 - ang2;
    r.col[6] = ar;
    r.col[7] = ang1;
    r.col[8] = ang2;
    r.vel[0] = uu;
    r.vel[1] = vv;
    r.vel[2] = ww;
    r.vol = vol;
    r.ami[0] = a[0][0];
    r.ami[1] = a[1][1];
    r.ami[2] = a[2][2];
    r.iz_periodic = iz_periodic;
    *out = r;
}

}  // namespace

extern "C" {

void orc_jacobi3(double* a9, double* x9, double abserr) {
    double a[3][3], x[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) a[r][c] = a9[3 * r + c];
    jacobi(a, x, abserr);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            a9[3 * r + c] = a[r][c];
            x9[3 * r + c] = x[r][c];
        }
}

void orc_bubble_tracking(int n1m, int n2m, int n3m, int ipx, int ipy, int ipz, double zl, const double* sdx,
                         const double* sdy, const double* sdz, const double* xp, const double* yp, const double* zp,
                         int nlvs, int llvs0, const double* psi, const double* u, const double* v, const double* w,
                         double time, int icacy, void* out) {
    const Grid g{n1m, n2m, n3m, ipx != 0, ipy != 0, ipz != 0, zl, sdx, sdy, sdz, xp, yp, zp};
    const long long fsize = (long long)(n1m + 2) * (n2m + 2) * (n3m + 2);
    Record* rec = static_cast<Record*>(out);
    for (int l = 0; l < nlvs; ++l) tracking(g, psi + l * fsize, u, v, w, time, llvs0 + l, icacy, rec + l);
}

}  // extern "C"
