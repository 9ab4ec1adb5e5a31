/* A compiled host driving the GPU entry points through include/lica_gpu.h alone, with host
 * arrays in the reference's layouts, as a Fortran or C solver would:
 *   - POISSON (lica_gpu_poisson) on a 1-D column with a variable 1/rho: the right-hand side
 *     is the operator applied to a known pressure, which must come back;
 *   - the 2-D multigrid (lica_mg_create / lica_mg_solve_host) on a bubble-like coefficient
 *     field: the residual the host computes from the header's operator must meet 1e-10;
 *   - whole RK3 steps of a column (lica_gpu_column_init / lica_gpu_column_steps), then the
 *     per-routine drop-ins REINITIALIZATION and GRID_COUPLING on the stepped state;
 *   - BUBBLE_TRACKING (lica_gpu_bubble_tracking) of a 3 x 2 x 4-cell gas block with uniform
 *     velocity in an 8^3 box: volume, centroid, velocity, second moments (n^2 - 1) h^2 / 12
 *     per axis, aspect ratio sqrt(5) and the smallest axis along y.
 * Usage: host_gpu.  Prints "ok" and exits 0, or names the failed check. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lica_gpu.h"

static int fail(const char* what) {
    fprintf(stderr, "FAILED: %s (%s)\n", what, lica_last_error());
    return 1;
}

/* ---- POISSON: P(0:M1,0:M2,0:M3), DIVGSUM(M1M,M2M,M3M), M1 = M2 = 2, M3 = N3M + 1 */
#define N3M 48
#define M3 (N3M + 1)
#define PIDX(k) (((k) * 3 + 1) * 3 + 1) /* (I, J, K) = (1, 1, k) of a (0:2, 0:2, 0:M3) array */

static int check_poisson(void) {
    static double p[3 * 3 * (M3 + 1)], denf[3 * 3 * (M3 + 1)], divg[N3M];
    double vvdz[M3 + 1], ssdz[M3 + 1], fixkl[M3 + 1], x[M3 + 2];
    int64_t kpv[M3 + 2];
    const double h = 1.0 / N3M;
    for (int k = 0; k <= M3; ++k) {
        ssdz[k] = 1.0 / h;
        if (k >= 1) vvdz[k - 1] = (k == 1 || k == M3) ? 2.0 / h : 1.0 / h;
    }
    for (int k = 1; k <= M3 - 1; ++k) fixkl[k - 1] = (k == 1) ? 1.0 : 0.0;
    for (int k = 0; k <= M3 + 1; ++k) kpv[k] = (k + 1 > M3) ? M3 : k + 1;
    memset(p, 0, sizeof p);
    memset(denf, 0, sizeof denf);
    for (int k = 0; k <= M3; ++k) denf[PIDX(k)] = (k > N3M / 3 && k < N3M / 2) ? 1.0 / 1000.0 : 1.0;
    /* the known pressure, zero at the top ghost (the face p = 0 of the Thomas system) */
    for (int k = 1; k <= N3M; ++k) x[k] = cos(0.5 * M_PI * (k - 0.5) * h) + 0.1 * sin(7.0 * k * h);
    x[0] = x[1];
    x[M3] = 0.0;
    for (int k = 1; k <= N3M; ++k) {
        const double ak = vvdz[k - 1] * ssdz[k] * denf[PIDX(k)] * (1.0 - fixkl[k - 1]);
        const int kp1 = (int)kpv[k];
        const double ck = vvdz[kp1 - 1] * ssdz[k] * denf[PIDX(kp1)];
        const double bk = -(ak + ck);
        divg[k - 1] = ak * x[k - 1] + bk * x[k] + ck * (k == N3M ? 0.0 : x[k + 1]);
    }
    if (lica_gpu_poisson(2, 2, M3, 1, 1, N3M, vvdz, ssdz, fixkl, kpv, p, divg, denf) != LICA_OK)
        return fail("lica_gpu_poisson");
    double err = 0.0, nrm = 0.0;
    for (int k = 1; k <= N3M; ++k) {
        err = fmax(err, fabs(p[PIDX(k)] - x[k]));
        nrm = fmax(nrm, fabs(x[k]));
    }
    if (!(err <= 1e-8 * nrm)) return fail("POISSON solution");
    if (p[PIDX(0)] != p[PIDX(1)] || p[PIDX(M3)] != p[PIDX(N3M)]) return fail("POISSON ghosts");
    return 0;
}

/* ---- 2-D multigrid: A u = sum over faces of beta/h^2 (u_nb - u), x periodic, Neumann
 * bottom, p = 0 on the top face (weight 2/h^2) */
#define NX 128
#define NY 128

static void apply(const double* u, const double* bx, const double* by, double h, double* out) {
    const double c = 1.0 / (h * h);
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const int ip = (i + 1) % NX, im = (i + NX - 1) % NX, q = j * NX + i;
            double s = bx[q] * c * (u[j * NX + im] - u[q]) + bx[j * NX + ip] * c * (u[j * NX + ip] - u[q]);
            if (j > 0) s += by[q] * c * (u[q - NX] - u[q]);
            if (j < NY - 1) s += by[q + NX] * c * (u[q + NX] - u[q]);
            else s += 2.0 * by[q + NX] * c * (0.0 - u[q]);
            out[q] = s;
        }
}

static int check_multigrid(void) {
    static double f[NX * NY], p[NX * NY], bx[NX * NY], by[(NY + 1) * NX], rho[NX * NY], r[NX * NY];
    const double h = 1.0 / NX;
    unsigned s = 12345u;
    double mean = 0.0;
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const double dx = (i + 0.5) * h - 0.4, dy = (j + 0.5) * h - 0.55;
            rho[j * NX + i] = (dx * dx + dy * dy < 0.04) ? 1000.0 : 1.0;
            s = s * 1664525u + 1013904223u;
            f[j * NX + i] = ((s >> 8) / 16777216.0) - 0.5;
            mean += f[j * NX + i];
        }
    mean /= NX * NY;
    for (int q = 0; q < NX * NY; ++q) f[q] -= mean;
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const int im = (i + NX - 1) % NX;
            const double a = rho[j * NX + i], b = rho[j * NX + im];
            bx[j * NX + i] = 2.0 / (a + b);
        }
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const double a = rho[(j < NY ? j : NY - 1) * NX + i], b = rho[(j > 0 ? j - 1 : 0) * NX + i];
            by[j * NX + i] = 2.0 / (a + b);
        }
    lica_mg_options opt = {3, 2, 2, 2, 0, 1};
    lica_mg* m = NULL;
    if (lica_mg_create(&m, NX, NY, h, h, &opt) != LICA_OK) return fail("lica_mg_create");
    memset(p, 0, sizeof p);
    lica_mg_result res;
    const int st = lica_mg_solve_host(m, p, f, bx, by, 1e-10, 100, &res, NULL);
    lica_mg_destroy(m);
    if (st != LICA_OK || res.status != LICA_OK || !(res.rel_residual <= 1e-10)) return fail("lica_mg_solve_host");
    apply(p, bx, by, h, r);
    double rr = 0.0, ff = 0.0;
    for (int q = 0; q < NX * NY; ++q) {
        rr += (f[q] - r[q]) * (f[q] - r[q]);
        ff += f[q] * f[q];
    }
    if (!(sqrt(rr / ff) <= 2e-10)) return fail("multigrid residual from the header's operator");
    return 0;
}

/* ---- whole steps of a column, then the single-routine drop-ins on its state */
#define N 32
#define NF (2 * N)

struct column {
    double w[N + 2], p[N + 2], t[N + 2], psi_cn[N + 2], psi_zn[N + 2], wo[N + 2];
    double phi[NF + 7], mflvs[NF + 7];
    int32_t layer[NF + 7], imask[N + 2];
    double psif[NF + 2], sfgas[NF + 2], sfgas2[NF + 2];
    double scal[5], stats[8];
};

static int check_column(void) {
    static struct column a;
    lica_col_props props = {1.42e-2, 20.0, 1000.0, 7.36e-8, 9.7, 1.0231, 2.077, 25.0, 1.0, 0.009, 0.3, 2.5e-6, 1, 1};
    lica_col_state sa = {a.w, a.p, a.t, a.psi_cn, a.psi_zn, a.phi, a.layer, a.psif,
                         a.wo, a.mflvs, a.sfgas, a.sfgas2, a.imask, a.scal, a.stats};
    if (lica_gpu_column_init(N, 1.0, 0.1, &props, &sa) != LICA_OK) return fail("lica_gpu_column_init");
    int32_t status = -1;
    if (lica_gpu_column_steps(1, N, 1.0, &props, &sa, 4, &status) != LICA_OK || status != LICA_OK)
        return fail("lica_gpu_column_steps");
    if (a.scal[2] != 4.0 || !(a.scal[1] > 0.0) || !(a.stats[5] > 0.1)) return fail("column state after 4 steps");
    /* REINITIALIZATION with no iterations leaves phi as it is; ten keep it finite */
    double phi0[NF + 7];
    memcpy(phi0, a.phi, sizeof phi0);
    if (lica_gpu_reinitialization(1, N, 1.0, a.phi, a.layer, 0, &status) != LICA_OK || status != LICA_OK)
        return fail("lica_gpu_reinitialization (0 iterations)");
    if (memcmp(phi0, a.phi, sizeof phi0) != 0) return fail("REINITIALIZATION with ILIMIT = 0 changed phi");
    if (lica_gpu_reinitialization(1, N, 1.0, a.phi, a.layer, 10, &status) != LICA_OK || status != LICA_OK)
        return fail("lica_gpu_reinitialization");
    for (int k = 0; k < NF + 7; ++k)
        if (!isfinite(a.phi[k])) return fail("REINITIALIZATION result");
    /* GRID_COUPLING(1) recomputes every flow cell: the fractions stay in [0, 1] and the
     * vapour film (psi = 0) stays at the wall */
    if (lica_gpu_grid_coupling(1, N, 1.0, 1, a.psif, a.layer, a.psi_cn, a.psi_zn) != LICA_OK)
        return fail("lica_gpu_grid_coupling");
    for (int k = 1; k <= N; ++k)
        if (a.psi_cn[k] < 0.0 || a.psi_cn[k] > 1.0 || a.psi_zn[k] < 0.0 || a.psi_zn[k] > 1.0)
            return fail("GRID_COUPLING fractions");
    if (a.psi_cn[1] != 0.0 || a.psi_cn[N] != 1.0) return fail("GRID_COUPLING film position");
    return 0;
}

#define BN 8
#define BIDX(i, j, k) ((i) + (BN + 2) * ((j) + (BN + 2) * (k)))

static int check_bubbles(void) {
    static double psi[(BN + 2) * (BN + 2) * (BN + 2)], u[(BN + 2) * (BN + 2) * (BN + 2)],
        v[(BN + 2) * (BN + 2) * (BN + 2)], w[(BN + 2) * (BN + 2) * (BN + 2)];
    double sd[BN + 2], xp[BN + 2];
    const double h = 1.0 / BN;
    for (int i = 0; i < BN + 2; ++i) {
        sd[i] = h;
        xp[i] = (i - 0.5) * h;
    }
    for (int q = 0; q < (BN + 2) * (BN + 2) * (BN + 2); ++q) {
        psi[q] = 1.0;
        u[q] = 1.0;
        v[q] = 2.0;
        w[q] = 3.0;
    }
    for (int k = 2; k <= 5; ++k)
        for (int j = 3; j <= 4; ++j)
            for (int i = 2; i <= 4; ++i) psi[BIDX(i, j, k)] = 0.0;
    lica_bub_grid g = {BN, BN, BN, 1, 1, 0, 1.0, sd, sd, sd, xp, xp, xp};
    lica_bub_record r;
    if (lica_gpu_bubble_tracking(&g, 1, 7, psi, u, v, w, 0.25, 1, &r) != LICA_OK)
        return fail("lica_gpu_bubble_tracking");
    const double h2 = h * h, ev[3] = {8.0 / 12.0 * h2, 3.0 / 12.0 * h2, 15.0 / 12.0 * h2};
    if (r.llvs != 7 || r.time != 0.25 || r.iz_periodic != 0) return fail("bubble record header");
    if (fabs(r.vol - 24.0 * h * h2) > 1e-15) return fail("bubble volume");
    if (fabs(r.col[0] - 2.5 * h) > 1e-14 || fabs(r.col[1] - 3.0 * h) > 1e-14 || fabs(r.col[2] - 3.0 * h) > 1e-14)
        return fail("bubble centroid");
    if (fabs(r.col[3] - 1.0) > 1e-13 || fabs(r.col[4] - 2.0) > 1e-13 || fabs(r.col[5] - 3.0) > 1e-13)
        return fail("bubble velocity");
    for (int a = 0; a < 3; ++a) {
        int found = 0;
        for (int b = 0; b < 3; ++b)
            if (fabs(r.ami[b] - ev[a]) <= 1e-12 * ev[a]) found = 1;
        if (!found) return fail("bubble second moments");
    }
    if (fabs(r.col[6] - sqrt(5.0)) > 1e-12) return fail("bubble aspect ratio");
    if (fabs(r.col[7] - 90.0) > 1e-9 || fabs(r.col[8] - 90.0) > 1e-9) return fail("bubble angles");
    return 0;
}

int main(void) {
    if (check_poisson() || check_multigrid() || check_column() || check_bubbles()) return 1;
    printf("ok\n");
    return 0;
}
