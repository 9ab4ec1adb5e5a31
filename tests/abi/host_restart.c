/* A compiled host driving the library through include/lica_gpu.h alone, as a Fortran or C
 * solver would: the initial column (MAKEFLD + LVSINIT + GRID_COUPLING), its fld restart file
 * written and read back (WRITEFIELD / PREFLD), the POISSON metrics of a stretched grid from
 * the generator's sections (grid.f, GEOMETRIC), its coupling tables to the level-set grid
 * (GEOM_COUPLING) and its 2-D pressure system for the multigrid.  Host entry points only: no GPU.
 * Usage: host_restart <directory>.  Prints "ok" and exits 0, or names the failed check. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lica_gpu.h"

#define N 32
#define NF (2 * N)

static int fail(const char* what) {
    fprintf(stderr, "FAILED: %s (%s)\n", what, lica_last_error());
    return 1;
}

struct column {
    double w[N + 2], p[N + 2], t[N + 2], psi_cn[N + 2], psi_zn[N + 2], wo[N + 2];
    double phi[NF + 7], mflvs[NF + 7];
    int32_t layer[NF + 7], imask[N + 2];
    double psif[NF + 2], sfgas[NF + 2], sfgas2[NF + 2];
    double scal[5], stats[8];
};

static lica_col_state view(struct column* c) {
    lica_col_state s = {c->w, c->p, c->t, c->psi_cn, c->psi_zn, c->phi, c->layer, c->psif,
                        c->wo, c->mflvs, c->sfgas, c->sfgas2, c->imask, c->scal, c->stats};
    return s;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    static struct column a, b;
    lica_col_props props = {1.42e-2, 22.22, 1605.36, 7.36e-8, 9.7, 1.0231, 2.077, 27.16, 1.0, 0.009, 0.5, 2.5e-6, 1, 1};
    lica_col_state sa = view(&a), sb = view(&b);
    if (lica_gpu_column_init(N, 1.0, 0.2, &props, &sa) != LICA_OK) return fail("lica_gpu_column_init");

    char name[16], path[4096];
    if (lica_fld_name(7, name, (int32_t)sizeof name) != LICA_OK || strcmp(name, "fld000007") != 0)
        return fail("lica_fld_name");
    snprintf(path, sizeof path, "%s/%s", argv[1], name);
    lica_fld_info info;
    memset(&info, 0, sizeof info);
    info.ihist = 7;
    info.ips = 1;
    info.ipx = 1;
    info.ipy = 1;
    info.ipz = 3;
    info.lvson = 1;
    info.t_con = 100.0;
    if (lica_col_fld_write(path, N, &props, &sa, &info) != LICA_OK) return fail("lica_col_fld_write");

    int32_t n = 0;
    if (lica_col_fld_dims(path, &n) != LICA_OK || n != N) return fail("lica_col_fld_dims");
    lica_fld_options opt = {0, 1, 0};
    lica_fld_info got;
    if (lica_col_fld_read(path, n, 1.0, &props, &opt, &sb, &got) != LICA_OK) return fail("lica_col_fld_read");
    if (got.ihist != 7 || got.n_max != 11 || got.t_con != 100.0) return fail("header values");
    for (int k = 0; k < NF + 7; ++k)
        if (a.layer[k] != b.layer[k]) return fail("band layers");
    for (int k = 1; k <= N; ++k)
        if (fabs(a.w[k] - b.w[k]) > 5e-13 * fabs(a.w[k]) || fabs(a.p[k] - b.p[k]) > 5e-13 * fabs(a.p[k]) ||
            fabs(a.t[k] - b.t[k]) > 5e-13 * fabs(a.t[k]))
            return fail("W, P, T to 13 digits");
    for (int k = 1; k <= N; ++k)
        if (fabs(a.psi_cn[k] - b.psi_cn[k]) > 1e-12) return fail("PSI_CN recomputed");
    if (b.scal[2] != 0.0 || fabs(b.scal[4] - a.scal[3]) > 5e-13) return fail("M and VOL_TOT_IPHS after a read");
    if (lica_col_fld_read("/nonexistent/fld000001", n, 1.0, &props, &opt, &sb, &got) != LICA_ERR_IO)
        return fail("a missing file is LICA_ERR_IO");

    /* a tanh-stretched column: GEOMETRIC of its 65 faces */
    double z[66], sdz[66], vdz[66], ssdz[66], vvdz[66], zp[66];
    if (lica_grid_section(3, 0.0, 1.0, 1, 65, 2.0, 1.0, z + 1) != LICA_OK) return fail("lica_grid_section");
    if (lica_grid_metrics(65, z, sdz, vdz, ssdz, vvdz, zp) != LICA_OK) return fail("lica_grid_metrics");
    double total = 0.0;
    for (int k = 1; k <= 64; ++k) total += sdz[k];
    if (fabs(total - 1.0) > 1e-14 || !(sdz[1] < sdz[64]) || vdz[1] != 0.5 * sdz[1] || vdz[65] != 0.5 * sdz[64])
        return fail("stretched metrics");
    /* GEOM_COUPLING's tables of that grid against a uniform 129-face level-set grid */
    double zf[130];
    for (int k = 1; k <= 129; ++k) zf[k] = (k - 1) / 128.0;
    int32_t kc1[69], kc2[69], km1[68], km2[68], kv[130], kmv[130];
    if (lica_grid_coupling_z(65, z, 129, zf, kc1, kc2, km1, km2, kv, kmv) != LICA_OK) return fail("coupling tables");
    for (int k = 1; k <= 64; ++k)
        if (kc2[k + 1] > kc1[k + 2] + 1 || zf[kc2[k + 1]] > z[k] + 1e-12 || zf[kc1[k + 2] + 1] < z[k + 1] - 1e-12)
            return fail("flow cell boxes cover their cells");
    /* the stretched pressure system of a 32 x 64 field on those faces */
    static double bx[64 * 32], by[65 * 32], f[64 * 32], bxo[64 * 32], byo[65 * 32], fo[64 * 32];
    for (int q = 0; q < 64 * 32; ++q) bx[q] = f[q] = 1.0;
    for (int q = 0; q < 65 * 32; ++q) by[q] = 1.0;
    if (lica_mg_stretched_system(32, 64, z + 1, bx, by, f, bxo, byo, fo) != LICA_OK) return fail("stretched system");
    if (fabs(fo[0] - sdz[1]) > 1e-15 || fabs(byo[64 * 32] - 1.0 / sdz[64]) > 1e-9 * byo[64 * 32])
        return fail("stretched system values");
    printf("ok\n");
    return 0;
}
