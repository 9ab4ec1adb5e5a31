// Geometry of the uniform 1-D boiling column and the refined-grid box integral, shared by
// the level-set (lvs.cu) and column-step (column.cu) kernels.
//   flow faces Z(k) = (k-1) h, centres ZP(k) = Z(k) + h/2 (ZP(0) = Z(1), ZP(n+1) = Z(n+1)),
//   refined faces ZF(k) = (k-1) hf, hf = h/2  (GEOMETRIC 1d.f:4808-4866, GEOMETRIC_LVS
//   1d.f:4885-4944, uniform grid).
#pragma once
#include <cmath>

namespace lica {
namespace col {

// Wall-normal geometry of a stretched column (device arrays, shared by the columns of a
// launch): GEOMETRIC's arrays (1d.f:4808-4882) and GEOM_COUPLING's z tables
// (1d.f:5037-5370) in the layout of lica_col_geometry (include/lica_gpu.h).  The level-set
// grid stays uniform.  A null pointer is the uniform column of the closed forms below.
struct ColGeoDev {
    const double *z, *zp, *sdz, *vdz, *ssdz, *vvdz;
    const int *kcou1, *kcou2, *kcoump1, *kcoump2, *kcou_vel, *kcoump_vel;
};

__device__ __forceinline__ double grid_z(double h, int k) { return (k - 1) * h; }
__device__ __forceinline__ double grid_zp(double h, int n, int k) {
    if (k <= 0) return 0.0;
    if (k >= n + 1) return n * h;
    return (k - 1) * h + 0.5 * h;
}
__device__ __forceinline__ double grid_zf(double hf, int k) { return (k - 1) * hf; }
__device__ __forceinline__ double grid_zpf(double hf, int k) { return (k - 1) * hf + 0.5 * hf; }

// KCOUMP_VEL(k) (GEOM_COUPLING 1d.f:5150-5188): the reference's search for the last flow
// centre at or below the refined centre ZPF(k).  Every q below k/2 - 2 has ZP(q) more than
// two flow cells under ZPF(k) and fails all four tests except the two that do not depend on
// q, so the search may start there and returns the same cell.
__device__ __forceinline__ int kcoump_vel(double h, double hf, int n, int k) {
    const double zz = grid_zpf(hf, k);
    for (int q = max(1, k / 2 - 2); q <= n; ++q) {
        if (fabs(zz - grid_zp(h, n, q)) <= 1e-10) return q;
        if (grid_zp(h, n, 1) > zz) return 1;
        if (grid_zp(h, n, q) > zz) return q - 1;
        if (grid_zp(h, n, n) < zz) return n;
    }
    return 1;
}

// z part of the box integrals INTER_PSI (two_phase.f:5123-5538), INTER_PSI_FACE
// (1d.f:2552-2958) and INTER_PSI_MTP (two_phase.f:4433-4862) over [z1,z2] x refined cells
// k1..k2: the x/y ranges cover both refined replicas whole, so the z loop runs once per
// (II,JJ) replica -- four times -- and the result is PSI_SUM/VOLF.  f is indexed [k],
// k = 1..nf; indices outside that range read the nearest end value.
__device__ __forceinline__ double box_mean(const double* f, int nf, int k1, int k2, double z1, double z2,
                                           double hf) {
    const double ssdzf = 1.0 / hf;
    double sum = 0.0, volf = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        for (int kk = k1; kk <= k2; ++kk) {
            const double v = f[kk < 1 ? 1 : (kk > nf ? nf : kk)];
            const double za = grid_zf(hf, kk), zb = grid_zf(hf, kk + 1);
            if (za <= z1 && zb >= z2) {
                sum = sum + v;
                volf = volf + 1.0;
                break;
            } else if (za < z1 && zb > z1) {
                sum = sum + v * (zb - z1) * ssdzf;
                volf = volf + (zb - z1) * ssdzf;
            } else if (za >= z1 && zb <= z2) {
                sum = sum + v;
                volf = volf + 1.0;
            } else if (za < z2 && zb > z2) {
                sum = sum + v * (z2 - za) * ssdzf;
                volf = volf + (z2 - za) * ssdzf;
            } else if (za >= z2) {
                break;
            }
        }
    }
    return sum / volf;
}

}  // namespace col
}  // namespace lica

// A stretched column's geometry on the device (lica_gpu_column_geometry_create): the
// column size and length it was checked for and one buffer holding its arrays.
struct lica_col_geo {
    int n = 0;
    double length = 0.0;
    void* buf = nullptr;
    lica::col::ColGeoDev dev{};
};
