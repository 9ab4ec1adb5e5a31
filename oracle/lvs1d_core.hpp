// ORACLE (test infrastructure only) -- internal routines of the 1-D level-set
// restatement, shared by lvs1d.cpp (TRANSPORT) and column1d.cpp (the RK3 column step).
// Every routine cites the Fortran it restates; see lvs1d.cpp for the 1-D reductions and
// the reference quirks kept.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

// Wall-normal geometry of a stretched column: GEOMETRIC's arrays (1d.f:4808-4882) and
// GEOM_COUPLING's z tables (1d.f:5037-5370) as lica_grid_metrics and lica_grid_coupling_z
// write them (the level-set grid stays uniform).  Flow arrays are n+2 long, indexed by the
// Fortran index: z (faces 1..n+1), zp (0..n+1), sdz, ssdz (1..n), vdz, vvdz (1..n+1).
// kcou1/kcou2: faces K = -1..n+2 at [K+1]; kcoump1/kcoump2: centres K = -1..n+1 at [K+1];
// kcou_vel, kcoump_vel: refined faces / centres K = 1..nf at [K].  A null geometry is the
// uniform column.
struct ColGeo {
    const double *z, *zp, *sdz, *vdz, *ssdz, *vvdz;
    const int *kcou1, *kcou2, *kcoump1, *kcoump2, *kcou_vel, *kcoump_vel;
};

constexpr int N_MAX = 11;          // M_MAX, 1dmodulesX.f:21
constexpr int NN1 = N_MAX - 3;     // two_phase.f:737
constexpr int NN2 = N_MAX - 1;     // two_phase.f:738
constexpr int GL = 2;              // offset of k = -2 (three ghost cells below k = 1)

struct Col {
    int n = 0, nf = 0;       // flow cells, refined cells
    double L = 1.0, h = 0, hf = 0, ssdzf = 0;
    const ColGeo* cg = nullptr;  // the flow grid's geometry (null: uniform)
    std::vector<double> phi;     // ALPHI_EXT(k), k = -2..nf+4 at [k + GL] (nf+7 values)
    std::vector<int> layer;      // band layer of refined cell k (0 = outside), same indexing
    std::vector<std::vector<int>> band;  // band[n] = z-levels of layer n (1-based k), reference order
    double& p(int k) { return phi[k + GL]; }
    int& lay(int k) { return layer[k + GL]; }
    void init(int n_, double L_) {
        n = n_;
        nf = 2 * n_;
        L = L_;
        h = L / n;
        hf = L / nf;
        ssdzf = 1.0 / hf;
        phi.assign(nf + 7, 0.0);
        layer.assign(nf + 7, 0);
        band.assign(N_MAX + 1, {});
    }
    void rebuild_layer() {
        std::fill(layer.begin(), layer.end(), 0);
        for (int m = 1; m <= N_MAX; ++m)
            for (int k : band[m]) lay(k) = m;
    }
};

// ALPHI_BC, two_phase.f:462-642, z part (IPZ != 1).
void alphi_bc(Col& c) {
    const int nf = c.nf;
    const double dz = c.hf;
    const double a1 = c.p(1);
    if (std::fabs(a1) < 1e-8) {
        c.p(0) = 0.0; c.p(-1) = 0.0; c.p(-2) = 0.0;
    } else if (a1 > 0.0) {
        c.p(0) = a1 + dz; c.p(-1) = c.p(0) + dz; c.p(-2) = c.p(-1) + dz;
    } else if (a1 < 0.0) {
        c.p(0) = a1 - dz; c.p(-1) = c.p(0) - dz; c.p(-2) = c.p(-1) - dz;
    }
    const double an = c.p(nf);
    if (std::fabs(an) < 1e-8) {
        for (int q = 1; q <= 4; ++q) c.p(nf + q) = 0.0;
    } else if (an > 0.0) {
        c.p(nf + 1) = an + dz;
        for (int q = 2; q <= 4; ++q) c.p(nf + q) = c.p(nf + q - 1) + dz;
    } else if (an < 0.0) {
        c.p(nf + 1) = an - dz;
        for (int q = 2; q <= 4; ++q) c.p(nf + q) = c.p(nf + q - 1) - dz;
    }
    // periodic copy that follows for IPZ != 1 (two_phase.f:624-634), N3F_BD = 2
    for (int k = 0; k <= 2; ++k) {
        c.p(-k) = c.p(nf - k);
        c.p(nf + 1 + k) = c.p(1 + k);
    }
}

// BAND_GENERATION, two_phase.f:1622-2030 (1-D).  Returns 1 if a new layer would leave
// the stored range k = -2..nf+4 (a band seeded at k = 1 grows downwards without end; the
// reference writes past ALPHI_EXT there), else 0.
int band_generation(Col& c) {
    const int nf = c.nf;
    std::vector<int> mask(nf + 7, 0);
    auto ms = [&](int k) -> int& { return mask[k + GL]; };
    std::vector<std::vector<int>> nb(N_MAX + 1);
    // S-tube from the old layers 1..NN2 (two_phase.f:1655-1680)
    for (int m = 1; m <= NN2; ++m)
        for (int k : c.band[m]) {
            if (c.p(k) * c.p(k + 1) < 0.0 || c.p(k) * c.p(k - 1) < 0.0) {
                nb[1].push_back(k);
                ms(k) = 1;
            } else {
                ms(k) = 2;
            }
        }
    const double d = std::sqrt(0.0 + 0.0 + c.hf * c.hf);  // dx = dy = 0, dz = SDZF (:1931-1936)
    int overflow = 0;
    for (int m = 2; m <= N_MAX; ++m) {
        for (int k : nb[m - 1]) {
            for (int k2 = k - 1; k2 <= k + 1; ++k2) {
                if (k2 == 1 || k2 == nf + 1) continue;     // boundary touch, :1704-1713
                if (k2 < -2 || k2 > nf + 4) { overflow = 1; continue; }
                if (ms(k2) == 1) continue;
                if (ms(k2) == 0 || m >= NN2) c.p(k2) = (c.p(k) >= 0.0) ? c.p(k) + d : c.p(k) - d;
                nb[m].push_back(k2);
                ms(k2) = 1;
            }
        }
    }
    c.band = nb;
    c.rebuild_layer();
    return overflow;
}

// HJWENO, two_phase.f:2477-2500.
inline double hjweno(double a, double b, double cc, double dd) {
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

// one-sided WENO5 derivatives at k from face differences dphi (dphi(k) = (phi(k+1)-phi(k))/dz)
inline void weno_z(const std::vector<double>& dp, int k, double& dm, double& dpl) {
    auto D = [&](int q) { return dp[q + GL]; };
    {
        const double v1 = D(k - 3), v2 = D(k - 2), v3 = D(k - 1), v4 = D(k), v5 = D(k + 1);
        const double w = hjweno(v2 - v1, v3 - v2, v4 - v3, v5 - v4);
        dm = 1.0 / 12.0 * (-v2 + 7.0 * v3 + 7.0 * v4 - v5) - w;
    }
    {
        const double v1 = D(k + 2), v2 = D(k + 1), v3 = D(k), v4 = D(k - 1), v5 = D(k - 2);
        const double w = hjweno(v1 - v2, v2 - v3, v3 - v4, v4 - v5);
        dpl = 1.0 / 12.0 * (-v5 + 7.0 * v4 + 7.0 * v3 - v2) + w;
    }
}

// Face differences of phi wherever a WENO stencil of a layer <= NN1 cell reaches.
std::vector<double> face_diff(Col& c) {
    std::vector<double> dp(c.nf + 7, 0.0);
    for (int k = -2; k <= c.nf + 3; ++k) dp[k + GL] = (c.p(k + 1) - c.p(k)) * c.ssdzf;  // k+1 <= nf+4
    return dp;
}

// TRANSPORT_RK3, two_phase.f:1133-1495 (1-D: x/y terms are exactly 0).
void transport_rk3(Col& c, double dtlvs, const std::vector<double>& wf, const std::vector<double>& mf,
                   const std::vector<double>& alphi_start, int iphs, double denr) {
    std::vector<double> dp = face_diff(c);
    std::vector<std::pair<int, double>> upd;
    for (int m = 1; m <= NN1; ++m)
        for (int k : c.band[m]) {
            const double uu1 = wf[k + GL], uu2 = wf[k + 1 + GL], uu3 = 0.5 * (uu1 + uu2);
            double az;
            if (uu1 >= 0.0 && uu2 >= 0.0 && uu3 >= 0.0) {
                double dm, dpl;
                weno_z(dp, k, dm, dpl);
                az = uu3 * dm;
            } else if (uu1 <= 0.0 && uu2 <= 0.0 && uu3 <= 0.0) {
                double dm, dpl;
                weno_z(dp, k, dm, dpl);
                az = uu3 * dpl;
            } else {
                double dm, dpl;
                weno_z(dp, k, dm, dpl);
                const double umax = std::max(std::max(std::fabs(uu1), std::fabs(uu2)), std::fabs(uu3));
                az = 0.5 * (uu3 * (dpl + dm) - umax * (dpl - dm));
            }
            double pn = c.p(k) - dtlvs * ((0.0 + 0.0) + az);
            if (iphs == 1) {
                if (alphi_start[k + GL] > 0.0) pn = pn - dtlvs * mf[k + GL] / denr;
                else pn = pn - dtlvs * mf[k + GL];
            }
            upd.push_back({k, pn});
        }
    for (auto& u : upd) c.p(u.first) = u.second;
}

// GODUNOV, two_phase.f:2448-2474.
inline double godunov(double s, double ap, double am) {
    const double aplus = s * ap, aminus = s * am;
    if (aplus >= 0.0 && aminus >= 0.0) return am;
    if (aplus <= 0.0 && aminus <= 0.0) return ap;
    if (aplus > 0.0 && aminus < 0.0) return 0.0;
    if (aplus + aminus > 0.0) return am;
    return ap;
}

// REINITIALIZATION_RK3, two_phase.f:2174-2445 (1-D).
void reinit_rk3(Col& c, double redtl, const std::vector<double>& alphio) {
    const double eps = c.hf * c.hf;  // MIN(SDXF,SDYF,SDZF)**2, :2200-2204
    std::vector<double> dp = face_diff(c);
    std::vector<std::pair<int, double>> upd;
    for (int m = 1; m <= NN2; ++m)
        for (int k : c.band[m]) {
            const double dz = 0.5 * (c.p(k + 1) - c.p(k - 1)) * c.ssdzf;
            const double dal = (0.0 + 0.0) + dz * dz;
            const double a0 = alphio[k + GL];
            const double s = a0 / std::sqrt(a0 * a0 + dal * eps);
            double dm, dpl;
            if (m <= NN1) {
                weno_z(dp, k, dm, dpl);
            } else {
                dm = (c.p(k) - c.p(k - 1)) * c.ssdzf;
                dpl = (c.p(k + 1) - c.p(k)) * c.ssdzf;
            }
            const double ax = godunov(s, 0.0, 0.0), ay = godunov(s, 0.0, 0.0);
            const double az = godunov(s, dpl, dm);
            const double drhs = s * (1.0 - std::sqrt(ax * ax + ay * ay + az * az));
            upd.push_back({k, c.p(k) + redtl * drhs});
        }
    for (auto& u : upd) c.p(u.first) = u.second;
}

// REINITIALIZATION, two_phase.f:2033-2170: SSP-RK3 pseudo-time, ILIMIT iterations.
void reinitialization(Col& c, int ilimit) {
    std::vector<double> alphio(c.phi);
    const double redtl = 0.5 * c.hf;  // 0.5*MIN(SDXF,SDYF,SDZF), :2063-2067
    for (int it = 0; it < ilimit; ++it) {
        std::vector<double> rk3(c.phi);
        reinit_rk3(c, redtl, alphio);
        reinit_rk3(c, redtl, alphio);
        for (int m = 1; m <= NN2; ++m)
            for (int k : c.band[m]) c.p(k) = 0.75 * rk3[k + GL] + 0.25 * c.p(k);
        reinit_rk3(c, redtl, alphio);
        for (int m = 1; m <= NN2; ++m)
            for (int k : c.band[m]) c.p(k) = 1.0 / 3.0 * rk3[k + GL] + 2.0 / 3.0 * c.p(k);
    }
}

// REIN_TRIGGER, two_phase.f:646-697.
void rein_trigger(Col& c, double& dmax, double& dmin) {
    dmax = 0.0;
    dmin = 1.0;
    for (int m = 1; m <= NN1; ++m)
        for (int k : c.band[m]) {
            const double dz = 0.5 * (c.p(k + 1) - c.p(k - 1)) * c.ssdzf;
            const double s = (0.0 + 0.0) + dz * dz;
            dmax = std::max(s, dmax);
            dmin = std::min(s, dmin);
        }
    dmax = std::sqrt(dmax);
    dmin = std::sqrt(dmin);
}

// VEL_INTP/VELASSIGN, two_phase.f:5539-6035 (1-D, z interpolation of W).
// Lagrange weights at ZZ = ZF(k) on nodes ZP(KK-1..KK+2), KK = KCOU_VEL(k).
void vel_intp(Col& c, const std::vector<double>& wt, std::vector<double>& wf) {
    const int n = c.n;
    const ColGeo* cg = c.cg;
    auto zp = [&](int k) { return cg ? cg->zp[k] : (k - 1) * c.h + 0.5 * c.h; };
    auto vdz = [&](int k) { return cg ? cg->vdz[k] : ((k == 1 || k == n + 1) ? 0.5 * c.h : c.h); };
    auto wtv = [&](int k) { return (k < 0 || k > n + 1) ? 0.0 : wt[k]; };
    std::fill(wf.begin(), wf.end(), 0.0);
    for (int m = 1; m <= NN2; ++m)
        for (int k : c.band[m]) {
            const double zz = (k - 1) * c.hf;
            int kk = 1;   // KCOU_VEL (GEOM_COUPLING 1d.f:5130-5240 pattern)
            for (int q = 1; q <= n; ++q) {
                if (std::fabs(zz - zp(q)) <= 1e-10) { kk = q; break; }
                if (zp(1) > zz) { kk = 1; break; }
                if (zp(q) > zz) { kk = q - 1; break; }
                if (zp(n) < zz) { kk = n; break; }
            }
            const double z2 = zp(kk), z1 = z2 - vdz(kk);
            double z3, z4;
            if (kk == n - 1) { z3 = z2 + vdz(kk + 1); z4 = z3 + 2.0 * vdz(n + 1); }
            else if (kk == n) { z3 = z2 + 2.0 * vdz(n + 1); z4 = z3 + vdz(n); }
            else { z3 = z2 + vdz(kk + 1); z4 = z3 + vdz(kk + 2); }
            const double cz1 = ((zz - z2) * (zz - z3) * (zz - z4)) / ((z1 - z2) * (z1 - z3) * (z1 - z4));
            const double cz2 = ((zz - z1) * (zz - z3) * (zz - z4)) / ((z2 - z1) * (z2 - z3) * (z2 - z4));
            const double cz3 = ((zz - z1) * (zz - z2) * (zz - z4)) / ((z3 - z1) * (z3 - z2) * (z3 - z4));
            const double cz4 = ((zz - z1) * (zz - z2) * (zz - z3)) / ((z4 - z1) * (z4 - z2) * (z4 - z3));
            const double w = cz1 * wtv(kk - 1) + cz2 * wtv(kk) + cz3 * wtv(kk + 1) + cz4 * wtv(kk + 2);
            wf[k + GL] = (m < NN2 - 1) ? w : w * 0.5;
        }
    for (int k : c.band[N_MAX]) wf[k + GL] = 0.0;
}

// CAL_PSIF_MTP, two_phase.f:2835-3060 (1-D) on band layers 1..nn1.  Returns psif_mtp
// on k = 1..nf (index k).
std::vector<double> cal_psif_mtp(Col& c, int iouter, int nn1 = NN1) {
    const int nf = c.nf;
    std::vector<double> ps(nf + 2, 0.0);
    std::vector<int> mask(nf + 2, 0);
    const double eps = 1e-8;
    for (int m = 1; m <= nn1; ++m)
        for (int k : c.band[m]) {
            const double d3 = 0.5 * std::fabs(c.p(k + 1) - c.p(k - 1));
            const double e1 = d3;   // D1 = D2 = 0: E1 = D3, E2 = E3 = 0
            double t;
            if (e1 > eps) {
                const double f1 = std::max(0.5 * (e1 + 0.0 + 0.0) - std::fabs(c.p(k)), 0.0);
                t = f1 / e1;
            } else {
                t = (c.p(k) != 0.0) ? 0.0 : 0.5;
            }
            ps[k] = (c.p(k) <= 0.0) ? t : 1.0 - t;
            mask[k] = 1;
        }
    for (int m = 1; m <= nn1; ++m)
        for (int k : c.band[m]) {
            if (ps[k] < 1e-5) ps[k] = 0.0;
            else if (ps[k] > 0.99999) ps[k] = 1.0;
        }
    if (iouter == 1) {
        std::vector<int> kc;
        for (int k = nf; k >= 1; --k)
            if (c.p(k) * c.p(k + 1) < 0.0) kc.push_back(k);
        if (kc.empty()) {
            for (int k = 1; k <= nf; ++k)
                if (!mask[k]) ps[k] = 1.0;   // PSIF_BACKGROUND = 1
        } else {
            const int knum = (int)kc.size();
            for (int l = 0; l < knum; ++l) {
                const double t = (c.p(kc[l]) < 0.0) ? 0.0 : 1.0;
                if (l == 0) {
                    const int k0 = (std::fabs(ps[1] - 0.5) < 0.5) ? 2 : 1;
                    for (int k = k0; k <= kc[l]; ++k)
                        if (!mask[k]) ps[k] = t;
                } else {
                    for (int k = kc[l - 1]; k <= kc[l]; ++k)   // empty when kc descends (Fortran DO)
                        if (!mask[k]) ps[k] = t;
                }
            }
            // KC(K_NUM+1) = 0 /= N3FM: the outer fill always runs (:3040-3049)
            const double t = (c.p(kc[knum - 1] + 1) < 0.0) ? 0.0 : 1.0;
            for (int k = kc[knum - 1] + 1; k <= nf; ++k)
                if (!mask[k]) ps[k] = t;
        }
    }
    return ps;
}

// GLOBAL_MASS_CORRECTION, two_phase.f:6196-6318 (1-D; DVOL = SDXF*SDYF*SDZF with
// SDXF = SDYF = 1/2, four (I,J) replicas per z-level).
void global_mass_correction(Col& c, double& vol_tot_ori, double vol_tot_iphs, int iphs) {
    const double sdxf = 0.5, sdyf = 0.5;
    const double recor = std::min(std::min(sdxf, sdyf), c.hf) * 1.5;
    const double dvol = sdxf * sdyf * c.hf;
    if (iphs == 1) vol_tot_ori = vol_tot_iphs;
    double vol_tot = 0.0, vol_in = 0.0;
    for (int l = 1; l <= 15; ++l) {
        double vol_band = 0.0;
        if (l == 1) {
            std::vector<double> ps = cal_psif_mtp(c, 1);
            vol_tot = 0.0;
            for (int k = 1; k <= c.nf; ++k)
                for (int r = 0; r < 4; ++r) vol_tot = vol_tot + (1.0 - ps[k]) * dvol;
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m])
                    for (int r = 0; r < 4; ++r) vol_band = vol_band + (1.0 - ps[k]) * dvol;
            vol_in = vol_tot - vol_band;
        } else {
            std::vector<double> ps = cal_psif_mtp(c, 0);
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m])
                    for (int r = 0; r < 4; ++r) vol_band = vol_band + (1.0 - ps[k]) * dvol;
            vol_tot = vol_in + vol_band;
        }
        if (std::fabs(vol_tot - vol_tot_ori) >= 1e-5) {
            const double cor = recor * (-(vol_tot_ori - vol_tot) / vol_tot_ori);
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m]) c.p(k) = c.p(k) + cor;
        } else {
            break;
        }
    }
}

// Uniform column geometry (GEOMETRIC 1d.f:4808-4866, GEOMETRIC_LVS 1d.f:4885-4944): flow
// faces Z(k) = (k-1) h, centres ZP(k) = Z(k) + h/2 (ZP(0) = Z(1), ZP(n+1) = Z(n+1)),
// refined faces ZF(k) = (k-1) hf with hf = h/2.
inline double grid_z(double h, int k) { return (k - 1) * h; }
inline double grid_zp(double h, int n, int k) {
    if (k <= 0) return 0.0;
    if (k >= n + 1) return n * h;
    return (k - 1) * h + 0.5 * h;
}
inline double grid_zf(double hf, int k) { return (k - 1) * hf; }

// KCOUMP_VEL(k) (GEOM_COUPLING 1d.f:5150-5188): the flow cell whose centre is the last at
// or below the refined centre ZPF(k), found by the reference's search.
inline int kcoump_vel(double h, double hf, int n, int k) {
    const double zz = (k - 1) * hf + 0.5 * hf;
    for (int q = 1; q <= n; ++q) {
        if (std::fabs(zz - grid_zp(h, n, q)) <= 1e-10) return q;
        if (grid_zp(h, n, 1) > zz) return 1;
        if (grid_zp(h, n, q) > zz) return q - 1;
        if (grid_zp(h, n, n) < zz) return n;
    }
    return 1;
}

// z part of the refined-grid box integrals INTER_PSI (two_phase.f:5123-5538),
// INTER_PSI_FACE (1d.f:2552-2958) and INTER_PSI_MTP (two_phase.f:4433-4862) over
// [z1,z2] x refined cells k1..k2.  In the 1-D column the x and y ranges cover both
// refined replicas whole, so the z loop runs once per (II,JJ) replica, four times, and
// the result is PSI_SUM/VOLF.  f is indexed [k] for k = 1..nf; an index outside that
// range reads the nearest end value (the reference reads its refined-array ghosts).
inline double box_mean(const double* f, int nf, int k1, int k2, double z1, double z2, double hf) {
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

// GRID_COUPLING (two_phase.f:4863-5118) on the 1-D column.  ini = 1: every flow cell;
// ini = 0: flow cells KCOUMP_VEL(k) of the refined cells MASK_GLOBAL marks (band layers
// 1..NN1, set by CAL_PSIF).  PSI_ZN(K), K = 2..n: box mean of PSIF over [ZP(K-1),ZP(K)],
// refined cells 2K-2..2K-1; PSI_CN(K): over [Z(K),Z(K+1)], cells 2K-1..2K; snaps at
// 1e-3 / 0.999; PSI_CN(0) = PSI_CN(1), PSI_CN(n+1) = PSI_CN(n).
inline void grid_coupling(int n, double L, const double* psif, const int* layer /* [k+GL] or null */, int ini,
                          double* psi_cn, double* psi_zn, const ColGeo* cg = nullptr) {
    const int nf = 2 * n;
    const double h = L / n, hf = L / nf;
    auto zp = [&](int k) { return cg ? cg->zp[k] : grid_zp(h, n, k); };
    auto zf = [&](int k) { return cg ? cg->z[k] : grid_z(h, k); };
    std::vector<int> mask(n + 2, ini ? 1 : 0);
    if (!ini)
        for (int k = 1; k <= nf; ++k) {
            const int m = layer[k + GL];
            if (m >= 1 && m <= NN1) mask[cg ? cg->kcoump_vel[k] : kcoump_vel(h, hf, n, k)] = 1;
        }
    // INTER_PSI over the face box [ZP(K-1), ZP(K)], refined cells KCOUMP2(K-1)..KCOUMP1(K)
    for (int k = 2; k <= n; ++k)
        if (mask[k])
            psi_zn[k] = box_mean(psif, nf, cg ? cg->kcoump2[k] : 2 * k - 2, cg ? cg->kcoump1[k + 1] : 2 * k - 1,
                                 zp(k - 1), zp(k), hf);
    for (int k = 1; k <= n; ++k) {
        if (psi_zn[k] < 1e-3) psi_zn[k] = 0.0;
        else if (psi_zn[k] > 0.999) psi_zn[k] = 1.0;
    }
    // over the cell box [Z(K), Z(K+1)], refined cells KCOU2(K)..KCOU1(K+1)
    for (int k = 1; k <= n; ++k)
        if (mask[k])
            psi_cn[k] = box_mean(psif, nf, cg ? cg->kcou2[k + 1] : 2 * k - 1, cg ? cg->kcou1[k + 2] : 2 * k, zf(k),
                                 zf(k + 1), hf);
    for (int k = 1; k <= n; ++k) {
        if (psi_cn[k] < 1e-3) psi_cn[k] = 0.0;
        else if (psi_cn[k] > 0.999) psi_cn[k] = 1.0;
    }
    psi_cn[0] = psi_cn[1];
    psi_cn[n + 1] = psi_cn[n];
}

struct State {
    Col c;
    std::vector<double> psif;    // PSIF(k), k = 1..nf (index k), persistent
    std::vector<double> wo;      // WO(k), flow faces 0..n+1
    double vol_tot_ori = 0.0;
};

}  // namespace
