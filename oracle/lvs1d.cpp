// ORACLE (test infrastructure only) -- CPU restatement of the reference's level-set
// transport path for the 1-D column (the shipped case: 1 x 1 x N flow cells, refined
// level-set grid 2 x 2 x 2N, replicated in x and y).  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU legs load it.
//
// Parity status: unpinned against the reference (no Fortran compiler here, no reference
// outputs).  Every routine follows the cited Fortran statement by statement in its 1-D
// form.  The 1-D reductions, each exact in real arithmetic:
//   * x/y derivatives vanish (two_phase.f:885-892 replicates phi over I,J), so every x/y
//     WENO/upwind/Godunov term is exactly 0 and |grad phi|^2 = 0 + 0 + dz^2;
//   * the 2x2 (I,J) replicas of a refined z-level carry identical values, so band
//     lists hold one entry per z-level, sums over the replicas add the value 4 times;
//   * x/y Lagrange weights sum to 1 in VELASSIGN (two_phase.f:5700-6000); the 1-D form
//     interpolates in z only;
//   * box integrals of INTER_PSI/INTER_PSI_MTP over a flow cell reduce to the mean of
//     its two refined cells (refinement ratio 2, aligned grids).
// Reference quirks kept on purpose (the reference's behaviour):
//   * ALPHI_BC (two_phase.f:555-634): with IPZ != 1 the wall extrapolation of the z
//     ghosts is followed by a periodic copy of ghosts 0,-1,-2 and N3F..N3F+2;
//   * BAND_GENERATION (two_phase.f:1719-1735) never adds k = 1 or k = N3F to the band;
//   * VEL_INTP (two_phase.f:6000-6035) interpolates the face velocity W with the flow
//     cell-centre positions ZP as nodes;
//   * TRANSPORT (two_phase.f:966-984) stores the band phi before its final
//     GLOBAL_MASS_CORRECTION, so that call only updates the target volume.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

constexpr int N_MAX = 11;          // M_MAX, 1dmodulesX.f:21
constexpr int NN1 = N_MAX - 3;     // two_phase.f:737
constexpr int NN2 = N_MAX - 1;     // two_phase.f:738
constexpr int GL = 2;              // offset of k = -2 (three ghost cells below k = 1)

struct Col {
    int n = 0, nf = 0;       // flow cells, refined cells
    double L = 1.0, h = 0, hf = 0, ssdzf = 0;
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
    auto zp = [&](int k) { return (k - 1) * c.h + 0.5 * c.h; };
    auto vdz = [&](int k) { return (k == 1 || k == n + 1) ? 0.5 * c.h : c.h; };
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

struct State {
    Col c;
    std::vector<double> psif;    // PSIF(k), k = 1..nf (index k), persistent
    std::vector<double> wo;      // WO(k), flow faces 0..n+1
    double vol_tot_ori = 0.0;
};

}  // namespace

extern "C" {

// Level-set state of one 1-D column, flattened for the C ABI:
//   phi  : nf+7 doubles, ALPHI_EXT(k) for k = -2..nf+4 at [k+2] (band values inside the
//          band, anything outside; TRANSPORT zeroes the outside on entry)
//   layer: nf+7 ints, band layer of refined cell k (0 outside, 1..11)
//   psif : nf+2 doubles, PSIF(k) at [k], k = 1..nf
//   wo   : n+2 doubles, WO(k) at [k], k = 0..n+1
// The band order inside a layer is ascending z in this 1-D form.

static void load(State& s, int n, double L, const double* phi, const int* layer, const double* psif,
                 const double* wo) {
    s.c.init(n, L);
    std::memcpy(s.c.phi.data(), phi, sizeof(double) * (s.c.nf + 7));
    for (int m = 1; m <= N_MAX; ++m)
        for (int k = -2; k <= s.c.nf + 4; ++k)
            if (layer[k + GL] == m) s.c.band[m].push_back(k);
    s.c.rebuild_layer();
    s.psif.assign(psif, psif + s.c.nf + 2);
    s.wo.assign(wo, wo + n + 2);
}

static void store(State& s, double* phi, int* layer, double* psif, double* wo) {
    std::memcpy(phi, s.c.phi.data(), sizeof(double) * (s.c.nf + 7));
    std::memcpy(layer, s.c.layer.data(), sizeof(int) * (s.c.nf + 7));
    std::memcpy(psif, s.psif.data(), sizeof(double) * (s.c.nf + 2));
    std::memcpy(wo, s.wo.data(), sizeof(double) * (s.c.n + 2));
}

// LVSINIT (two_phase.f:116-388, ITRACKING = 2) for the 1-D column.  ASSIGN_LVS (:102-113)
// gives phi = z - z0 + 1e-12 at refined cell centres; cells with |phi| <= CRI =
// 1.2*MAX(SDXF,SDYF,SDZF) (= 0.6: SDXF = SDYF = 1/2) seed the band (the ghosts stay 0:
// no ALPHI_BC here), BAND_GENERATION builds the layers, band cells get the exact distance
// again, PSIF = CAL_PSIF_MTP(1, N_MAX) with the column fill, and the initial vapour
// volume is the sum of (1 - PSIF_MTP) dV over the column (four replicas per level).
int orc_lvs_init(int n, double L, double z0, double* phi, int* layer, double* psif, double* wo,
                 double* vol_tot_ori) {
    State s;
    s.c.init(n, L);
    Col& c = s.c;
    const double cri = 1.2 * std::max(std::max(0.5, 0.5), c.hf);
    auto assign = [&](int k) { return (((k - 1) * c.hf + 0.5 * c.hf) - z0) + 1e-12; };
    c.band.assign(N_MAX + 1, {});
    for (int k = 1; k <= c.nf; ++k) {
        const double a = assign(k);
        if (std::fabs(a) <= cri) {
            c.p(k) = a;
            c.band[1].push_back(k);   // candidates (the reference splits them into layers 1..N)
        }
    }
    if (band_generation(c)) return 2;
    for (int m = 1; m <= N_MAX; ++m)
        for (int k : c.band[m]) c.p(k) = assign(k);
    std::vector<double> ps = cal_psif_mtp(c, 1, N_MAX);
    s.psif.assign(c.nf + 2, 0.0);
    for (int k = 1; k <= c.nf; ++k) {
        double v = ps[k];
        if (v < 1e-5) v = 0.0;
        else if (v > 0.99999) v = 1.0;
        s.psif[k] = v;
    }
    const double dvol = 0.5 * 0.5 * c.hf;
    double vol = 0.0;
    for (int k = 1; k <= c.nf; ++k)
        for (int r = 0; r < 4; ++r) vol = vol + (1.0 - ps[k]) * dvol;
    *vol_tot_ori = vol;
    s.wo.assign(n + 2, 0.0);
    store(s, phi, layer, psif, wo);
    return 0;
}

// TRANSPORT (two_phase.f:701-984) for one column and one RK3 substep, followed by
// GRID_COUPLING (two_phase.f:4863-5118):
//   w       : W(k) on flow faces, k = 0..n+1 (n+2 doubles)
//   mflvs   : interfacial mass flux per refined cell (nf+7, indexed like phi), used when iphs=1
//   first   : 1 on the first substep of the run (VEL_INTP keeps UO = U, :5567-5577)
//   m_step  : time step number M (the MOD(M,50) mass trigger, :903)
//   psi_cn  : out, PSI_CN(k) k = 0..n+1;  psi_zn: out, PSI_ZN(k) k = 0..n+1
//   stats   : out [0] subcycles, [1] DALPHIMAX, [2] DALPHIMIN, [3] IMASS
int orc_lvs_transport(int n, double L, double* phi, int* layer, double* psif, double* wo, const double* w,
                      const double* mflvs, int iphs, double denr, double dtconst, int first, int m_step,
                      double* vol_tot_ori, double vol_tot_iphs, int mglobal, double* psi_cn, double* psi_zn,
                      double* stats) {
    State s;
    load(s, n, L, phi, layer, psif, wo);
    Col& c = s.c;
    const int nf = c.nf;
    // ALPHI_EXT = 0, band values copied in (:750-767)
    std::vector<double> alphi_start(c.phi.size(), 0.0);
    for (size_t q = 0; q < c.phi.size(); ++q) {
        if (c.layer[q] == 0) c.phi[q] = 0.0;
        alphi_start[q] = c.phi[q];
    }
    alphi_bc(c);
    std::vector<double> mf(mflvs, mflvs + nf + 7);
    // VEL_INTP(2, ...): UT = (U + UO)/2, UO = U
    std::vector<double> wt(n + 2);
    if (first) s.wo.assign(w, w + n + 2);
    for (int k = 0; k <= n + 1; ++k) wt[k] = 0.5 * (w[k] + s.wo[k]);
    s.wo.assign(w, w + n + 2);
    std::vector<double> wf(nf + 7, 0.0);
    vel_intp(c, wt, wf);
    double time_tran = 0.0, dmax = 0.0, dmin = 0.0, vo = *vol_tot_ori;
    int imass = 0, isub = 0;
    for (isub = 1; isub <= 10; ++isub) {
        double cflm = 0.0;
        for (int m = 1; m <= NN1; ++m)
            for (int k : c.band[m]) {
                const double cz = std::fabs(0.5 * (wf[k - 1 + GL] + wf[k + GL])) * c.ssdzf;
                const double ci = (0.0 + 0.0) + cz;
                cflm = std::max(cflm, ci);
            }
        double dtlvs;
        if (cflm == 0.0) {
            double uvw = 0.0;
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m]) uvw = uvw + ((0.0 + 0.0) + wf[k + GL]);
            if (uvw == 0.0) {
                if (iphs != 1) { isub = 0; goto done_noupdate; }
                dtlvs = dtconst / 10.0;
            } else {
                dtlvs = 1.0 / cflm;
            }
        } else {
            dtlvs = 1.0 / cflm;
        }
        if (time_tran + dtlvs >= dtconst) dtlvs = dtconst - time_tran;
        time_tran = time_tran + dtlvs;
        {
            std::vector<double> rk3(c.phi);
            transport_rk3(c, dtlvs, wf, mf, alphi_start, iphs, denr);
            transport_rk3(c, dtlvs, wf, mf, alphi_start, iphs, denr);
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m]) c.p(k) = 0.75 * rk3[k + GL] + 0.25 * c.p(k);
            transport_rk3(c, dtlvs, wf, mf, alphi_start, iphs, denr);
            for (int m = 1; m <= NN1; ++m)
                for (int k : c.band[m]) c.p(k) = 1.0 / 3.0 * rk3[k + GL] + 2.0 / 3.0 * c.p(k);
        }
        rein_trigger(c, dmax, dmin);
        imass = (dmax > 2.0 || dmin < 1e-4) ? 1 : 0;
        if (iphs == 1) {
            reinitialization(c, NN2);
            if (m_step % 50 == 0) imass = 1;
        }
        if (dmax > 2.0 || dmin < 1e-4 || imass == 1) {
            if (mglobal == 1 && imass == 1) global_mass_correction(c, vo, vol_tot_iphs, iphs);
            alphi_bc(c);
            if (band_generation(c)) return 2;   // LICA_BAND_OVERFLOW; outputs untouched
            alphi_bc(c);
            reinitialization(c, NN2);
        }
        alphi_bc(c);
        if (time_tran == dtconst) break;
        if (dmax > 2.0 || dmin < 1e-4) vel_intp(c, wt, wf);
    }
    if (isub > 10) isub = 10;
    {
        // CAL_PSIF(0, ...): PSIF = PSIF_MTP on layers <= NN1, then the snap (:2600-2680)
        std::vector<double> ps = cal_psif_mtp(c, 0);
        for (int m = 1; m <= NN1; ++m)
            for (int k : c.band[m]) s.psif[k] = ps[k];
        for (int k = 1; k <= nf; ++k) {
            if (s.psif[k] < 1e-5) s.psif[k] = 0.0;
            else if (s.psif[k] > 0.99999) s.psif[k] = 1.0;
        }
    }
    // band values stored; the final GLOBAL_MASS_CORRECTION only updates the target volume
    if (imass == 0 && iphs == 1) vo = vol_tot_iphs;
    *vol_tot_ori = vo;
    {
        // GRID_COUPLING(0): flow cells touched by a band cell (layers <= NN1)
        std::vector<int> mask(n + 2, 0);
        for (int m = 1; m <= NN1; ++m)
            for (int k : c.band[m])
                if (k >= 1 && k <= nf) mask[(k + 1) / 2] = 1;   // KCOUMP_VEL
        for (int k = 2; k <= n; ++k)
            if (mask[k]) psi_zn[k] = 0.5 * (s.psif[2 * k - 2] + s.psif[2 * k - 1]);
        for (int k = 1; k <= n; ++k) {
            if (psi_zn[k] < 1e-3) psi_zn[k] = 0.0;
            else if (psi_zn[k] > 0.999) psi_zn[k] = 1.0;
        }
        for (int k = 1; k <= n; ++k)
            if (mask[k]) psi_cn[k] = 0.5 * (s.psif[2 * k - 1] + s.psif[2 * k]);
        for (int k = 1; k <= n; ++k) {
            if (psi_cn[k] < 1e-3) psi_cn[k] = 0.0;
            else if (psi_cn[k] > 0.999) psi_cn[k] = 1.0;
        }
        psi_cn[0] = psi_cn[1];
        psi_cn[n + 1] = psi_cn[n];
    }
    stats[0] = isub;
    stats[1] = dmax;
    stats[2] = dmin;
    stats[3] = imass;
    store(s, phi, layer, psif, wo);
    return 0;
done_noupdate:
    *vol_tot_ori = vo;
    stats[0] = 0;
    store(s, phi, layer, psif, wo);
    return 0;
}

// Unit entry points on one column (tests): ALPHI_BC, BAND_GENERATION and
// REINITIALIZATION(NN1, NN2, ilimit) on phi/layer.
int orc_lvs_alphi_bc(int n, double L, double* phi) {
    Col c;
    c.init(n, L);
    std::memcpy(c.phi.data(), phi, sizeof(double) * (c.nf + 7));
    alphi_bc(c);
    std::memcpy(phi, c.phi.data(), sizeof(double) * (c.nf + 7));
    return 0;
}

int orc_lvs_band(int n, double L, double* phi, int* layer) {
    State s;
    std::vector<double> dummy_psif(2 * n + 2, 0.0), dummy_wo(n + 2, 0.0);
    load(s, n, L, phi, layer, dummy_psif.data(), dummy_wo.data());
    if (band_generation(s.c)) return 2;
    std::memcpy(phi, s.c.phi.data(), sizeof(double) * (s.c.nf + 7));
    std::memcpy(layer, s.c.layer.data(), sizeof(int) * (s.c.nf + 7));
    return 0;
}

int orc_lvs_reinit(int n, double L, double* phi, const int* layer, int ilimit) {
    State s;
    std::vector<double> dummy_psif(2 * n + 2, 0.0), dummy_wo(n + 2, 0.0);
    load(s, n, L, phi, layer, dummy_psif.data(), dummy_wo.data());
    reinitialization(s.c, ilimit);
    std::memcpy(phi, s.c.phi.data(), sizeof(double) * (s.c.nf + 7));
    return 0;
}

}  // extern "C"
