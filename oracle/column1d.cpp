// ORACLE (test infrastructure only) -- CPU restatement of one time step of the
// reference's 1-D boiling column: the RK3 flow / energy / phase-change step of MAIN
// (1d.f:190-250) on the 1 x 1 x n flow column with its 2 x 2 x 2n refined level-set grid.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// Parity status: unpinned against the reference (no Fortran compiler here and the
// reference as shipped does not compile: PASSIVE_SCALAR uses names it does not declare,
// LHSPS2 is undefined).  Each routine follows the cited Fortran statement by statement in
// its 1-D form.  Exact 1-D reductions: with IPX = IPY = 1 and N1M = N2M = 1 every x/y
// neighbour of the flow cell is the cell itself (IPV(1) = IMV(1) = 1, 1d.f:4682-4708), and
// U = V = 0 (BC, 1d.f:1829-1850), so every x/y convection, diffusion and gradient term is
// exactly zero; the 2 x 2 refined replicas carry equal values.
// Documented substitutions (the reference gives no defined behaviour):
//   * LHSPS2 (called at 1d.f:3665, defined nowhere; chphase.f:32 is an empty LSHPS2): the
//     implicit energy solve of LHSPS (1d.f:4380-4497) is used, with PSI_C and DF_C from
//     CAL_CONTINUITY (PASSIVE_SCALAR references them without having them in scope);
//   * step 1 (M = 1) runs the non-phase-change energy path (1d.f:3669-3684); TEMP_GRAD is
//     not called, so MFLVS, SFGAS, SFGAS2 and IMASK_PH are zero during that step;
//   * TEMP_EXTP's retry loop (chphase.f:650-790, "GOTO 998/1002" with a halved step, no
//     limit) stops after 40 halvings and reports non-convergence;
//   * the ghosts K = 0 and n+1 of DTEMPN (a TEMP_EXTP local never set there) read 0.
#include "lvs1d_core.hpp"

#include <cstdio>

extern "C" int orc_lvs_transport(int n, double L, double* phi, int* layer, double* psif, double* wo, const double* w,
                                 const double* mflvs, int iphs, double denr, double dtconst, int first, int m_step,
                                 double* vol_tot_ori, double vol_tot_iphs, int mglobal, double* psi_cn,
                                 double* psi_zn, double* stats);
extern "C" int orc_lvs_init(int n, double L, double z0, double* phi, int* layer, double* psif, double* wo,
                            double* vol_tot_ori);
extern "C" int orc_lvs_transport_geo(int n, double L, double* phi, int* layer, double* psif, double* wo,
                                     const double* w, const double* mflvs, int iphs, double denr, double dtconst,
                                     int first, int m_step, double* vol_tot_ori, double vol_tot_iphs, int mglobal,
                                     double* psi_cn, double* psi_zn, double* stats, const void* geo);

namespace {

// place of the latest VOL_TOT_MFDOT on this thread (0 until one runs in a step)
thread_local double g_place = 0.0;

// lica.in inputs of the two-phase / heat block (INPUT_SIMULATION 1d.f:346-379).
struct ColProps {
    double re, visr, denr, weber, fr, prm, scr, tcr, t_sat, jakob, cflmax, dt0;
    int32_t iphs, mglobal;
};

// Derived constants, 1d.f:437-489.
struct Phys {
    double rei, denm, denp, den_diff, vism, visp, denscm, denscp, densc_diff, tcm, tcp, tc_diff, prai, surf,
        gravity, time_st, time_gv, denr, re, prm, ja, t_sat, cflmax;
    int iphs, mglobal;
    explicit Phys(const ColProps& p) {
        const double pi = std::acos(-1.0);
        re = p.re;
        rei = 1.0 / re;
        denm = 1.0;
        denp = p.denr;
        den_diff = denp - denm;
        vism = 1.0 * rei;
        visp = p.visr * rei;
        denscm = denm * 1.0;
        denscp = denscm * (p.denr * p.scr);
        densc_diff = denscp - denscm;
        tcm = 1.0;
        tcp = p.tcr;
        tc_diff = tcp - tcm;
        prm = p.prm;
        prai = 1.0 / p.prm;
        surf = (p.weber == 0.0) ? 0.0 : 1.0 / p.weber;
        gravity = (p.fr == 0.0) ? 0.0 : 1.0 / (p.fr * p.fr);
        time_st = surf * pi / (denm + denp);
        time_gv = den_diff / (denm + denp) * gravity / pi;
        denr = p.denr;
        ja = p.jakob;
        t_sat = p.t_sat;
        cflmax = p.cflmax;
        iphs = p.iphs;
        mglobal = p.mglobal;
    }
};

// RK3COEF, 1d.f:1310-1322.
const double GAMMA[4] = {0.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double RO[4] = {0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0};

// Flat column state (C ABI layout; flow arrays k = 0..n+1 at [k]).
struct ColView {
    int n;
    double L;
    double *w, *p, *t, *psi_cn, *psi_zn;
    double *phi;       // nf+7, ALPHI band values at [k+2]
    int* layer;        // nf+7
    double *psif, *wo; // nf+2, n+2
    double *mflvs;     // nf+7, MFLVS of the last TEMP_GRAD (band layers 1..6)
    double *sfgas, *sfgas2;  // nf+2
    int* imask;        // n+2, IMASK_PH
    double* scal;      // [0] DT, [1] TIME, [2] M, [3] VOL_TOT_ORI, [4] VOL_TOT_IPHS
};

struct Geo {
    int n, nf;
    double h, hf;
    const ColGeo* cg = nullptr;   // null: the uniform column
    explicit Geo(int n_, double L, const ColGeo* cg_ = nullptr)
        : n(n_), nf(2 * n_), h(L / n_), hf(L / (2 * n_)), cg(cg_) {}
    double sdz(int k) const { return cg ? cg->sdz[k] : ((k >= 1 && k <= n) ? h : 0.0); }
    double ssdz(int k) const { return cg ? cg->ssdz[k] : 1.0 / h; }                 // SSDZ(1..n)
    double vdz(int k) const { return cg ? cg->vdz[k] : ((k == 1 || k == n + 1) ? 0.5 * h : h); }
    double vvdz(int k) const { return cg ? cg->vvdz[k] : 1.0 / vdz(k); }
    double z(int k) const { return cg ? cg->z[k] : grid_z(h, k); }
    double zp(int k) const { return cg ? cg->zp[k] : grid_zp(h, n, k); }
    double zf(int k) const { return grid_zf(hf, k); }
    double zpf(int k) const { return grid_zf(hf, k) + 0.5 * hf; }
    // GEOM_COUPLING's refined faces (uniform column: face K is refined face 2K-1, centre K
    // refined face 2K)
    int kcou1(int k) const { return cg ? cg->kcou1[k + 1] : 2 * k - 2; }
    int kcou2(int k) const { return cg ? cg->kcou2[k + 1] : 2 * k - 1; }
    int kcoump1(int k) const { return cg ? cg->kcoump1[k + 1] : 2 * k - 1; }
    int kcoump2(int k) const { return cg ? cg->kcoump2[k + 1] : 2 * k; }
    int kcoump_vel(int k) const { return cg ? cg->kcoump_vel[k] : ::kcoump_vel(h, hf, n, k); }
    // LHSINIT, 1d.f:1927-1990
    double akw(int k) const { return -vvdz(k) * ssdz(k - 1); }
    double ckw(int k) const { return -vvdz(k) * ssdz(k); }
    double akuv(int k) const { return -vvdz(k) * ssdz(k); }
    double ckuv(int k) const { return -vvdz(k + 1) * ssdz(k); }
};

// Thomas algorithm of TRDIAG3 (1d.f:3783-3811) for one line, unknowns l1..l2 of x[].
void thomas(const std::vector<double>& a, const std::vector<double>& b, const std::vector<double>& c,
            std::vector<double>& r, int l1, int l2) {
    std::vector<double> gam(r.size(), 0.0), uu(r.size(), 0.0);
    double bet = 1.0 / b[l1];
    uu[l1] = r[l1] * bet;
    for (int j = l1 + 1; j <= l2; ++j) {
        gam[j] = c[j - 1] * bet;
        bet = 1.0 / (b[j] - a[j] * gam[j]);
        uu[j] = (r[j] - a[j] * uu[j - 1]) * bet;
    }
    for (int j = l2 - 1; j >= l1; --j) uu[j] = uu[j] - gam[j + 1] * uu[j + 1];
    for (int j = l1; j <= l2; ++j) r[j] = uu[j];
}

// DETERMINE_DT + CFL, 1d.f:683-817, 1325-1373 (N1M = 1 branch; SDY = 1).
void determine_dt(const Geo& g, const Phys& ph, const ColView& s, double& cflm_out) {
    const int n = g.n;
    double& dt = s.scal[0];
    const double dt_old = dt;
    double dt_source;
    if (ph.time_st == 0.0) {
        dt_source = 1000000.0;
    } else {
        dt_source = 1000.0;
        for (int k = 1; k <= n; ++k)
            if (std::fabs(s.psi_cn[k] - 0.5) < 0.5) {
                const double dx1 = std::min(1.0, g.sdz(k));
                const double t1 = 0.5 * dx1 / std::sqrt(ph.time_st / dx1 + ph.time_gv * dx1);
                const double dx2 = std::max(1.0, g.sdz(k));
                const double t2 = 0.5 * dx2 / std::sqrt(ph.time_st / dx2 + ph.time_gv * dx2);
                dt_source = std::min(dt_source, std::min(t1, t2));
            }
    }
    double cflm = 0.0;
    for (int k = 1; k <= n; ++k) {
        const double c3 = std::fabs(s.w[k] + s.w[k + 1]) * g.ssdz(k);
        const double cfli = 0.5 * ((0.0 + 0.0) + c3) * dt;
        cflm = std::max(cfli, cflm);
    }
    cflm_out = cflm;
    const double cfl_surf = dt / dt_source;
    const double cfl_sum = 0.5 * (cflm + std::sqrt(cflm * cflm + 4.0 * cfl_surf));
    dt = dt * ph.cflmax / cfl_sum;
    if (dt / dt_old > 2.0) dt = dt_old * 1.2;
}

struct Work {
    std::vector<double> df_z, vf_z, psi_z, df_c, psi_c, denf_z, denf_zi, denf_c, rhs1, rk3zo, rhsps, divgsum;
    std::vector<int> region;  // index k+1, k = -1..n+2
    explicit Work(int n)
        : df_z(n + 2), vf_z(n + 2), psi_z(n + 2), df_c(n + 2), psi_c(n + 2), denf_z(n + 2), denf_zi(n + 2),
          denf_c(n + 2), rhs1(n + 2), rk3zo(n + 2), rhsps(n + 2), divgsum(n + 2), region(n + 4) {}
    int& reg(int k) { return region[k + 1]; }
};

// REGION of CAL_CONTINUITY / CAL_CONTINUITY2 (1d.f:2038-2056, 3030-3048), serial order.
void make_region(const Geo& g, const ColView& s, Work& wk) {
    std::fill(wk.region.begin(), wk.region.end(), 0);
    for (int k = 1; k <= g.n; ++k) {
        if ((s.psi_cn[k + 1] - s.psi_cn[k] != 0.0) || (s.psi_cn[k] - s.psi_cn[k - 1] != 0.0)) {
            for (int k2 = k - 2; k2 <= k + 2; ++k2) wk.reg(k2) = 2;
        } else if (s.psi_cn[k] == 1.0) {
            if (wk.reg(k) != 2) wk.reg(k) = 1;
        }
    }
}

// CAL_CONTINUITY (1d.f:1994-2068) = REGION + CONTI_Z (2071-2214) + CONTI_C (2217-2346),
// with PSIFACE_Z / PSIFACE_C (2349-2550) and INTER_PSI_FACE (2552-2958).
void cal_continuity(const Geo& g, const Phys& ph, const ColView& s, double dtconst, Work& wk) {
    const int n = g.n, nf = g.nf;
    make_region(g, s, wk);
    const double* w = s.w;
    // CONTI_Z (KBG = 2)
    std::fill(wk.df_z.begin(), wk.df_z.end(), 0.0);
    auto psiface_z = [&](int k, double uu) {
        double z1, z2;
        int k1, k2;
        if (uu >= 0.0) {
            z1 = g.zp(k) - uu * dtconst;
            z2 = g.zp(k);
            k1 = g.kcoump2(k - 1);
            k2 = g.kcoump1(k);
        } else {
            z1 = g.zp(k);
            z2 = g.zp(k) - uu * dtconst;
            k1 = g.kcoump2(k);
            k2 = g.kcoump1(k + 1);
        }
        return box_mean(s.psif, nf, k1, k2, z1, z2, g.hf);
    };
    for (int k = 2; k <= n; ++k) {
        if (wk.reg(k) == 0) {
            wk.vf_z[k] = ph.vism;
            wk.vf_z[k - 1] = ph.vism;
            wk.df_z[k] = ph.denm;
            wk.df_z[k - 1] = ph.denm;
            wk.psi_z[k] = s.psi_zn[k];
        } else if (wk.reg(k) == 1) {
            wk.vf_z[k] = ph.visp;
            wk.vf_z[k - 1] = ph.visp;
            wk.df_z[k] = ph.denp;
            wk.df_z[k - 1] = ph.denp;
            wk.psi_z[k] = s.psi_zn[k];
        } else {
            const double wt = 0.5 * (w[k + 1] + w[k]);
            const double wb = 0.5 * (w[k] + w[k - 1]);
            if (wk.df_z[k] == 0.0) {
                const double ps = (std::fabs(wt) <= 1e-8) ? 0.5 * (s.psi_zn[k] + s.psi_zn[k + 1]) : psiface_z(k, wt);
                wk.vf_z[k] = ph.vism + (ph.visp - ph.vism) * ps;
                wk.df_z[k] = ph.denm + ph.den_diff * ps;
            }
            if (wk.df_z[k - 1] == 0.0) {
                const double ps =
                    (std::fabs(wb) <= 1e-8) ? 0.5 * (s.psi_zn[k] + s.psi_zn[k - 1]) : psiface_z(k - 1, wb);
                wk.vf_z[k - 1] = ph.vism + (ph.visp - ph.vism) * ps;
                wk.df_z[k - 1] = ph.denm + ph.den_diff * ps;
            }
            const double flux_z = (wk.df_z[k] * wt - wk.df_z[k - 1] * wb) * g.vvdz(k);
            const double den_zn = ph.denm + ph.den_diff * s.psi_zn[k];
            const double den_z = den_zn - dtconst * flux_z;
            wk.psi_z[k] = (den_z - ph.denm) / ph.den_diff;
        }
    }
    for (int k = 2; k <= n; ++k) {
        if (wk.psi_z[k] > 1.0) wk.psi_z[k] = 1.0;
        else if (wk.psi_z[k] < 0.0) wk.psi_z[k] = 0.0;
    }
    wk.psi_z[1] = wk.psi_z[2];
    wk.psi_z[n + 1] = wk.psi_z[n];
    // CONTI_C
    std::fill(wk.df_c.begin(), wk.df_c.end(), 0.0);
    auto psiface_c = [&](int k, double uu) {
        double z1, z2;
        int k1, k2;
        if (uu >= 0.0) {
            z1 = g.z(k + 1) - uu * dtconst;
            z2 = g.z(k + 1);
            k1 = g.kcou2(k);
            k2 = g.kcou1(k + 1);
        } else {
            z1 = g.z(k + 1);
            z2 = g.z(k + 1) - uu * dtconst;
            k1 = g.kcou2(k + 1);
            k2 = g.kcou1(k + 2);
        }
        return box_mean(s.psif, nf, k1, k2, z1, z2, g.hf);
    };
    for (int k = 1; k <= n; ++k) {
        if (wk.reg(k) == 0) {
            wk.psi_c[k] = s.psi_cn[k];
            wk.df_c[k] = ph.denm;
            wk.df_c[k - 1] = ph.denm;
        } else if (wk.reg(k) == 1) {
            wk.psi_c[k] = s.psi_cn[k];
            wk.df_c[k] = ph.denp;
            wk.df_c[k - 1] = ph.denp;
        } else {
            const double wt = w[k + 1], wb = w[k];
            if (wk.df_c[k] == 0.0) {
                const double ps = (std::fabs(wt) <= 1e-8) ? s.psi_cn[k + 1] : psiface_c(k, wt);
                wk.df_c[k] = ph.denm + ph.den_diff * ps;
            }
            if (wk.df_c[k - 1] == 0.0) {
                const double ps = (std::fabs(wb) <= 1e-8) ? s.psi_cn[k] : psiface_c(k - 1, wb);
                wk.df_c[k - 1] = ph.denm + ph.den_diff * ps;
            }
            const double flux_z = (wk.df_c[k] * wt - wk.df_c[k - 1] * wb) * g.ssdz(k);
            const double den_cn = ph.denm + ph.den_diff * s.psi_cn[k];
            const double den_c = den_cn - dtconst * flux_z;
            wk.psi_c[k] = (den_c - ph.denm) / ph.den_diff;
        }
    }
    for (int k = 1; k <= n; ++k) {
        if (wk.psi_c[k] > 1.0) wk.psi_c[k] = 1.0;
        else if (wk.psi_c[k] < 0.0) wk.psi_c[k] = 0.0;
    }
    wk.psi_c[1] = wk.psi_c[2];
    wk.psi_c[n + 1] = wk.psi_c[n];
}

// CAL_CONT_BC, 1d.f:2961-3003.
void cal_cont_bc(const Geo& g, const Phys& ph, Work& wk) {
    const int n = g.n;
    for (int k = 1; k <= n; ++k) {
        wk.denf_z[k] = ph.denm + ph.den_diff * wk.psi_z[k];
        wk.denf_zi[k] = 1.0 / wk.denf_z[k];
    }
    wk.denf_z[n + 1] = wk.denf_z[n];
    wk.denf_zi[n + 1] = wk.denf_zi[n];
    wk.denf_z[0] = wk.denf_z[1];
    wk.denf_zi[0] = wk.denf_zi[1];
    for (int k = 1; k <= n; ++k) wk.denf_c[k] = ph.denm + ph.den_diff * wk.psi_c[k];
}

// LHSPS, 1d.f:4380-4497: implicit z diffusion of T (one line), T += solution, T(0) = 0,
// T(n) = 1, T(n+1) = T(n).
void lhsps(const Geo& g, const Phys& ph, const ColView& s, double alpha, Work& wk) {
    const int n = g.n;
    const double dt = s.scal[0];
    const double den_diffi = (ph.den_diff == 0.0) ? 1.0 : 1.0 / ph.den_diff;
    const double acops = alpha * dt / (ph.re * ph.prm);
    std::vector<double> ak(n + 2), bk(n + 2), ck(n + 2), gk(n + 2);
    for (int k = 1; k <= n; ++k) {
        const double denscf = ph.denscm + ph.densc_diff * wk.psi_c[k];
        const double coef = acops / denscf;
        double psi_tmp = (wk.df_c[k - 1] - ph.denm) * den_diffi;
        const double tcb = ph.tcm + ph.tc_diff * psi_tmp;
        psi_tmp = (wk.df_c[k] - ph.denm) * den_diffi;
        const double tct = ph.tcm + ph.tc_diff * psi_tmp;
        ak[k] = coef * tcb * g.akuv(k);
        ck[k] = coef * tct * g.ckuv(k);
        bk[k] = 1.0 - (ak[k] + ck[k]);
        gk[k] = wk.rhsps[k];
        if (std::fabs(s.psi_cn[k] - 0.5) != 0.5) {
            if (s.psi_cn[k] <= 0.5) ck[k] = 0.0;
            else if (s.psi_cn[k] > 0.5) ak[k] = 0.0;
        }
    }
    thomas(ak, bk, ck, gk, 1, n);
    for (int k = 1; k <= n; ++k) {
        wk.rhsps[k] = gk[k];
        s.t[k] = gk[k] + s.t[k];
    }
    s.t[0] = 0.0;
    s.t[n] = 1.0;
    s.t[n + 1] = s.t[n];
}

// Band lists (ascending within a layer) and ALPHI_EXT of TEMP_GRAD (chphase.f:121-139):
// zero everywhere, band values on the band, no ghost boundary condition.
void load_band(const Geo& g, double L, const ColView& s, Col& c) {
    c.init(g.n, L);
    c.cg = g.cg;
    for (int k = -2; k <= g.nf + 4; ++k) {
        const int m = s.layer[k + GL];
        c.phi[k + GL] = (m >= 1 && m <= N_MAX) ? s.phi[k + GL] : 0.0;
    }
    for (int m = 1; m <= N_MAX; ++m)
        for (int k = -2; k <= g.nf + 4; ++k)
            if (s.layer[k + GL] == m) c.band[m].push_back(k);
    c.rebuild_layer();
}

// PHINSINTP, chphase.f:1258-1325 (1-D): trilinear interpolation of ALPHI_EXT to the flow
// centre of cell kk from refined cells K1 = 2kk-1, K2 = 2kk (the x/y weights act on equal
// replicas); zero if any stencil value is zero; IC keeps its previous value when the
// result is exactly zero.
double phinsintp(const Geo& g, const Col& c, int kk, int& ic) {
    const int k1 = g.kcou2(kk), k2 = g.kcoump2(kk);   // PHINSINTP's K1 = KCOU2(KO), K2 = KCOUMP2(KO)
    const double zd = (k1 == k2) ? 0.0 : (g.zp(kk) - g.zpf(k1)) / (g.zpf(k2) - g.zpf(k1));
    const double a1 = const_cast<Col&>(c).p(k1), a2 = const_cast<Col&>(c).p(k2);
    const double c00 = a1 * (1.0 - 0.5) + a1 * 0.5;
    const double c01 = a2 * (1.0 - 0.5) + a2 * 0.5;
    const double c0 = c00 * (1.0 - 0.5) + c00 * 0.5;
    const double c1 = c01 * (1.0 - 0.5) + c01 * 0.5;
    double nsphi = c0 * (1.0 - zd) + c1 * zd;
    if (nsphi > 0.0) ic = 1;
    if (nsphi < 0.0) ic = 0;
    if (a1 == 0.0 || a2 == 0.0) nsphi = 0.0;
    return nsphi;
}

// TEMP_EXTP_RK3, chphase.f:806-956 (1-D): one Godunov upwind step of the extension PDE on
// the flow grid.  nd = 0 extends DTEMPN (tempo is DTEMPN itself), nd = 1 extends the phase
// temperature with DTEMPN as the source.
void temp_extp_rk3(const Geo& g, std::vector<double>& tempo, const std::vector<double>& psih,
                   const std::vector<double>& nphi, int im, double redtl, int nd, std::vector<double>& dtempn) {
    const int n = g.n;
    const double sm_grid = std::min(std::min(1.0, 1.0), 2.0 * g.hf);
    std::vector<double> temp_new(tempo);
    for (int k = 1; k <= n; ++k) {
        if (nphi[k] == 0.0) continue;
        double dpz;
        if (nphi[k - 1] == 0.0) dpz = (nphi[k + 1] - nphi[k]) * g.vvdz(k + 1);
        else if (nphi[k + 1] == 0.0) dpz = (nphi[k] - nphi[k - 1]) * g.vvdz(k);
        else dpz = 0.5 * (nphi[k + 1] - nphi[k - 1]) * g.vvdz(k);
        const double dalphi = (0.0 + 0.0) + dpz * dpz;   // DPX = DPY = 0 (periodic self-neighbours)
        if (dalphi == 0.0) continue;
        double nz = 1.0;
        const double apzm = (tempo[k] - tempo[k - 1]) * g.vvdz(k);
        const double apzp = (tempo[k + 1] - tempo[k]) * g.vvdz(k);
        if (im == 1) nz = (-1.0) * nz;
        const double ax = 0.0, ay = 0.0;
        const double az = std::min(nz, 0.0) * apzp + std::max(nz, 0.0) * apzm;
        double drhs;
        if (im == 1) {
            drhs = (ax + ay + az) + nd * dtempn[k];
            temp_new[k] = tempo[k] - redtl * drhs * (1 - psih[k]);
        } else {
            drhs = (ax + ay + az) - nd * dtempn[k];
            temp_new[k] = tempo[k] - redtl * drhs * psih[k];
        }
        if (nd == 0 && std::fabs(nphi[k]) <= sm_grid) {
            drhs = (ax + ay + az);
            temp_new[k] = tempo[k] - redtl * drhs;
        }
    }
    for (int k = 1; k <= n; ++k) {
        tempo[k] = temp_new[k];
        if (nd == 0) dtempn[k] = tempo[k];
    }
}

constexpr int kMaxHalvings = 40;

// TEMP_EXTP, chphase.f:467-805 (1-D).  temp[im][k], k = 0..n+1.  Returns the number of
// pseudo-time iterations, or -1 if a phase did not converge within kMaxHalvings retries.
int temp_extp(const Geo& g, const Phys& ph, const ColView& s, std::vector<double> temp[2],
              const std::vector<double>& psih, const std::vector<double>& nphi) {
    const int n = g.n;
    const double sm_grid = std::min(std::min(2.0 * 0.5, 2.0 * 0.5), 2.0 * g.hf);
    const double eps = 1e-4;
    int total = 0;
    for (int im = 0; im <= 1; ++im) {
        std::vector<double> dtempn(n + 2, 0.0), dtempn_rk3(n + 2, 0.0);
        std::vector<double>& tm = temp[im];
        for (int k = 1; k <= n; ++k) {
            dtempn[k] = 0.0;
            const bool ca = ((std::fabs(nphi[k]) > 1.5 * sm_grid) && (nphi[k] != 0.0)) ||
                            ((std::fabs(s.psi_cn[k] - 0.5) == 0.5) && (nphi[k] != 0.0));
            if (ca) {
                double dpz, dtdz;
                if (nphi[k - 1] == 0.0) {
                    dpz = (nphi[k + 1] - nphi[k]) * g.vvdz(k + 1);
                    dtdz = (tm[k + 1] - tm[k]) * g.vvdz(k + 1);
                } else if (nphi[k + 1] == 0.0) {
                    dpz = (nphi[k] - nphi[k - 1]) * g.vvdz(k);
                    dtdz = (tm[k] - tm[k - 1]) * g.vvdz(k);
                } else {
                    dpz = 0.5 * (nphi[k + 1] - nphi[k - 1]) * g.vvdz(k);
                    dtdz = 0.5 * (tm[k + 1] - tm[k - 1]) * g.vvdz(k);
                }
                const double dalphi = (0.0 + 0.0) + dpz * dpz;
                if (dalphi != 0.0) {
                    const double nz = 1.0;
                    if (im == 1) dtempn[k] = (0.0 + 0.0) + nz * dtdz * psih[k];
                    else dtempn[k] = (0.0 + 0.0) + nz * dtdz * (1 - psih[k]);
                }
            } else if (((std::fabs(nphi[k]) <= 1.5 * sm_grid) || (std::fabs(s.psi_cn[k] - 0.5) != 0.5)) &&
                       ((nphi[k] != 1e-7) && (nphi[k] != 0.0))) {
                if (im == 1) dtempn[k] = (tm[k] - ph.t_sat) / nphi[k] * psih[k];
                else dtempn[k] = (tm[k] - ph.t_sat) / nphi[k] * (1.0 - psih[k]);
            }
        }
        // extension of the normal gradient (nd = 0)
        double redtl = 0.2 * sm_grid;
        bool conv = false;
        for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
            for (int it = 1; it <= 100; ++it) {
                ++total;
                for (int k = 1; k <= n; ++k) dtempn_rk3[k] = dtempn[k];
                temp_extp_rk3(g, dtempn, psih, nphi, im, redtl, 0, dtempn);
                temp_extp_rk3(g, dtempn, psih, nphi, im, redtl, 0, dtempn);
                for (int k = 1; k <= n; ++k) dtempn[k] = 0.75 * dtempn_rk3[k] + 0.25 * dtempn[k];
                temp_extp_rk3(g, dtempn, psih, nphi, im, redtl, 0, dtempn);
                for (int k = 1; k <= n; ++k) dtempn[k] = 1.0 / 3.0 * dtempn_rk3[k] + 2.0 / 3.0 * dtempn[k];
                double rat = 0.0;
                for (int k = 1; k <= n; ++k) {
                    if (dtempn_rk3[k] != 0.0) rat = std::max(std::fabs(dtempn[k] / dtempn_rk3[k] - 1.0), rat);
                    else if (dtempn[k] != 0.0) rat = std::max(std::fabs(dtempn_rk3[k] / dtempn[k] - 1.0), rat);
                }
                if (std::fabs(rat) < eps) {
                    conv = true;
                    break;
                }
            }
            if (!conv) redtl = 0.5 * redtl;
        }
        if (!conv) return -1;
        // extension of the phase temperature (nd = 1)
        redtl = 0.2 * sm_grid;
        conv = false;
        std::vector<double> temp_rk3(n + 2), tempo(n + 2);
        for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
            for (int it = 1; it <= 100; ++it) {
                ++total;
                for (int k = 0; k <= n + 1; ++k) {
                    temp_rk3[k] = tm[k];
                    tempo[k] = tm[k];
                }
                temp_extp_rk3(g, tempo, psih, nphi, im, redtl, 1, dtempn);
                temp_extp_rk3(g, tempo, psih, nphi, im, redtl, 1, dtempn);
                for (int k = 1; k <= n; ++k) tempo[k] = 0.75 * temp_rk3[k] + 0.25 * tempo[k];
                temp_extp_rk3(g, tempo, psih, nphi, im, redtl, 1, dtempn);
                for (int k = 1; k <= n; ++k) {
                    tempo[k] = 1.0 / 3.0 * temp_rk3[k] + 2.0 / 3.0 * tempo[k];
                    tm[k] = tempo[k];
                }
                double rat = 0.0;
                for (int k = 1; k <= n; ++k)
                    if (temp_rk3[k] != 0.0) rat = std::max(std::fabs(tm[k] / temp_rk3[k] - 1.0), rat);
                if (std::fabs(rat) < eps) {
                    conv = true;
                    break;
                }
            }
            if (!conv) redtl = 0.5 * redtl;
        }
        if (!conv) return -1;
    }
    return total;
}

// TEMP_GRAD (chphase.f:55-368) with TEMPASSIGN, TEMP_EXTP, TF_GRAD (959-1159),
// VOL_TOT_MFDOT (1328-1493) and CAL_PSI_TMP(1) (two_phase.f:3167-3316), 1-D.  Writes
// MFLVS, SFGAS, SFGAS2, VOL_TOT_IPHS and IMASK_PH.  Returns the TEMP_EXTP iteration count
// or -1.
int temp_grad(const Geo& g, double L, const Phys& ph, const ColView& s, double dtconst) {
    const int n = g.n, nf = g.nf;
    for (int k = 0; k < nf + 7; ++k) s.mflvs[k] = 0.0;
    for (int k = 0; k <= n + 1; ++k) s.imask[k] = 0;
    std::vector<double> temp[2] = {std::vector<double>(s.t, s.t + n + 2), std::vector<double>(s.t, s.t + n + 2)};
    std::vector<double> nphi(n + 2, 0.0), psih(n + 2, 0.0);
    Col c;
    load_band(g, L, s, c);
    // (1) phase and distance of the flow cells near the band (:147-186)
    int ic = 0;
    for (int m = 1; m <= NN2; ++m)
        for (int k : c.band[m]) {
            const int kk = g.kcoump_vel(k);
            if (nphi[kk] == 0.0) {
                const double nsphi = phinsintp(g, c, kk, ic);
                nphi[kk] = 1e-7;
                nphi[kk] = nsphi;
                if (std::fabs(s.psi_cn[kk] - 0.5) != 0.5) psih[kk] = (double)ic;
                else psih[kk] = s.psi_cn[kk];
            }
        }
    for (int k : c.band[N_MAX]) {
        const int kk = g.kcoump_vel(k);
        const double dx = 0.25, dy = 0.25;            // XPF - XP of either replica, squared below
        const double dz = g.zpf(k) - g.zp(kk);
        const double pre = c.p(k) + std::sqrt(dx * dx + dy * dy + dz * dz);
        for (int rep = 0; rep < 4; ++rep) {
            nphi[kk] = std::min(nphi[kk], pre);
            psih[kk] = s.psi_cn[kk];
        }
    }
    // (2) TEMP_EXTP
    const int iters = temp_extp(g, ph, s, temp, psih, nphi);
    if (iters < 0) return -1;
    // (3) TF by TEMPASSIGN on layers 1..NN1 (chphase.f:372-463)
    std::vector<double> tf0(nf + 7, 0.0), tf1(nf + 7, 0.0);
    for (int m = 1; m <= NN1; ++m)
        for (int k : c.band[m]) {
            const int kk = g.kcoump_vel(k);
            int kk1, kk2;
            double zd;
            if (g.zp(kk) > g.zpf(k)) {
                kk1 = kk - 1;
                kk2 = kk;
                zd = (kk1 == kk2) ? 0.0 : (g.zpf(k) - (g.zp(kk) - g.vdz(kk))) / (g.zp(kk2) - g.zp(kk1));
            } else {
                kk1 = kk;
                kk2 = kk + 1;
                zd = (kk1 == kk2) ? 0.0 : (g.zpf(k) - g.zp(kk1)) / (g.zp(kk2) - g.zp(kk1));
            }
            for (int im = 0; im <= 1; ++im) {
                const double c0 = temp[im][kk], c1 = temp[im][kk2];
                const double v = c0 * (1.0 - zd) + c1 * zd;
                (im ? tf1 : tf0)[k + GL] = v;
            }
        }
    // (4)-(6) TF_GRAD: PSIF_MTP with the column fill, DTDN on layers 1..NN1-2, MFDOT
    std::vector<double> psif_mtp = cal_psif_mtp(c, 1);
    for (int m = 1; m <= NN1 - 2; ++m)
        for (int k : c.band[m]) {
            const double gz = 0.5 * (c.p(k + 1) - c.p(k - 1)) * c.ssdzf;
            const double agi = 1.0 / std::sqrt((0.0 + 0.0) + gz * gz);
            const double dtz0 = 0.5 * (tf0[k + 1 + GL] - tf0[k - 1 + GL]) * c.ssdzf;
            const double dtdn0 = ((0.0 + 0.0) + dtz0 * gz) * agi;
            const double dtz1 = 0.5 * (tf1[k + 1 + GL] - tf1[k - 1 + GL]) * c.ssdzf;
            const double dtdn1 = ((0.0 + 0.0) + dtz1 * gz) * agi;
            s.mflvs[k + GL] = ph.ja * ph.prai * ph.rei * (-ph.tcp * dtdn1 + ph.tcm * dtdn0);
        }
    // VOL_TOT_MFDOT: trial advance of the band by the mass flux, reinitialisation, new
    // volume fraction; SFGAS, SFGAS2 and VOL_TOT_IPHS
    {
        Col t = c;
        std::vector<double> mfd(nf + 7, 0.0);
        for (int m = 1; m <= NN1 - 2; ++m)
            for (int k : t.band[m]) mfd[k + GL] = (t.p(k) > 0.0) ? s.mflvs[k + GL] / ph.denr : s.mflvs[k + GL];
        for (int m = 1; m <= NN1 - 2; ++m)
            for (int k : t.band[m]) {
                const double a0 = t.p(k);
                double a = a0 - 2 * dtconst * mfd[k + GL];
                a = 0.75 * a0 + 0.25 * a;
                a = a - dtconst * mfd[k + GL];
                a = 1.0 / 3.0 * a0 + 2.0 / 3.0 * a;
                t.p(k) = a;
            }
        reinitialization(t, NN2);
        // the interface position the reference prints and appends to 0interface.dat
        // (chphase.f:1419-1431): zpf(k) + |phi(k)| of the last sign change of the trial
        // band phi over k = 1..N3FM (phi outside the band is 0 here, so it makes none)
        g_place = 0.0;
        for (int k = 1; k <= nf; ++k)
            if (t.p(k) * t.p(k + 1) < 0.0) g_place = g.zpf(k) + std::fabs(t.p(k));
        std::vector<double> psif_mtp2 = cal_psif_mtp(t, 1);
        const double dvol = 0.5 * 0.5 * g.hf;
        double vol = 0.0;
        for (int k = 1; k <= nf; ++k)
            for (int r = 0; r < 4; ++r) vol = vol + (1.0 - psif_mtp2[k]) * dvol;
        s.scal[4] = vol;
        for (int k = 0; k <= nf + 1; ++k) {
            s.sfgas[k] = 0.0;
            s.sfgas2[k] = 0.0;
        }
        for (int m = 1; m <= NN1 - 2; ++m)
            for (int k : c.band[m]) {
                if (s.mflvs[k + GL] == 0.0) continue;
                if (std::fabs(psif_mtp[k] - 0.5) == 0.5) continue;
                if (c.p(k) > 0.0) {
                    s.sfgas[k] = -(psif_mtp2[k] - psif_mtp[k]) * ph.denr;
                    s.sfgas2[k] = -(psif_mtp2[k] - psif_mtp[k]);
                } else {
                    s.sfgas[k] = -(psif_mtp2[k] - psif_mtp[k]);
                    s.sfgas2[k] = -(psif_mtp2[k] - psif_mtp[k]);
                }
            }
    }
    // (7) CAL_PSI_TMP(1) and the phase-change mask (chphase.f:297-357, z faces only)
    std::vector<double> psi_tmp(n + 2, 1.0);
    for (int k = 1; k <= n; ++k) {
        const double v = box_mean(psif_mtp.data(), nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
        if (v <= 1e-3) psi_tmp[k] = 0.0;
        else if (v >= 0.999) psi_tmp[k] = 1.0;
        else psi_tmp[k] = v;
    }
    for (int k = 2; k <= n; ++k)
        if (std::fabs(psi_tmp[k] - psi_tmp[k - 1]) != 0.0) s.imask[k] = 1;
    return iters;
}

// CAL_CONTINUITY2, 1d.f:3006-3169: remove the phase-change volume SFGAS2 from PSI_Z and
// PSI_C in the interface region.
void cal_continuity2(const Geo& g, const Phys& ph, const ColView& s, Work& wk) {
    const int n = g.n, nf = g.nf;
    if (ph.denm != ph.denp || ph.vism != ph.visp) make_region(g, s, wk);
    for (int k = 2; k <= n; ++k)
        if (wk.reg(k) == 2) {
            const double ssum = box_mean(s.sfgas2, nf, g.kcou2(k), g.kcou1(k + 1), g.zp(k - 1), g.zp(k), g.hf);
            wk.psi_z[k] = wk.psi_z[k] - ssum;
        }
    for (int k = 2; k <= n; ++k) {
        if (wk.psi_z[k] > 1.0) wk.psi_z[k] = 1.0;
        else if (wk.psi_z[k] < 0.0) wk.psi_z[k] = 0.0;
    }
    for (int k = 1; k <= n; ++k)
        if (wk.reg(k) == 2) {
            const double ssum = box_mean(s.sfgas2, nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
            wk.psi_c[k] = wk.psi_c[k] - ssum;
        }
    for (int k = 1; k <= n; ++k) {
        if (wk.psi_c[k] > 1.0) wk.psi_c[k] = 1.0;
        else if (wk.psi_c[k] < 0.0) wk.psi_c[k] = 0.0;
    }
    wk.psi_z[1] = wk.psi_z[2];
    wk.psi_z[n + 1] = wk.psi_z[n];
    wk.psi_c[1] = wk.psi_c[2];
    wk.psi_c[n + 1] = wk.psi_c[n];
}

// PASSIVE_SCALAR, 1d.f:3630-3707 (IPS = 1).
int passive_scalar(const Geo& g, double L, const Phys& ph, const ColView& s, int msub, double alpha, double dtconst,
                   Work& wk) {
    const int n = g.n;
    const double dt = s.scal[0];
    const int m_step = (int)s.scal[2];
    int iters = 0;
    if (ph.iphs == 1 && m_step != 1) {
        // CAL_RHSPS2 (1d.f:4175-4377): with IPHS = 1 only the dilatation term survives
        for (int k = 1; k <= n; ++k) wk.rhsps[k] = (GAMMA[msub] * s.t[k] * (s.w[k + 1] - s.w[k]) * g.vvdz(k)) * dt;
        for (int k = 1; k <= n; ++k) {
            double densc, denscf;
            if (s.psi_cn[k] > 0.5) {
                densc = ph.denscm + ph.densc_diff;
                denscf = densc;
            } else {
                densc = ph.denscm;
                denscf = densc;
            }
            wk.rhsps[k] = ((densc - denscf) * s.t[k] + wk.rhsps[k]) / denscf;
        }
        lhsps(g, ph, s, alpha, wk);   // LHSPS2 substitute
        iters = temp_grad(g, L, ph, s, dtconst);
        if (iters < 0) return -1;
        cal_continuity2(g, ph, s, wk);
        cal_cont_bc(g, ph, wk);
    } else {
        // CAL_RHSPS (1d.f:4038-4172): convection and diffusion are zeroed there, TGR = 0
        for (int k = 1; k <= n; ++k) {
            const double anps = 0.0, alps = 0.0, anpso = 0.0, tgr = 0.0;
            const double densc = ph.denscm + ph.densc_diff * s.psi_cn[k];
            const double uu = 0.5 * (s.w[k + 1] + s.w[k]);
            const double ameant1 = densc * uu * tgr;
            const double tct = ph.tcm + ph.tc_diff * ((wk.df_c[k] - ph.denm) * (1.0 / ph.den_diff));
            const double tcb = ph.tcm + ph.tc_diff * ((wk.df_c[k - 1] - ph.denm) * (1.0 / ph.den_diff));
            const double ameant2 = (1.0 / (ph.re * ph.prm)) * (tct - tcb) * g.ssdz(k) * tgr;
            wk.rhsps[k] =
                ((GAMMA[msub] * anps + RO[msub] * anpso) + 2. * alpha * alps + 2. * alpha * (ameant1 - ameant2)) * dt;
        }
        for (int k = 1; k <= n; ++k) {
            const double densc = ph.denscm + ph.densc_diff * s.psi_cn[k];
            const double denscf = ph.denscm + ph.densc_diff * wk.psi_c[k];
            wk.rhsps[k] = ((densc - denscf) * s.t[k] + wk.rhsps[k]) / denscf;
        }
        lhsps(g, ph, s, alpha, wk);
    }
    return iters;
}

// RHSZ, 1d.f:1603-1745 (1-D: x/y terms are exactly zero, SUR_Z = 0, no buoyancy, PMI = 0).
void rhsz(const Geo& g, const Phys& ph, const ColView& s, int msub, double alpha, Work& wk) {
    const int n = g.n;
    const double dt = s.scal[0];
    const double* w = s.w;
    for (int k = 2; k <= n; ++k) {
        const double wt = 0.5 * (w[k + 1] + w[k]);
        const double wb = 0.5 * (w[k] + w[k - 1]);
        const double anzz = (wk.df_z[k] * (wt * wt) - wk.df_z[k - 1] * (wb * wb)) * g.vvdz(k);
        const double anz = -0.0 - 0.0 - anzz;
        const double alz5 = (w[k + 1] - w[k]) * g.ssdz(k);
        const double alz6 = (w[k] - w[k - 1]) * g.ssdz(k - 1);
        const double alzz = (wk.vf_z[k] * alz5 - wk.vf_z[k - 1] * alz6) * g.vvdz(k);
        const double alz_sum1 = 0.0 + 0.0 + alzz + alzz;
        const double alz_sum2 = 0.0 + 0.0;
        const double pgr_z = (s.p[k] - s.p[k - 1]) * g.vvdz(k);
        const double den_zn = ph.denm + ph.den_diff * s.psi_zn[k];
        const double rk3z = anz + alz_sum2;
        const double cn2z = alz_sum1;
        const double sur_z = 0.0, buoy = 0.0, pmi = 0.0;
        double r = den_zn * w[k] + (GAMMA[msub] * rk3z + RO[msub] * wk.rk3zo[k] + 2. * alpha * cn2z +
                                     2. * alpha * (sur_z - pgr_z) - 2. * alpha * buoy - 2. * alpha * (pmi + 0.0)) *
                                        dt;
        if (ph.iphs == 1 && s.imask[k] == 1 && std::fabs(s.psi_zn[k] - 0.5) != 0.5)
            r = r + GAMMA[msub] * dt * den_zn * w[k] * ((0.0 - 0.0) * 1.0 + (0.0 - 0.0) * 1.0 + (wt - wb) * g.vvdz(k));
        wk.rhs1[k] = r;
        wk.rk3zo[k] = rk3z;
    }
}

// DIVGS, 1d.f:3180-3303.
void divgs(const Geo& g, const Phys& ph, const ColView& s, double dtconsti, Work& wk) {
    const int n = g.n;
    for (int k = 1; k <= n - 1; ++k) wk.divgsum[k] = (s.w[k + 1] - s.w[k]) * g.ssdz(k);
    wk.divgsum[n] = 0.0;
    if (ph.iphs == 1)
        for (int k = 1; k <= n; ++k) {
            const double ssum = box_mean(s.sfgas, g.nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
            wk.divgsum[k] = wk.divgsum[k] - ssum * (ph.den_diff / (ph.denp * ph.denm));
        }
    for (int k = 2; k <= n; ++k) wk.divgsum[k] = wk.divgsum[k] * dtconsti;
}

// POISSON (1d.f:3492-3578) + UCALC (3582-3627) + the reference shift of
// PRESSURE_CORRECTION (3403-3488).
void pressure_correction(const Geo& g, const ColView& s, double dtconst, double dtconsti, Work& wk, const Phys& ph) {
    const int n = g.n;
    divgs(g, ph, s, dtconsti, wk);
    std::vector<double> ak(n + 2), bk(n + 2), ck(n + 2), gk(n + 2);
    for (int k = 1; k <= n; ++k) {
        const double fixkl = (k == 1) ? 1.0 : 0.0;
        ak[k] = g.vvdz(k) * g.ssdz(k) * wk.denf_zi[k] * (1.0 - fixkl);
        ck[k] = g.vvdz(k + 1) * g.ssdz(k) * wk.denf_zi[k + 1];
        bk[k] = -(ak[k] + ck[k]);
        gk[k] = wk.divgsum[k];
    }
    thomas(ak, bk, ck, gk, 1, n);
    for (int k = 1; k <= n; ++k) s.p[k] = gk[k];
    s.p[0] = s.p[1];
    s.p[n + 1] = s.p[n];
    for (int k = 2; k <= n; ++k) s.w[k] = s.w[k] - dtconst * (s.p[k] - s.p[k - 1]) * g.vvdz(k) * wk.denf_zi[k];
    s.w[1] = 0.0;
    s.w[n + 1] = s.w[n];
    const double phiref = s.p[1];
    for (int k = 1; k <= n; ++k) s.p[k] = s.p[k] - phiref;
    s.p[0] = s.p[1];
}

// One substep of RHSNLHS (1d.f:1444-1600).
int rhsnlhs(const Geo& g, double L, const Phys& ph, const ColView& s, int msub, double alpha, double acoef,
            double dtconst, double dtconsti, Work& wk) {
    const int n = g.n;
    std::fill(wk.rhs1.begin(), wk.rhs1.end(), 0.0);
    cal_continuity(g, ph, s, dtconst, wk);
    cal_cont_bc(g, ph, wk);
    const int iters = passive_scalar(g, L, ph, s, msub, alpha, dtconst, wk);
    if (iters < 0) return -1;
    rhsz(g, ph, s, msub, alpha, wk);
    for (int k = 2; k <= n; ++k) wk.rhs1[k] = wk.rhs1[k] * wk.denf_zi[k] - s.w[k];
    // LHSW, 1d.f:1749-1809
    {
        std::vector<double> ak(n + 2), bk(n + 2), ck(n + 2), gk(n + 2);
        for (int k = 2; k <= n; ++k) {
            const double dk1 = 2. * acoef * wk.denf_zi[k] * wk.vf_z[k - 1] * g.akw(k);
            const double dk3 = 2. * acoef * wk.denf_zi[k] * wk.vf_z[k] * g.ckw(k);
            const double dk2 = -dk1 - dk3;
            ak[k] = dk1;
            ck[k] = dk3;
            bk[k] = 1. + dk2;
            gk[k] = wk.rhs1[k];
        }
        thomas(ak, bk, ck, gk, 2, n);
        for (int k = 2; k <= n; ++k) s.w[k] = gk[k] + s.w[k];
    }
    // BC + BC_FLUX, 1d.f:1812-1923 (AA = 2 XL YL)
    s.w[1] = 0.0;
    s.w[n + 1] = s.w[n];
    {
        double qq3 = 0.0;
        qq3 = qq3 + (s.w[n + 1] - s.w[1]) * 1.0 * 1.0;
        double aa = 0.0;
        aa = aa + 2. * 1.0 * 1.0;
        const double ubc_avg = -qq3 / aa;
        s.w[1] = 0.0;
        s.w[n + 1] = s.w[n + 1] + ubc_avg;
    }
    // FSM_CHOI, 1d.f:3365-3400
    for (int k = 2; k <= n; ++k) s.w[k] = s.w[k] + dtconst * ((s.p[k] - s.p[k - 1]) * g.vvdz(k)) * wk.denf_zi[k];
    pressure_correction(g, s, dtconst, dtconsti, wk, ph);
    return iters;
}

// CONVRGE1, 1d.f:3306-3362.
double convrge1(const Geo& g, const Phys& ph, const ColView& s) {
    double dvmax = 0.0;
    for (int k = 1; k <= g.n; ++k) {
        double d = (s.w[k + 1] - s.w[k]) * g.ssdz(k);
        if (ph.iphs == 1) {
            const double ssum = box_mean(s.sfgas, g.nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
            d = d - ssum * (ph.den_diff / ph.denp);
        }
        dvmax = std::max(std::fabs(d), dvmax);
    }
    return dvmax;
}

ColView view(int n, double L, double* w, double* p, double* t, double* psi_cn, double* psi_zn, double* phi,
             int* layer, double* psif, double* wo, double* mflvs, double* sfgas, double* sfgas2, int* imask,
             double* scal) {
    return ColView{n, L, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2, imask, scal};
}

}  // namespace

extern "C" {

// Column state for the C ABI (flow arrays n+2 doubles at [k], k = 0..n+1):
//   w, p, t, psi_cn, psi_zn; level set phi/layer (nf+7), psif (nf+2), wo (n+2);
//   phase change mflvs (nf+7), sfgas, sfgas2 (nf+2), imask (n+2 ints);
//   scal[5] = DT, TIME, M (steps taken), VOL_TOT_ORI, VOL_TOT_IPHS.
// Properties: props[12] = RE, VISR, DENR, WEBER, FR, PRM, SCR, TCR, T_SAT, JAKOB,
//   CFLMAX, DT (initial); iprops[2] = IPHS, MGLOBAL.

static ColProps props_of(const double* props, const int* iprops) {
    return ColProps{props[0], props[1], props[2], props[3], props[4], props[5], props[6], props[7],
                    props[8], props[9], props[10], props[11], iprops[0], iprops[1]};
}

// MAKEFLD (1d.f:821-946, IPHS = 1 branch) + LVSINIT (two_phase.f:116-388) +
// GRID_COUPLING(1) for a planar film of thickness z0 at the wall.
static int col_init(int n, double L, double z0, const double* props, const int* iprops, double* w, double* p,
                    double* t, double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo,
                    double* mflvs, double* sfgas, double* sfgas2, int* imask, double* scal, const ColGeo* cg) {
    const ColProps cp = props_of(props, iprops);
    Geo g(n, L, cg);
    const int nf = g.nf;
    for (int k = 0; k <= n + 1; ++k) {
        w[k] = 0.0;
        p[k] = 0.0;
        t[k] = 0.0;
        psi_cn[k] = 0.0;
        psi_zn[k] = 0.0;
        imask[k] = 0;
    }
    for (int k = 1; k <= n; ++k) {
        const double pbody = (g.zp(k) - z0) + 1e-12;
        if (pbody > 0.0) {
            t[k] = 1.0;
            w[k] = 1.0;
            w[n + 1] = 1.0;
        } else {
            t[k] = 16.47 * g.zp(k);
            t[0] = 0.0;
            w[k] = 0.0;
            w[1] = 0.0;
        }
    }
    double vol = 0.0;
    const int rc = orc_lvs_init(n, L, z0, phi, layer, psif, wo, &vol);
    if (rc) return rc;
    grid_coupling(n, L, psif, layer, 1, psi_cn, psi_zn, cg);
    for (int k = 0; k < nf + 7; ++k) mflvs[k] = 0.0;
    for (int k = 0; k <= nf + 1; ++k) {
        sfgas[k] = 0.0;
        sfgas2[k] = 0.0;
    }
    scal[0] = cp.dt0;
    scal[1] = 0.0;
    scal[2] = 0.0;
    scal[3] = vol;
    scal[4] = vol;
    return 0;
}

int orc_col_init(int n, double L, double z0, const double* props, const int* iprops, double* w, double* p,
                 double* t, double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo,
                 double* mflvs, double* sfgas, double* sfgas2, int* imask, double* scal) {
    return col_init(n, L, z0, props, iprops, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2,
                    imask, scal, nullptr);
}

// The same on a stretched flow grid; geo holds the pointers of a ColGeo (lvs1d_core.hpp),
// in its member order.
int orc_col_init_geo(int n, double L, double z0, const double* props, const int* iprops, double* w, double* p,
                     double* t, double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo,
                     double* mflvs, double* sfgas, double* sfgas2, int* imask, double* scal, const void* geo) {
    return col_init(n, L, z0, props, iprops, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2,
                    imask, scal, static_cast<const ColGeo*>(geo));
}

// The start-up after a restart read, for one column: LVSINIT's read branch
// (two_phase.f:148-205) on the band PREFLD listed -- phi holds the listed values and 0
// elsewhere, layer the list each cell came from -- ALPHI_BC, CAL_PSIF(1, N_MAX) with its
// global snap (two_phase.f:2711-2722), then GRID_COUPLING(1) (1d.f:138).
int orc_col_resume(int n, double L, double* phi, const int* layer, double* psif, double* psi_cn, double* psi_zn) {
    Col c;
    c.init(n, L);
    std::memcpy(c.phi.data(), phi, sizeof(double) * (c.nf + 7));
    for (int m = 1; m <= N_MAX; ++m)
        for (int k = -2; k <= c.nf + 4; ++k)
            if (layer[k + GL] == m) c.band[m].push_back(k);
    c.rebuild_layer();
    alphi_bc(c);
    std::vector<double> ps = cal_psif_mtp(c, 1, N_MAX);
    for (int k = 0; k <= c.nf + 1; ++k) {
        double v = (k >= 1 && k <= c.nf) ? ps[k] : 0.0;
        if (v < 1e-5) v = 0.0;
        else if (v > 0.99999) v = 1.0;
        psif[k] = v;
    }
    for (int k = 0; k <= n + 1; ++k) {
        psi_cn[k] = 0.0;
        psi_zn[k] = 0.0;
    }
    grid_coupling(n, L, psif, c.layer.data(), 1, psi_cn, psi_zn);
    std::memcpy(phi, c.phi.data(), sizeof(double) * (c.nf + 7));
    return 0;
}

// One time step of MAIN (1d.f:190-250): DETERMINE_DT, three RK3 substeps of RHSNLHS,
// CONVRGE1, TRANSPORT and GRID_COUPLING(0), TIME += DT.
//   stats[8]: CFL of the flow, max |div u - source| (last substep), TEMP_EXTP iterations,
//             level-set subcycles (sum), reinitialisation/mass triggers (IMASS sum),
//             interface height, vapour volume VOL_TOT_IPHS, DT.
// Returns 0, 1 (TEMP_EXTP did not converge) or 2 (band overflow).
static int col_step(int n, double L, const double* props, const int* iprops, double* w, double* p, double* t,
                    double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo, double* mflvs,
                    double* sfgas, double* sfgas2, int* imask, double* scal, double* stats, const ColGeo* cg) {
    const ColProps cp = props_of(props, iprops);
    const Phys ph(cp);
    Geo g(n, L, cg);
    ColView s = view(n, L, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2, imask, scal);
    Work wk(n);
    g_place = 0.0;
    scal[2] = scal[2] + 1.0;
    const int m_step = (int)scal[2];
    if (m_step == 1)
        for (int k = 0; k < g.nf + 7; ++k) mflvs[k] = 0.0;
    double cflm = 0.0;
    determine_dt(g, ph, s, cflm);
    std::fill(wk.rk3zo.begin(), wk.rk3zo.end(), 0.0);
    double dvmax = 0.0, subcycles = 0.0, imass = 0.0, iters = 0.0;
    for (int msub = 1; msub <= 3; ++msub) {
        const double alpha = 0.5 * (GAMMA[msub] + RO[msub]);
        const double acoef = alpha * scal[0];
        const double dtconst = 2. * alpha * scal[0];
        const double dtconsti = 1. / dtconst;
        const int it = rhsnlhs(g, L, ph, s, msub, alpha, acoef, dtconst, dtconsti, wk);
        if (it < 0) return 1;
        iters += it;
        dvmax = convrge1(g, ph, s);
        double lst[4];
        const int rc = orc_lvs_transport_geo(n, L, phi, layer, psif, wo, w, mflvs, ph.iphs, ph.denr, dtconst,
                                             (m_step == 1 && msub == 1) ? 1 : 0, m_step, &scal[3], scal[4],
                                             ph.mglobal, psi_cn, psi_zn, lst, cg);
        if (rc) return rc;
        subcycles += lst[0];
        imass += (lst[0] > 0) ? lst[3] : 0.0;
    }
    scal[1] = scal[1] + scal[0];
    // interface height: the first sign change of the band phi from the wall
    double zi = 0.0;
    for (int k = 1; k < g.nf; ++k)
        if (layer[k + GL] > 0 && layer[k + 1 + GL] > 0 && phi[k + GL] < 0.0 && phi[k + 1 + GL] >= 0.0) {
            zi = g.zpf(k) - phi[k + GL] * (g.zpf(k + 1) - g.zpf(k)) / (phi[k + 1 + GL] - phi[k + GL]);
            break;
        }
    stats[0] = cflm;
    stats[1] = dvmax;
    stats[2] = iters;
    stats[3] = subcycles;
    stats[4] = imass;
    stats[5] = zi;
    stats[6] = scal[4];
    stats[7] = scal[0];
    return 0;
}

int orc_col_step(int n, double L, const double* props, const int* iprops, double* w, double* p, double* t,
                 double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo, double* mflvs,
                 double* sfgas, double* sfgas2, int* imask, double* scal, double* stats) {
    return col_step(n, L, props, iprops, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2, imask,
                    scal, stats, nullptr);
}

// One time step on a stretched flow grid (geo: a ColGeo, lvs1d_core.hpp).
int orc_col_step_geo(int n, double L, const double* props, const int* iprops, double* w, double* p, double* t,
                     double* psi_cn, double* psi_zn, double* phi, int* layer, double* psif, double* wo, double* mflvs,
                     double* sfgas, double* sfgas2, int* imask, double* scal, double* stats, const void* geo) {
    return col_step(n, L, props, iprops, w, p, t, psi_cn, psi_zn, phi, layer, psif, wo, mflvs, sfgas, sfgas2, imask,
                    scal, stats, static_cast<const ColGeo*>(geo));
}

// TEMP_GRAD (chphase.f:55-368, with TEMP_EXTP, TF_GRAD and VOL_TOT_MFDOT) of one column as a
// single routine: reads T, PSI_CN and the band (phi, layer); writes MFLVS, SFGAS, SFGAS2,
// IMASK_PH and VOL_TOT_IPHS (*vol).  Returns the TEMP_EXTP iterations, or -1 when it did
// not converge.
int orc_col_temp_grad(int n, double L, const double* props, const int* iprops, double dtconst, const double* t,
                      const double* psi_cn, const double* phi, const int* layer, double* mflvs, double* sfgas,
                      double* sfgas2, int* imask, double* vol) {
    const ColProps cp = props_of(props, iprops);
    const Phys ph(cp);
    Geo g(n, L);
    std::vector<double> tv(t, t + n + 2), cn(psi_cn, psi_cn + n + 2), pv(phi, phi + 2 * n + 7);
    std::vector<int> lv(layer, layer + 2 * n + 7);
    double scal[5] = {0.0, 0.0, 0.0, 0.0, *vol};
    ColView s = view(n, L, nullptr, nullptr, tv.data(), cn.data(), nullptr, pv.data(), lv.data(), nullptr, nullptr,
                     mflvs, sfgas, sfgas2, imask, scal);
    const int it = temp_grad(g, L, ph, s, dtconst);
    *vol = scal[4];
    return it;
}

// PRESSURE_CORRECTION (1d.f:3403-3488: DIVGS, POISSON, UCALC, the shift by P(1)) of one
// column as a single routine: W and P in place; DENF_ZI and (IPHS = 1) SFGAS read.
int orc_col_pressure_correction(int n, double L, const double* props, const int* iprops, double dtconst, double* w,
                                double* p, const double* denf_zi, const double* sfgas) {
    const ColProps cp = props_of(props, iprops);
    const Phys ph(cp);
    Geo g(n, L);
    ColView s = view(n, L, w, p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                     const_cast<double*>(sfgas), nullptr, nullptr, nullptr);
    Work wk(n);
    for (int k = 0; k <= n + 1; ++k) wk.denf_zi[k] = denf_zi[k];
    pressure_correction(g, s, dtconst, 1. / dtconst, wk, ph);
    return 0;
}

// The record the reference appends to 0interface.dat at the end of the last substep of a
// step (chphase.f:1432-1438, TIME before MAIN adds DT at 1d.f:260) for the step just taken
// by orc_col_step on this thread: place of VOL_TOT_MFDOT in the third substep (0 when the
// step ran no phase change).
double orc_col_last_place() { return g_place; }

}  // extern "C"
