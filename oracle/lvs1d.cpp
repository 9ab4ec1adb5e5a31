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
#include "lvs1d_core.hpp"

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
    // ALPHI exists on the band only: band cells get the exact distance again, the rest 0
    std::fill(c.phi.begin(), c.phi.end(), 0.0);
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
static int transport(int n, double L, double* phi, int* layer, double* psif, double* wo, const double* w,
                     const double* mflvs, int iphs, double denr, double dtconst, int first, int m_step,
                     double* vol_tot_ori, double vol_tot_iphs, int mglobal, double* psi_cn, double* psi_zn,
                     double* stats, const ColGeo* cg) {
    State s;
    load(s, n, L, phi, layer, psif, wo);
    s.c.cg = cg;
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
    // GRID_COUPLING(0)
    grid_coupling(n, L, s.psif.data(), c.layer.data(), 0, psi_cn, psi_zn, cg);
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

int orc_lvs_transport(int n, double L, double* phi, int* layer, double* psif, double* wo, const double* w,
                      const double* mflvs, int iphs, double denr, double dtconst, int first, int m_step,
                      double* vol_tot_ori, double vol_tot_iphs, int mglobal, double* psi_cn, double* psi_zn,
                      double* stats) {
    return transport(n, L, phi, layer, psif, wo, w, mflvs, iphs, denr, dtconst, first, m_step, vol_tot_ori,
                     vol_tot_iphs, mglobal, psi_cn, psi_zn, stats, nullptr);
}

// The same on a stretched flow grid (geo: a ColGeo, lvs1d_core.hpp).
int orc_lvs_transport_geo(int n, double L, double* phi, int* layer, double* psif, double* wo, const double* w,
                          const double* mflvs, int iphs, double denr, double dtconst, int first, int m_step,
                          double* vol_tot_ori, double vol_tot_iphs, int mglobal, double* psi_cn, double* psi_zn,
                          double* stats, const void* geo) {
    return transport(n, L, phi, layer, psif, wo, w, mflvs, iphs, denr, dtconst, first, m_step, vol_tot_ori,
                     vol_tot_iphs, mglobal, psi_cn, psi_zn, stats, static_cast<const ColGeo*>(geo));
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

// REINITIALIZATION(NN1, NN2, ILIMIT) (two_phase.f:2033-2474) of one column as a single
// routine: ALPHI_EXT is the caller's phi array (every cell, ghosts included), the band
// the cells whose layer is 1..N_MAX (ascending k per layer); ILIMIT SSP-RK3 iterations on
// layers 1..NN2.  Only the band cells are written back.
int orc_reinitialization(int n, double L, double* phi, const int* layer, int ilimit) {
    Col c;
    c.init(n, L);
    for (int k = -2; k <= c.nf + 4; ++k) c.phi[k + GL] = phi[k + GL];
    for (int m = 1; m <= N_MAX; ++m)
        for (int k = -2; k <= c.nf + 4; ++k)
            if (layer[k + GL] == m) c.band[m].push_back(k);
    c.rebuild_layer();
    reinitialization(c, ilimit);
    for (int m = 1; m <= N_MAX; ++m)
        for (int k : c.band[m]) phi[k + GL] = c.p(k);
    return 0;
}

// GRID_COUPLING(INI_PSI) (two_phase.f:4863-5118) of one column as a single routine.
int orc_grid_coupling(int n, double L, int ini, const double* psif, const int* layer, double* psi_cn,
                      double* psi_zn) {
    grid_coupling(n, L, psif, layer, ini, psi_cn, psi_zn);
    return 0;
}

}  // extern "C"
