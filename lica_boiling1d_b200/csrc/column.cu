// One or many time steps of the 1-D boiling column on the GPU: MAIN's RK3 step
// (1d.f:190-250) -- DETERMINE_DT, three substeps of RHSNLHS (CAL_CONTINUITY, CAL_CONT_BC,
// PASSIVE_SCALAR with TEMP_GRAD / TEMP_EXTP / TF_GRAD / VOL_TOT_MFDOT / CAL_CONTINUITY2,
// RHSZ, LHSW, BC, FSM_CHOI, PRESSURE_CORRECTION), CONVRGE1, TRANSPORT and GRID_COUPLING --
// fused into one persistent kernel.
//
// Parallel structure: one CTA per column; the CTA loops over the time steps without
// returning to the host.  Per-cell work is spread over the CTA's threads with a barrier
// between phases; the three tridiagonal solves per substep (LHSPS, LHSW, POISSON) run as
// the Thomas algorithm on one thread, in the reference's order; the band work (TEMP_GRAD's
// interface pieces, TEMP_EXTP's narrow extension region, TRANSPORT) runs on warp 0 with the
// band window of lvs_device.cuh in shared memory.  Columns of a batch are independent.
//
// CONTI_Z / CONTI_C (1d.f:2071-2346) are serial loops that set a face value only while it
// is still zero; they are evaluated here per face in closed form: the value seen by cell K
// for its lower face is the one cell K-1 set (a region-0/1 constant, or the swept-volume
// value of that face, which cell K would compute identically), and the final face value is
// cell K+1's constant when that cell is in region 0/1, else cell K's value.
//
// Every floating-point expression keeps the reference's operation order; with the
// library's -fmad=false the results agree bit for bit with the CPU restatement.
#include "lvs_device.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

extern "C" void lica_count_launches(int64_t n);

namespace lica {
namespace colk {

// lica.in properties and the derived constants of INPUT_SIMULATION (1d.f:437-489).
struct Phys {
    double re, rei, denm, denp, den_diff, vism, visp, denscm, denscp, densc_diff, tcm, tcp, tc_diff, prm, prai,
        surf, gravity, time_st, time_gv, denr, ja, t_sat, cflmax;
    int iphs, mglobal;
};

constexpr int NT_DEFAULT = 128;  // threads per column CTA of the single-routine kernel
constexpr int NFLOW = 30;        // flow-sized scratch arrays per column
constexpr int XR = 132;          // TEMP_EXTP extension range held in shared memory (+halo)

__constant__ double c_gamma[4] = {0.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
__constant__ double c_ro[4] = {0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0};

// scratch array indices (each n+2 doubles)
enum {
    S_DFZ, S_VFZ, S_PSIZ, S_DFC, S_PSIC, S_DENFZ, S_DENFZI, S_DENFC, S_RHS1, S_RK3ZO, S_RHSPS, S_DIVG,
    S_AK, S_BK, S_CK, S_GK, S_GAM, S_VZD, S_VZV, S_VCD, S_TEMP0, S_TEMP1, S_NPHI, S_PSIH, S_PSITMP, S_SPARE0,
    S_SPARE1, S_SPARE2, S_SPARE3, S_SPARE4
};

// One column of a batch of uneven columns: size, length, constants and the offsets of
// its arrays in the packed state (flow, refined phi-like, refined psif-like) and scratch.
struct ColDesc {
    int n, pad;
    double L;
    Phys ph;
    long long off_f, off_p, off_q, off_d, off_i;
};

struct Args {
    int ncol, n, nsteps;
    double L;
    Phys ph;
    const ColDesc* desc;   // per-column descriptors, or null for ncol columns of size n
    const int* order;      // launch order (CTA b runs column order[b]), or null
    double *w, *p, *t, *psi_cn, *psi_zn, *phi, *psif, *wo, *mflvs, *sfgas, *sfgas2, *scal, *stats;
    int *layer, *imask, *status;
    double* dscr;
    int* iscr;
    long long* prof;   // optional per-phase cycle totals (PH_COUNT per column) or null
    double* hist;      // optional interface history (HIST_REC doubles per column and step) or null
    int hist_cap;      // steps of one launch the history holds per column
    int tri_smem;      // 1: the tridiagonal arrays of columns with n <= tri_cap live in dynamic shared memory
    int tri_cap;       // longest column whose arrays fit the dynamic shared memory (longer ones use scratch)
    int has_geo;       // 1: every column is the stretched column geo describes (device arrays)
    col::ColGeoDev geo;
};

// one record of the optional interface history: TIME before the step, place, VOL_TOT_IPHS, DT
constexpr int HIST_REC = 4;

// phases of the optional cycle profile
enum { PH_DT, PH_CONT, PH_ENERGY, PH_TEMPGRAD, PH_EXTP, PH_CONT2, PH_RHSZ, PH_LHSW, PH_PRESS, PH_CONV, PH_TRANSPORT,
       PH_COUNT };

// The column's wall-normal geometry: GEOMETRIC's arrays and GEOM_COUPLING's z tables of a
// stretched column (cg), or the closed forms of the uniform one.
struct Geo {
    int n, nf;
    double h, hf;
    double ih, ihalf;   // 1/h (SSDZ, VVDZ inside) and 1/(h/2) (VVDZ at the walls), computed once
    const col::ColGeoDev* cg;
    __device__ Geo(int n_, double L, const col::ColGeoDev* cg_ = nullptr)
        : n(n_), nf(2 * n_), h(L / n_), hf(L / (2 * n_)), cg(cg_) {
        ih = 1.0 / h;
        ihalf = 1.0 / (0.5 * h);
    }
    __device__ double sdz(int k) const { return cg ? cg->sdz[k] : ((k >= 1 && k <= n) ? h : 0.0); }
    __device__ double ssdz(int k) const { return cg ? cg->ssdz[k] : ih; }
    __device__ double vdz(int k) const { return cg ? cg->vdz[k] : ((k == 1 || k == n + 1) ? 0.5 * h : h); }
    __device__ double vvdz(int k) const { return cg ? cg->vvdz[k] : ((k == 1 || k == n + 1) ? ihalf : ih); }
    __device__ double z(int k) const { return cg ? cg->z[k] : col::grid_z(h, k); }
    __device__ double zp(int k) const { return cg ? cg->zp[k] : col::grid_zp(h, n, k); }
    // GEOM_COUPLING's refined faces (uniform column: face K is refined face 2K-1, centre K
    // refined face 2K) and KCOUMP_VEL of a refined cell
    __device__ int kcou1(int k) const { return cg ? cg->kcou1[k + 1] : 2 * k - 2; }
    __device__ int kcou2(int k) const { return cg ? cg->kcou2[k + 1] : 2 * k - 1; }
    __device__ int kcoump1(int k) const { return cg ? cg->kcoump1[k + 1] : 2 * k - 1; }
    __device__ int kcoump2(int k) const { return cg ? cg->kcoump2[k + 1] : 2 * k; }
    __device__ int kcoump_vel(int k) const { return cg ? cg->kcoump_vel[k] : col::kcoump_vel(h, hf, n, k); }
    __device__ double zpf(int k) const { return col::grid_zpf(hf, k); }
    __device__ double akw(int k) const { return -vvdz(k) * ssdz(k - 1); }
    __device__ double ckw(int k) const { return -vvdz(k) * ssdz(k); }
    __device__ double akuv(int k) const { return -vvdz(k) * ssdz(k); }
    __device__ double ckuv(int k) const { return -vvdz(k + 1) * ssdz(k); }
};

// One column's arrays.
struct Col {
    double *w, *p, *t, *psi_cn, *psi_zn, *phi, *psif, *wo, *mflvs, *sfgas, *sfgas2, *scal, *stats, *psif_mtp;
    int *layer, *imask, *region;   // region indexed k+1, k = -1..n+2
    double* a[NFLOW];
    long long* prof;
    long long t0;
    // cycle profile: thread 0 adds the cycles since the last mark to phase ph
    __device__ __forceinline__ void mark(int ph) {
        if (prof && threadIdx.x == 0) {
            const long long t = clock64();
            prof[ph] += t - t0;
            t0 = t;
        }
    }
};

// TEMP_EXTP arrays of one phase over the flow window [xk0, xk0+XR)
struct XPhase {
    double tm[XR], dt[XR], dtrk[XR], to[XR], trk[XR], nw[XR];
};

struct Shared {
    lvs::Win win;
    double red[32];
    // flow cells xk0 .. xk0+XR-1 around the band (xk0 = the band window's flow origin):
    // NPHI, PSIH and PSI_CN of TEMP_GRAD, and the two phases' extension arrays
    double x_nphi[XR], x_psih[XR], x_pcn[XR];
    XPhase xp[2];
    int ibuf[8];
    double dbuf[8];
};

__device__ __forceinline__ double block_max(double v, Shared& sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh.red[warp] = v;
    __syncthreads();
    double r = sh.red[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) r = fmax(r, sh.red[q]);
    return r;
}
__device__ __forceinline__ double block_min(double v, Shared& sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh.red[warp] = v;
    __syncthreads();
    double r = sh.red[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) r = fmin(r, sh.red[q]);
    return r;
}

// Thomas algorithm of TRDIAG3 (1d.f:3783-3811) on one line, unknowns l1..l2; r becomes the
// solution.  One thread.
// The coefficients are read in blocks of PF ahead of the dependent recurrence, so the
// memory latency overlaps instead of adding to every step of the chain.
constexpr int PF = 4;
__device__ void thomas(const double* a, const double* b, const double* c, double* r, double* gam, int l1, int l2) {
    double bet = 1.0 / b[l1];
    double u = r[l1] * bet;
    r[l1] = u;
    double cprev = c[l1];
    for (int j0 = l1 + 1; j0 <= l2; j0 += PF) {
        double A[PF], B[PF], Cc[PF], R[PF];
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            const int j = min(j0 + q, l2);
            A[q] = a[j];
            B[q] = b[j];
            Cc[q] = c[j];
            R[q] = r[j];
        }
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            const int j = j0 + q;
            if (j <= l2) {
                const double gm = cprev * bet;
                gam[j] = gm;
                bet = 1.0 / (B[q] - A[q] * gm);
                u = (R[q] - A[q] * u) * bet;
                r[j] = u;
                cprev = Cc[q];
            }
        }
    }
    for (int j0 = l2 - 1; j0 >= l1; j0 -= PF) {
        double G[PF], R[PF];
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            const int j = max(j0 - q, l1);
            G[q] = gam[j + 1];
            R[q] = r[j];
        }
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            const int j = j0 - q;
            if (j >= l1) {
                u = R[q] - G[q] * u;
                r[j] = u;
            }
        }
    }
}

#define FOR_K(lo, hi) for (int k = (lo) + (int)threadIdx.x; k <= (hi); k += (int)blockDim.x)

// REGION (1d.f:2038-2056), evaluated per cell: 2 within two cells of a PSI_CN jump, else 1
// in liquid, else 0 (the serial loop's final state).
__device__ void make_region(const Geo& g, Col& c) {
    const int n = g.n;
    FOR_K(-1, n + 2) {
        int r = 0;
        for (int kk = max(1, k - 2); kk <= min(n, k + 2); ++kk)
            if ((c.psi_cn[kk + 1] - c.psi_cn[kk] != 0.0) || (c.psi_cn[kk] - c.psi_cn[kk - 1] != 0.0)) r = 2;
        if (r == 0 && k >= 1 && k <= n && c.psi_cn[k] == 1.0) r = 1;
        c.region[k + 1] = r;
    }
    __syncthreads();
}

// CAL_CONTINUITY (1d.f:1994-2068): CONTI_Z and CONTI_C with PSIFACE_Z / PSIFACE_C and the
// swept-volume box integrals (1d.f:2349-2958).
__device__ void cal_continuity(const Geo& g, const Phys& ph, Col& c, double dtconst) {
    const int n = g.n, nf = g.nf;
    double *df_z = c.a[S_DFZ], *vf_z = c.a[S_VFZ], *psi_z = c.a[S_PSIZ], *df_c = c.a[S_DFC], *psi_c = c.a[S_PSIC];
    double *vzd = c.a[S_VZD], *vzv = c.a[S_VZV], *vcd = c.a[S_VCD];
    const double* w = c.w;
    const int* reg = c.region + 1;
    make_region(g, c);
    // face values as cell K sees them: V(j) (z: j = 1..n; c: j = 0..n)
    FOR_K(0, n) {
        if (k >= 1) {
            const int r = reg[k];
            if (k >= 2 && r == 0) {
                vzd[k] = ph.denm;
                vzv[k] = ph.vism;
            } else if (k >= 2 && r == 1) {
                vzd[k] = ph.denp;
                vzv[k] = ph.visp;
            } else {
                const double wt = 0.5 * (w[k + 1] + w[k]);
                double ps;
                if (fabs(wt) <= 1e-8) {
                    ps = 0.5 * (c.psi_zn[k] + c.psi_zn[k + 1]);
                } else {
                    double z1, z2;
                    int k1, k2;
                    if (wt >= 0.0) {
                        z1 = g.zp(k) - wt * dtconst;
                        z2 = g.zp(k);
                        k1 = g.kcoump2(k - 1);
                        k2 = g.kcoump1(k);
                    } else {
                        z1 = g.zp(k);
                        z2 = g.zp(k) - wt * dtconst;
                        k1 = g.kcoump2(k);
                        k2 = g.kcoump1(k + 1);
                    }
                    ps = col::box_mean(c.psif, nf, k1, k2, z1, z2, g.hf);
                }
                vzv[k] = ph.vism + (ph.visp - ph.vism) * ps;
                vzd[k] = ph.denm + ph.den_diff * ps;
            }
        }
        {
            const int r = reg[k];
            if (k >= 1 && r == 0) {
                vcd[k] = ph.denm;
            } else if (k >= 1 && r == 1) {
                vcd[k] = ph.denp;
            } else {
                const double wt = w[k + 1];
                double ps;
                if (fabs(wt) <= 1e-8) {
                    ps = c.psi_cn[k + 1];
                } else {
                    double z1, z2;
                    int k1, k2;
                    if (wt >= 0.0) {
                        z1 = g.z(k + 1) - wt * dtconst;
                        z2 = g.z(k + 1);
                        k1 = g.kcou2(k);
                        k2 = g.kcou1(k + 1);
                    } else {
                        z1 = g.z(k + 1);
                        z2 = g.z(k + 1) - wt * dtconst;
                        k1 = g.kcou2(k + 1);
                        k2 = g.kcou1(k + 2);
                    }
                    ps = col::box_mean(c.psif, nf, k1, k2, z1, z2, g.hf);
                }
                vcd[k] = ph.denm + ph.den_diff * ps;
            }
        }
    }
    __syncthreads();
    FOR_K(0, n) {
        // final face values
        if (k >= 1) {
            const int rn = (k + 1 <= n) ? reg[k + 1] : 2;
            if (rn == 0) {
                df_z[k] = ph.denm;
                vf_z[k] = ph.vism;
            } else if (rn == 1) {
                df_z[k] = ph.denp;
                vf_z[k] = ph.visp;
            } else {
                df_z[k] = vzd[k];
                vf_z[k] = vzv[k];
            }
        }
        {
            const int rn = (k + 1 <= n) ? reg[k + 1] : 2;
            df_c[k] = (rn == 0) ? ph.denm : (rn == 1 ? ph.denp : vcd[k]);
        }
        // cell values
        if (k >= 2) {
            if (reg[k] == 2) {
                const double wt = 0.5 * (w[k + 1] + w[k]);
                const double wb = 0.5 * (w[k] + w[k - 1]);
                const double flux_z = (vzd[k] * wt - vzd[k - 1] * wb) * g.vvdz(k);
                const double den_zn = ph.denm + ph.den_diff * c.psi_zn[k];
                const double den_z = den_zn - dtconst * flux_z;
                double v = (den_z - ph.denm) / ph.den_diff;
                psi_z[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
            } else {
                const double v = c.psi_zn[k];
                psi_z[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
            }
        }
        if (k >= 1) {
            if (reg[k] == 2) {
                const double wt = w[k + 1], wb = w[k];
                const double flux_z = (vcd[k] * wt - vcd[k - 1] * wb) * g.ssdz(k);
                const double den_cn = ph.denm + ph.den_diff * c.psi_cn[k];
                const double den_c = den_cn - dtconst * flux_z;
                const double v = (den_c - ph.denm) / ph.den_diff;
                psi_c[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
            } else {
                const double v = c.psi_cn[k];
                psi_c[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        psi_z[1] = psi_z[2];
        psi_z[n + 1] = psi_z[n];
        psi_c[1] = psi_c[2];
        psi_c[n + 1] = psi_c[n];
    }
    __syncthreads();
}

// Arrays that are live only inside one routine share the slots of the Thomas arrays, which
// are dead between the tridiagonal solves: CAL_DENVIS's face and centre values (inside
// CAL_CONTINUITY, before the substep's first solve) take AK, BK, CK; TEMP_GRAD's two phase
// temperatures take GK and GAM, and its PSI_TMP takes AK (after LHSPS, before LHSW).  Fewer
// distinct arrays per column keep more of the columns in flight inside L2.
__device__ __forceinline__ void share_scratch(Col& c) {
    c.a[S_VZD] = c.a[S_AK];
    c.a[S_VZV] = c.a[S_BK];
    c.a[S_VCD] = c.a[S_CK];
    c.a[S_TEMP0] = c.a[S_GK];
    c.a[S_TEMP1] = c.a[S_GAM];
    c.a[S_PSITMP] = c.a[S_AK];
}

// CAL_CONT_BC, 1d.f:2961-3003.
__device__ void cal_cont_bc(const Geo& g, const Phys& ph, Col& c) {
    const int n = g.n;
    // DENF_Z and DENF_C themselves are read by no routine of the step: only 1/DENF_Z is kept
    double* dzi = c.a[S_DENFZI];
    const double* psi_z = c.a[S_PSIZ];
    FOR_K(1, n) {
        const double d = ph.denm + ph.den_diff * psi_z[k];
        dzi[k] = 1.0 / d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dzi[n + 1] = dzi[n];
        dzi[0] = dzi[1];
    }
    __syncthreads();
}

// LHSPS, 1d.f:4380-4497.
__device__ void lhsps(const Geo& g, const Phys& ph, Col& c, double alpha, double dt) {
    const int n = g.n;
    const double den_diffi = (ph.den_diff == 0.0) ? 1.0 : 1.0 / ph.den_diff;
    const double acops = alpha * dt / (ph.re * ph.prm);
    double *ak = c.a[S_AK], *bk = c.a[S_BK], *ck = c.a[S_CK], *gk = c.a[S_GK];
    const double *psi_c = c.a[S_PSIC], *df_c = c.a[S_DFC];
    double* rhsps = c.a[S_RHSPS];
    FOR_K(1, n) {
        const double denscf = ph.denscm + ph.densc_diff * psi_c[k];
        const double coef = acops / denscf;
        double psi_tmp = (df_c[k - 1] - ph.denm) * den_diffi;
        const double tcb = ph.tcm + ph.tc_diff * psi_tmp;
        psi_tmp = (df_c[k] - ph.denm) * den_diffi;
        const double tct = ph.tcm + ph.tc_diff * psi_tmp;
        double a = coef * tcb * g.akuv(k);
        double cc = coef * tct * g.ckuv(k);
        bk[k] = 1.0 - (a + cc);
        gk[k] = rhsps[k];
        const double pc = c.psi_cn[k];
        if (fabs(pc - 0.5) != 0.5) {
            if (pc <= 0.5) cc = 0.0;
            else if (pc > 0.5) a = 0.0;
        }
        ak[k] = a;
        ck[k] = cc;
    }
    __syncthreads();
    if (threadIdx.x == 0) thomas(ak, bk, ck, gk, c.a[S_GAM], 1, n);
    __syncthreads();
    FOR_K(1, n) {
        rhsps[k] = gk[k];
        c.t[k] = gk[k] + c.t[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        c.t[0] = 0.0;
        c.t[n] = 1.0;
        c.t[n + 1] = c.t[n];
    }
    __syncthreads();
}

// TEMP_EXTP_RK3, chphase.f:806-956 (1-D), on the extension range in shared memory: x[i]
// holds flow cell xk0 + i.  nd = 0: tempo is the DTEMPN array X.dt itself.
__device__ void extp_sweep(const Geo& g, const Shared& sh, XPhase& X, int xk0, int lo, int hi, double* tempo, int im,
                           double redtl, int nd) {
    const int lane = threadIdx.x & 31;
    const double sm_grid = fmin(fmin(1.0, 1.0), 2.0 * g.hf);
    for (int i = lo + lane; i <= hi; i += 32) {
        const int k = xk0 + i;
        double nv = tempo[i];
        const double nph = sh.x_nphi[i];
        if (nph != 0.0) {
            double dpz;
            if (sh.x_nphi[i - 1] == 0.0) dpz = (sh.x_nphi[i + 1] - nph) * g.vvdz(k + 1);
            else if (sh.x_nphi[i + 1] == 0.0) dpz = (nph - sh.x_nphi[i - 1]) * g.vvdz(k);
            else dpz = 0.5 * (sh.x_nphi[i + 1] - sh.x_nphi[i - 1]) * g.vvdz(k);
            const double dalphi = (0.0 + 0.0) + dpz * dpz;
            if (dalphi != 0.0) {
                double nz = 1.0;
                const double apzm = (tempo[i] - tempo[i - 1]) * g.vvdz(k);
                const double apzp = (tempo[i + 1] - tempo[i]) * g.vvdz(k);
                if (im == 1) nz = (-1.0) * nz;
                const double ax = 0.0, ay = 0.0;
                const double az = fmin(nz, 0.0) * apzp + fmax(nz, 0.0) * apzm;
                double drhs;
                if (im == 1) {
                    drhs = (ax + ay + az) + nd * X.dt[i];
                    nv = tempo[i] - redtl * drhs * (1 - sh.x_psih[i]);
                } else {
                    drhs = (ax + ay + az) - nd * X.dt[i];
                    nv = tempo[i] - redtl * drhs * sh.x_psih[i];
                }
                if (nd == 0 && fabs(nph) <= sm_grid) {
                    drhs = (ax + ay + az);
                    nv = tempo[i] - redtl * drhs;
                }
            }
        }
        X.nw[i] = nv;
    }
    __syncwarp();
    for (int i = lo + lane; i <= hi; i += 32) tempo[i] = X.nw[i];
    __syncwarp();
}

__device__ __forceinline__ double warp_maxd(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

constexpr int kMaxHalvings = 40;

struct ExtpLane {
    int lane, R;
    bool act, small;
    double vv, psh, fmn, fmx;
    int im;
    // one TEMP_EXTP_RK3 step (chphase.f:806-956) of the cell this lane holds
    __device__ __forceinline__ double sweep(double x, double hl, double hr, int nd, double dtn, double redtl) const {
        double xm = __shfl_up_sync(0xffffffffu, x, 1);
        double xp = __shfl_down_sync(0xffffffffu, x, 1);
        if (lane == 0) xm = hl;
        if (lane == R - 1) xp = hr;
        double nv = x;
        if (act) {
            const double apzm = (x - xm) * vv;
            const double apzp = (xp - x) * vv;
            const double ax = 0.0, ay = 0.0;
            const double az = fmn * apzp + fmx * apzm;
            double drhs;
            if (im == 1) {
                drhs = (ax + ay + az) + nd * dtn;
                nv = x - redtl * drhs * (1 - psh);
            } else {
                drhs = (ax + ay + az) - nd * dtn;
                nv = x - redtl * drhs * psh;
            }
            if (nd == 0 && small) {
                drhs = (ax + ay + az);
                nv = x - redtl * drhs;
            }
        }
        return nv;
    }
};

// TEMP_EXTP's two pseudo-time loops for an extension range of at most 32 cells: lane i
// holds cell xk0 + lo + i in registers, neighbours come by shuffle, the halo cells (one
// each side, never updated) are constants.  Same operations and order as extp_sweep.
// Returns the iteration count, or -1 when kMaxHalvings halvings did not converge.
__device__ int extp_registers(const Geo& g, const Shared& sh, XPhase& X, int xk0, int lo, int hi, int im,
                              double eps) {
    const int lane = threadIdx.x & 31;
    ExtpLane L;
    L.lane = lane;
    L.R = hi - lo + 1;
    L.im = im;
    const bool valid = lane < L.R;
    const int xi = valid ? lo + lane : lo;
    const int k = xk0 + xi;
    const double sm_grid = fmin(fmin(1.0, 1.0), 2.0 * g.hf);
    const double nph = sh.x_nphi[xi];
    L.act = false;
    if (valid && nph != 0.0) {
        double dpz;
        if (sh.x_nphi[xi - 1] == 0.0) dpz = (sh.x_nphi[xi + 1] - nph) * g.vvdz(k + 1);
        else if (sh.x_nphi[xi + 1] == 0.0) dpz = (nph - sh.x_nphi[xi - 1]) * g.vvdz(k);
        else dpz = 0.5 * (sh.x_nphi[xi + 1] - sh.x_nphi[xi - 1]) * g.vvdz(k);
        L.act = ((0.0 + 0.0) + dpz * dpz) != 0.0;
    }
    L.small = fabs(nph) <= sm_grid;
    L.vv = g.vvdz(k);
    L.psh = sh.x_psih[xi];
    const double nz = (im == 1) ? (-1.0) * 1.0 : 1.0;
    L.fmn = fmin(nz, 0.0);
    L.fmx = fmax(nz, 0.0);
    int total = 0;
    // extension of the normal gradient (nd = 0); its halo values are 0
    double x = X.dt[xi];
    double redtl = 0.2 * sm_grid;
    bool conv = false;
    for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
        for (int it = 1; it <= 100; ++it) {
            ++total;
            const double rk = x;
            x = L.sweep(x, 0.0, 0.0, 0, x, redtl);
            x = L.sweep(x, 0.0, 0.0, 0, x, redtl);
            x = 0.75 * rk + 0.25 * x;
            x = L.sweep(x, 0.0, 0.0, 0, x, redtl);
            x = 1.0 / 3.0 * rk + 2.0 / 3.0 * x;
            double rat = 0.0;
            if (valid) {
                if (rk != 0.0) rat = fabs(x / rk - 1.0);
                else if (x != 0.0) rat = fabs(rk / x - 1.0);
            }
            rat = warp_maxd(rat);
            if (fabs(rat) < eps) {
                conv = true;
                break;
            }
        }
        if (!conv) redtl = 0.5 * redtl;
    }
    if (!conv) return -1;
    const double dtn = x;
    // extension of the phase temperature (nd = 1); halo = the unchanged neighbours
    const double hl = X.tm[lo - 1], hr = X.tm[hi + 1];
    double tm = X.tm[xi];
    redtl = 0.2 * sm_grid;
    conv = false;
    for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
        for (int it = 1; it <= 100; ++it) {
            ++total;
            const double rk = tm;
            double to = tm;
            to = L.sweep(to, hl, hr, 1, dtn, redtl);
            to = L.sweep(to, hl, hr, 1, dtn, redtl);
            to = 0.75 * rk + 0.25 * to;
            to = L.sweep(to, hl, hr, 1, dtn, redtl);
            to = 1.0 / 3.0 * rk + 2.0 / 3.0 * to;
            tm = to;
            double rat = 0.0;
            if (valid && rk != 0.0) rat = fabs(tm / rk - 1.0);
            rat = warp_maxd(rat);
            if (fabs(rat) < eps) {
                conv = true;
                break;
            }
        }
        if (!conv) redtl = 0.5 * redtl;
    }
    if (!conv) return -1;
    if (valid) {
        X.dt[xi] = dtn;
        X.tm[xi] = tm;
    }
    __syncwarp();
    return total;
}

// TEMP_EXTP, chphase.f:467-805 (1-D), one phase (im = 0 vapour, 1 liquid) on one warp;
// the two phases are independent and run on warps 0 and 1 at once.  Only cells with
// NPHI != 0 change; they lie in [xk0+lo, xk0+hi], held with one halo cell each side in
// shared memory.  temp_g: the phase temperature (global, k = 0..n+1).  Returns the number
// of pseudo-time iterations or -1 if the phase does not converge within kMaxHalvings
// halvings of the step.
__device__ int temp_extp(const Geo& g, const Phys& ph, Shared& sh, int xk0, int lo, int hi, int im, double* temp_g) {
    const int lane = threadIdx.x & 31;
    const double sm_grid = fmin(fmin(2.0 * 0.5, 2.0 * 0.5), 2.0 * g.hf);
    const double eps = 1e-4;
    XPhase& X = sh.xp[im];
    int total = 0;
    for (int i = lo - 1 + lane; i <= hi + 1; i += 32) {
        X.tm[i] = temp_g[xk0 + i];
        X.dt[i] = 0.0;   // DTEMPN: 0 outside the cells set below (halo included)
    }
    __syncwarp();
    for (int i = lo + lane; i <= hi; i += 32) {
        const double nph = sh.x_nphi[i];
        double d = 0.0;
        const int k = xk0 + i;
        const bool ca = ((fabs(nph) > 1.5 * sm_grid) && (nph != 0.0)) ||
                        ((fabs(sh.x_pcn[i] - 0.5) == 0.5) && (nph != 0.0));
        if (ca) {
            double dpz, dtdz;
            if (sh.x_nphi[i - 1] == 0.0) {
                dpz = (sh.x_nphi[i + 1] - nph) * g.vvdz(k + 1);
                dtdz = (X.tm[i + 1] - X.tm[i]) * g.vvdz(k + 1);
            } else if (sh.x_nphi[i + 1] == 0.0) {
                dpz = (nph - sh.x_nphi[i - 1]) * g.vvdz(k);
                dtdz = (X.tm[i] - X.tm[i - 1]) * g.vvdz(k);
            } else {
                dpz = 0.5 * (sh.x_nphi[i + 1] - sh.x_nphi[i - 1]) * g.vvdz(k);
                dtdz = 0.5 * (X.tm[i + 1] - X.tm[i - 1]) * g.vvdz(k);
            }
            const double dalphi = (0.0 + 0.0) + dpz * dpz;
            if (dalphi != 0.0) {
                const double nz = 1.0;
                if (im == 1) d = (0.0 + 0.0) + nz * dtdz * sh.x_psih[i];
                else d = (0.0 + 0.0) + nz * dtdz * (1 - sh.x_psih[i]);
            }
        } else if (((fabs(nph) <= 1.5 * sm_grid) || (fabs(sh.x_pcn[i] - 0.5) != 0.5)) &&
                   ((nph != 1e-7) && (nph != 0.0))) {
            if (im == 1) d = (X.tm[i] - ph.t_sat) / nph * sh.x_psih[i];
            else d = (X.tm[i] - ph.t_sat) / nph * (1.0 - sh.x_psih[i]);
        }
        X.dt[i] = d;
    }
    __syncwarp();
    if (hi - lo + 1 <= 32) {
        const int it = extp_registers(g, sh, X, xk0, lo, hi, im, eps);
        if (it < 0) return -1;
        total += it;
    } else {
        // extension of the normal gradient (nd = 0)
        double redtl = 0.2 * sm_grid;
        bool conv = false;
        for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
            for (int it = 1; it <= 100; ++it) {
                ++total;
                for (int i = lo + lane; i <= hi; i += 32) X.dtrk[i] = X.dt[i];
                __syncwarp();
                extp_sweep(g, sh, X, xk0, lo, hi, X.dt, im, redtl, 0);
                extp_sweep(g, sh, X, xk0, lo, hi, X.dt, im, redtl, 0);
                for (int i = lo + lane; i <= hi; i += 32) X.dt[i] = 0.75 * X.dtrk[i] + 0.25 * X.dt[i];
                __syncwarp();
                extp_sweep(g, sh, X, xk0, lo, hi, X.dt, im, redtl, 0);
                double rat = 0.0;
                for (int i = lo + lane; i <= hi; i += 32) {
                    const double v = 1.0 / 3.0 * X.dtrk[i] + 2.0 / 3.0 * X.dt[i];
                    X.dt[i] = v;
                    if (X.dtrk[i] != 0.0) rat = fmax(fabs(v / X.dtrk[i] - 1.0), rat);
                    else if (v != 0.0) rat = fmax(fabs(X.dtrk[i] / v - 1.0), rat);
                }
                rat = warp_maxd(rat);
                __syncwarp();
                if (fabs(rat) < eps) {
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
        for (int halving = 0; halving <= kMaxHalvings && !conv; ++halving) {
            for (int it = 1; it <= 100; ++it) {
                ++total;
                for (int i = lo - 1 + lane; i <= hi + 1; i += 32) {
                    X.trk[i] = X.tm[i];
                    X.to[i] = X.tm[i];
                }
                __syncwarp();
                extp_sweep(g, sh, X, xk0, lo, hi, X.to, im, redtl, 1);
                extp_sweep(g, sh, X, xk0, lo, hi, X.to, im, redtl, 1);
                for (int i = lo + lane; i <= hi; i += 32) X.to[i] = 0.75 * X.trk[i] + 0.25 * X.to[i];
                __syncwarp();
                extp_sweep(g, sh, X, xk0, lo, hi, X.to, im, redtl, 1);
                double rat = 0.0;
                for (int i = lo + lane; i <= hi; i += 32) {
                    const double v = 1.0 / 3.0 * X.trk[i] + 2.0 / 3.0 * X.to[i];
                    X.to[i] = v;
                    X.tm[i] = v;
                    if (X.trk[i] != 0.0) rat = fmax(fabs(v / X.trk[i] - 1.0), rat);
                }
                rat = warp_maxd(rat);
                __syncwarp();
                if (fabs(rat) < eps) {
                    conv = true;
                    break;
                }
            }
            if (!conv) redtl = 0.5 * redtl;
        }
        if (!conv) return -1;
    }
    for (int i = lo + lane; i <= hi; i += 32) temp_g[xk0 + i] = X.tm[i];
    __syncwarp();
    return total;
}

// TEMP_GRAD (chphase.f:55-368) with PHINSINTP, TEMP_EXTP, TEMPASSIGN, TF_GRAD,
// VOL_TOT_MFDOT and CAL_PSI_TMP(1); 1-D.  All threads call it; the band work runs on warp
// 0.  Returns the TEMP_EXTP iteration count, or a negative lica_status.
__device__ int temp_grad(const Geo& g, const Phys& ph, Col& c, Shared& sh, double L, double dtconst) {
    const int n = g.n, nf = g.nf;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *temp0 = c.a[S_TEMP0], *temp1 = c.a[S_TEMP1];
    FOR_K(0, nf + 6) c.mflvs[k] = 0.0;
    FOR_K(0, nf + 1) {
        c.sfgas[k] = 0.0;
        c.sfgas2[k] = 0.0;
    }
    FOR_K(0, n + 1) {
        c.imask[k] = 0;
        temp0[k] = c.t[k];
        temp1[k] = c.t[k];
    }
    __syncthreads();
    lvs::Win* s = &sh.win;
    lvs::Ctx cx;
    cx.s = s;
    int st = 0;
    if (warp == 0) {
        st = lvs::load_band_window(cx, lane, n, L, c.phi, c.layer);
        if (lane == 0) sh.ibuf[0] = st;
        // NPHI, PSIH, PSI_CN of the flow cells xk0 .. xk0+XR-1 (the window's flow range)
        for (int j = lane; j < XR; j += 32) {
            const int k = cx.kw0 + j;
            sh.x_nphi[j] = 0.0;
            sh.x_psih[j] = 0.0;
            sh.x_pcn[j] = (k >= 0 && k <= n + 1) ? c.psi_cn[k] : 0.0;
        }
    }
    __syncthreads();
    st = sh.ibuf[0];
    if (st != LICA_OK) return -st;
    const int xk0 = cx.kw0;   // valid on warp 0; shared below through ibuf
    if (warp == 0) {
        // (1) NPHI / PSIH of the flow cells of the band (:147-211), in list order; every
        // band cell's flow cell lies in [xk0+2, xk0+66]
        if (lane == 0) {
            int ic = 0;
            for (int j = s->lstart[1]; j < s->lstart[lvs::NN2 + 1]; ++j) {
                const int k = cx.w0 + s->lst[j];
                const int kk = g.kcoump_vel(k);
                const int x = kk - xk0;
                if (sh.x_nphi[x] == 0.0) {
                    const int k1 = g.kcou2(kk), k2 = g.kcoump2(kk);   // PHINSINTP's KCOU2(KO), KCOUMP2(KO)
                    const double zd = (k1 == k2) ? 0.0 : (g.zp(kk) - g.zpf(k1)) / (g.zpf(k2) - g.zpf(k1));
                    const double a1 = cx.p(k1), a2 = cx.p(k2);
                    const double c00 = a1 * (1.0 - 0.5) + a1 * 0.5;
                    const double c01 = a2 * (1.0 - 0.5) + a2 * 0.5;
                    const double c0 = c00 * (1.0 - 0.5) + c00 * 0.5;
                    const double c1 = c01 * (1.0 - 0.5) + c01 * 0.5;
                    double nsphi = c0 * (1.0 - zd) + c1 * zd;
                    if (nsphi > 0.0) ic = 1;
                    if (nsphi < 0.0) ic = 0;
                    if (a1 == 0.0 || a2 == 0.0) nsphi = 0.0;
                    sh.x_nphi[x] = 1e-7;
                    sh.x_nphi[x] = nsphi;
                    if (fabs(sh.x_pcn[x] - 0.5) != 0.5) sh.x_psih[x] = (double)ic;
                    else sh.x_psih[x] = sh.x_pcn[x];
                }
            }
            for (int j = s->lstart[lvs::N_MAX]; j < s->lstart[lvs::N_MAX + 1]; ++j) {
                const int k = cx.w0 + s->lst[j];
                const int kk = g.kcoump_vel(k);
                const int x = kk - xk0;
                const double dx = 0.25, dy = 0.25;
                const double dz = g.zpf(k) - g.zp(kk);
                const double pre = s->phi[s->lst[j]] + sqrt(dx * dx + dy * dy + dz * dz);
                sh.x_nphi[x] = fmin(sh.x_nphi[x], pre);
                sh.x_psih[x] = sh.x_pcn[x];
            }
            // extension range: the cells with NPHI != 0
            int ka = n + 1, kb = 0;
            for (int j = s->lstart[1]; j < s->lstart[lvs::N_MAX + 1]; ++j) {
                const int kk = g.kcoump_vel(cx.w0 + s->lst[j]);
                if (sh.x_nphi[kk - xk0] != 0.0) {
                    ka = min(ka, kk);
                    kb = max(kb, kk);
                }
            }
            sh.ibuf[1] = ka;
            sh.ibuf[2] = kb;
            sh.ibuf[7] = xk0;
        }
    }
    __syncthreads();
    c.mark(PH_TEMPGRAD);
    {
        // (2) TEMP_EXTP: the vapour phase on warp 0, the liquid phase on warp 1 (one after the
        // other on warp 0 in a one-warp CTA)
        const int ka = sh.ibuf[1], kb = sh.ibuf[2], x0 = sh.ibuf[7];
        const int nw = (int)(blockDim.x >> 5);
        for (int phs = warp; phs < 2; phs += nw) {
            int it = 0;
            if (kb >= ka) it = temp_extp(g, ph, sh, x0, ka - x0, kb - x0, phs, phs ? temp1 : temp0);
            if (lane == 0) sh.ibuf[3 + phs * 2] = it;   // ibuf[3], ibuf[5]
            __syncwarp();
        }
    }
    __syncthreads();
    c.mark(PH_EXTP);
    if (warp == 0) {
        const int i0 = sh.ibuf[3], i1 = sh.ibuf[5];
        const int iters = (i0 < 0 || i1 < 0) ? -1 : i0 + i1;
        __syncwarp();
        if (lane == 0) sh.ibuf[3] = iters;
        __syncwarp();
        if (iters >= 0) {
            // (3) TF on layers 1..NN1 by TEMPASSIGN (chphase.f:372-463); tf0 in win.rk3, tf1
            // in win.alphio (window-indexed, 0 elsewhere).  TF_GRAD's central differences
            // read one slot past the band on either side -- past the wall where the band is
            // cut off there -- so those slots are zeroed too, not left to whatever the
            // shared memory held.
            for (int i = max(cx.blo - 1, 0) + lane; i <= min(cx.bhi + 1, lvs::WIN - 1); i += 32) {
                const int k = cx.w0 + i, m = s->layer[i];
                double v0 = 0.0, v1 = 0.0;
                if (m >= 1 && m <= lvs::NN1) {
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
                    v0 = temp0[kk] * (1.0 - zd) + temp0[kk2] * zd;
                    v1 = temp1[kk] * (1.0 - zd) + temp1[kk2] * zd;
                }
                s->rk3[i] = v0;
                s->alphio[i] = v1;
            }
            __syncwarp();
            // (4)-(6) TF_GRAD: MFDOT on layers 1..NN1-2
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int k = cx.w0 + i, m = s->layer[i];
                if (m >= 1 && m <= lvs::NN1 - 2) {
                    const double gz = 0.5 * (s->phi[i + 1] - s->phi[i - 1]) * cx.ssdzf;
                    const double agi = 1.0 / sqrt((0.0 + 0.0) + gz * gz);
                    const double dtz0 = 0.5 * (s->rk3[i + 1] - s->rk3[i - 1]) * cx.ssdzf;
                    const double dtdn0 = ((0.0 + 0.0) + dtz0 * gz) * agi;
                    const double dtz1 = 0.5 * (s->alphio[i + 1] - s->alphio[i - 1]) * cx.ssdzf;
                    const double dtdn1 = ((0.0 + 0.0) + dtz1 * gz) * agi;
                    const double mf = ph.ja * ph.prai * ph.rei * (-ph.tcp * dtdn1 + ph.tcm * dtdn0);
                    c.mflvs[k + 2] = mf;
                    s->mf[i] = mf;
                } else {
                    s->mf[i] = 0.0;
                }
            }
            // PSIF_MTP = CAL_PSIF_MTP(1, NN1) of the band (snapped band values, column fill)
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int m = s->layer[i];
                s->start[i] = (m >= 1 && m <= lvs::NN1) ? lvs::psif_band(s, i) : 0.0;
            }
            __syncwarp();
            {
                int ktop, kbot;
                lvs::window_crossings(cx, ktop, kbot);
                if (lane == 0) {
                    sh.ibuf[4] = ktop;
                    sh.ibuf[5] = kbot;
                }
            }
            __syncwarp();
            {
                const int ktop = sh.ibuf[4], kbot = sh.ibuf[5];
                double t1 = 1.0, t2 = 1.0;
                if (ktop >= 0) {
                    t1 = (cx.p(ktop) < 0.0) ? 0.0 : 1.0;
                    t2 = (cx.p(kbot + 1) < 0.0) ? 0.0 : 1.0;
                }
                for (int k = 1 + lane; k <= nf; k += 32) {
                    const int i = k - cx.w0;
                    double v;
                    if (cx.in(k) && s->layer[i] >= 1 && s->layer[i] <= lvs::NN1) v = s->start[i];
                    else if (ktop < 0) v = 1.0;
                    else v = (k > kbot) ? t2 : t1;
                    c.psif_mtp[k] = v;
                }
            }
            __syncwarp();
            // VOL_TOT_MFDOT: trial advance of layers 1..NN1-2 by the mass flux, reinit,
            // volume of CAL_PSIF_MTP(1) of the trial band, SFGAS / SFGAS2
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int m = s->layer[i];
                s->wf[i] = s->phi[i];   // ALPHI at entry
                if (m >= 1 && m <= lvs::NN1 - 2) {
                    const double mfd = (s->phi[i] > 0.0) ? s->mf[i] / ph.denr : s->mf[i];
                    const double a0 = s->phi[i];
                    double a = a0 - 2 * dtconst * mfd;
                    a = 0.75 * a0 + 0.25 * a;
                    a = a - dtconst * mfd;
                    a = 1.0 / 3.0 * a0 + 2.0 / 3.0 * a;
                    s->nv[i] = a;
                }
            }
            __syncwarp();
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int m = s->layer[i];
                if (m >= 1 && m <= lvs::NN1 - 2) s->phi[i] = s->nv[i];
            }
            __syncwarp();
            lvs::reinitialization(cx, lvs::NN2);
            {
                // the interface position of 0interface.dat (chphase.f:1419-1431): zpf(k) +
                // |phi(k)| of the last sign change over k = 1..N3FM of the trial phi (0 off
                // the band; phi(nf+1) is ALPHI_BC's ghost)
                int kb = 0;
                for (int i = lane; i < lvs::WIN; i += 32) {
                    const int k = cx.w0 + i;
                    if (k < 1 || k > nf) continue;
                    const double a = s->phi[i];
                    const double b = (i + 1 < lvs::WIN) ? s->phi[i + 1] : (k == nf ? s->ghost[3] : 0.0);
                    if (a * b < 0.0) kb = k;
                }
                for (int o = 16; o > 0; o >>= 1) kb = max(kb, __shfl_xor_sync(0xffffffffu, kb, o));
                if (lane == 0) sh.dbuf[5] = (kb > 0) ? g.zpf(kb) + fabs(s->phi[kb - cx.w0]) : 0.0;
            }
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int m = s->layer[i];
                s->nv[i] = (m >= 1 && m <= lvs::NN1) ? lvs::psif_band(s, i) : 0.0;
            }
            __syncwarp();
            {
                int ktop, kbot;
                lvs::window_crossings(cx, ktop, kbot);
                if (lane == 0) c.scal[4] = lvs::column_vapour_volume(cx, s->nv, ktop, kbot, 0.5 * 0.5 * g.hf);
            }
            for (int i = cx.blo + lane; i <= cx.bhi; i += 32) {
                const int k = cx.w0 + i, m = s->layer[i];
                if (m >= 1 && m <= lvs::NN1 - 2 && s->mf[i] != 0.0 && fabs(c.psif_mtp[k] - 0.5) != 0.5) {
                    const double d = -(s->nv[i] - c.psif_mtp[k]);
                    if (s->wf[i] > 0.0) {
                        c.sfgas[k] = -(s->nv[i] - c.psif_mtp[k]) * ph.denr;
                        c.sfgas2[k] = d;
                    } else {
                        c.sfgas[k] = d;
                        c.sfgas2[k] = d;
                    }
                }
            }
        }
    }
    __syncthreads();
    const int iters = sh.ibuf[3];
    if (iters < 0) return iters == -1 ? -LICA_NOT_CONVERGED : iters;
    // (7) CAL_PSI_TMP(1) and IMASK_PH on the z faces (chphase.f:297-357)
    double* psi_tmp = c.a[S_PSITMP];
    FOR_K(1, n) {
        const double v = col::box_mean(c.psif_mtp, nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
        psi_tmp[k] = (v <= 1e-3) ? 0.0 : (v >= 0.999 ? 1.0 : v);
    }
    __syncthreads();
    FOR_K(2, n) c.imask[k] = (fabs(psi_tmp[k] - psi_tmp[k - 1]) != 0.0) ? 1 : 0;
    __syncthreads();
    return iters;
}

// CAL_CONTINUITY2, 1d.f:3006-3169 (the REGION of CAL_CONTINUITY is unchanged: same PSI_CN).
__device__ void cal_continuity2(const Geo& g, const Phys& ph, Col& c) {
    const int n = g.n, nf = g.nf;
    double *psi_z = c.a[S_PSIZ], *psi_c = c.a[S_PSIC];
    const int* reg = c.region + 1;
    FOR_K(1, n) {
        if (k >= 2) {
            double v = psi_z[k];
            if (reg[k] == 2)
                v = v - col::box_mean(c.sfgas2, nf, g.kcou2(k), g.kcou1(k + 1), g.zp(k - 1), g.zp(k), g.hf);
            psi_z[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
        }
        double v = psi_c[k];
        if (reg[k] == 2) v = v - col::box_mean(c.sfgas2, nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
        psi_c[k] = (v > 1.0) ? 1.0 : (v < 0.0 ? 0.0 : v);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        psi_z[1] = psi_z[2];
        psi_z[n + 1] = psi_z[n];
        psi_c[1] = psi_c[2];
        psi_c[n + 1] = psi_c[n];
    }
    __syncthreads();
}

// One substep of RHSNLHS (1d.f:1444-1600).  Returns the TEMP_EXTP iterations or a negative
// lica_status.
__device__ void pressure_correction(const Geo& g, const Phys& ph, Col& c, Shared& sh, double dtconst,
                                    double dtconsti, const double* denf_zi);

__device__ int rhsnlhs(const Geo& g, const Phys& ph, Col& c, Shared& sh, double L, int msub, int m_step) {
    const int n = g.n;
    const double dt = c.scal[0];
    const double alpha = 0.5 * (c_gamma[msub] + c_ro[msub]);
    const double acoef = alpha * dt;
    const double dtconst = 2. * alpha * dt;
    const double dtconsti = 1. / dtconst;
    double *rhs1 = c.a[S_RHS1], *rhsps = c.a[S_RHSPS], *rk3zo = c.a[S_RK3ZO];
    const double *denf_zi = c.a[S_DENFZI], *psi_c = c.a[S_PSIC], *df_c = c.a[S_DFC];
    c.mark(PH_DT);
    cal_continuity(g, ph, c, dtconst);
    cal_cont_bc(g, ph, c);
    c.mark(PH_CONT);
    // PASSIVE_SCALAR (1d.f:3630-3707)
    int iters = 0;
    if (ph.iphs == 1 && m_step != 1) {
        FOR_K(1, n) {
            const double r = (c_gamma[msub] * c.t[k] * (c.w[k + 1] - c.w[k]) * g.vvdz(k)) * dt;
            double densc, denscf;
            if (c.psi_cn[k] > 0.5) {
                densc = ph.denscm + ph.densc_diff;
                denscf = densc;
            } else {
                densc = ph.denscm;
                denscf = densc;
            }
            rhsps[k] = ((densc - denscf) * c.t[k] + r) / denscf;
        }
        __syncthreads();
        lhsps(g, ph, c, alpha, dt);   // substitute for the undefined LHSPS2
        c.mark(PH_ENERGY);
        iters = temp_grad(g, ph, c, sh, L, dtconst);
        if (iters < 0) return iters;
        c.mark(PH_TEMPGRAD);
        cal_continuity2(g, ph, c);
        cal_cont_bc(g, ph, c);
        c.mark(PH_CONT2);
    } else {
        FOR_K(1, n) {
            const double anps = 0.0, alps = 0.0, anpso = 0.0, tgr = 0.0;
            const double densc = ph.denscm + ph.densc_diff * c.psi_cn[k];
            const double uu = 0.5 * (c.w[k + 1] + c.w[k]);
            const double ameant1 = densc * uu * tgr;
            const double tct = ph.tcm + ph.tc_diff * ((df_c[k] - ph.denm) * (1.0 / ph.den_diff));
            const double tcb = ph.tcm + ph.tc_diff * ((df_c[k - 1] - ph.denm) * (1.0 / ph.den_diff));
            const double ameant2 = (1.0 / (ph.re * ph.prm)) * (tct - tcb) * g.ssdz(k) * tgr;
            const double r = ((c_gamma[msub] * anps + c_ro[msub] * anpso) + 2. * alpha * alps +
                              2. * alpha * (ameant1 - ameant2)) *
                             dt;
            const double denscf = ph.denscm + ph.densc_diff * psi_c[k];
            rhsps[k] = ((densc - denscf) * c.t[k] + r) / denscf;
        }
        __syncthreads();
        lhsps(g, ph, c, alpha, dt);
        c.mark(PH_ENERGY);
    }
    // RHSZ (1d.f:1603-1745) and RHS1 = RHS1 / rho - W (1564-1568)
    {
        const double *df_z = c.a[S_DFZ], *vf_z = c.a[S_VFZ];
        const double* w = c.w;
        FOR_K(2, n) {
            const double wt = 0.5 * (w[k + 1] + w[k]);
            const double wb = 0.5 * (w[k] + w[k - 1]);
            const double anzz = (df_z[k] * (wt * wt) - df_z[k - 1] * (wb * wb)) * g.vvdz(k);
            const double anz = -0.0 - 0.0 - anzz;
            const double alz5 = (w[k + 1] - w[k]) * g.ssdz(k);
            const double alz6 = (w[k] - w[k - 1]) * g.ssdz(k - 1);
            const double alzz = (vf_z[k] * alz5 - vf_z[k - 1] * alz6) * g.vvdz(k);
            const double alz_sum1 = 0.0 + 0.0 + alzz + alzz;
            const double alz_sum2 = 0.0 + 0.0;
            const double pgr_z = (c.p[k] - c.p[k - 1]) * g.vvdz(k);
            const double den_zn = ph.denm + ph.den_diff * c.psi_zn[k];
            const double rk3z = anz + alz_sum2;
            const double cn2z = alz_sum1;
            const double sur_z = 0.0, buoy = 0.0, pmi = 0.0;
            double r = den_zn * w[k] + (c_gamma[msub] * rk3z + c_ro[msub] * rk3zo[k] + 2. * alpha * cn2z +
                                        2. * alpha * (sur_z - pgr_z) - 2. * alpha * buoy - 2. * alpha * (pmi + 0.0)) *
                                           dt;
            if (ph.iphs == 1 && c.imask[k] == 1 && fabs(c.psi_zn[k] - 0.5) != 0.5)
                r = r + c_gamma[msub] * dt * den_zn * w[k] *
                            ((0.0 - 0.0) * 1.0 + (0.0 - 0.0) * 1.0 + (wt - wb) * g.vvdz(k));
            rhs1[k] = r * denf_zi[k] - w[k];
            rk3zo[k] = rk3z;
        }
        __syncthreads();
        c.mark(PH_RHSZ);
    }
    // LHSW (1d.f:1749-1809)
    {
        double *ak = c.a[S_AK], *bk = c.a[S_BK], *ck = c.a[S_CK], *gk = c.a[S_GK];
        const double* vf_z = c.a[S_VFZ];
        FOR_K(2, n) {
            const double dk1 = 2. * acoef * denf_zi[k] * vf_z[k - 1] * g.akw(k);
            const double dk3 = 2. * acoef * denf_zi[k] * vf_z[k] * g.ckw(k);
            const double dk2 = -dk1 - dk3;
            ak[k] = dk1;
            ck[k] = dk3;
            bk[k] = 1. + dk2;
            gk[k] = rhs1[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) thomas(ak, bk, ck, gk, c.a[S_GAM], 2, n);
        __syncthreads();
        FOR_K(2, n) c.w[k] = gk[k] + c.w[k];
        __syncthreads();
        c.mark(PH_LHSW);
    }
    // BC + BC_FLUX (1d.f:1812-1923)
    if (threadIdx.x == 0) {
        c.w[1] = 0.0;
        c.w[n + 1] = c.w[n];
        double qq3 = 0.0;
        qq3 = qq3 + (c.w[n + 1] - c.w[1]) * 1.0 * 1.0;
        double aa = 0.0;
        aa = aa + 2. * 1.0 * 1.0;
        const double ubc_avg = -qq3 / aa;
        c.w[1] = 0.0;
        c.w[n + 1] = c.w[n + 1] + ubc_avg;
    }
    __syncthreads();
    // FSM_CHOI (1d.f:3365-3400), then PRESSURE_CORRECTION
    FOR_K(2, n) c.w[k] = c.w[k] + dtconst * ((c.p[k] - c.p[k - 1]) * g.vvdz(k)) * denf_zi[k];
    __syncthreads();
    pressure_correction(g, ph, c, sh, dtconst, dtconsti, denf_zi);
    c.mark(PH_PRESS);
    return iters;
}

// PRESSURE_CORRECTION (1d.f:3403-3488): DIVGS (3180-3303), POISSON (3492-3578), UCALC
// (3582-3627) and the shift P -= P(1) with the ghost copies.  All threads call it.
__device__ void pressure_correction(const Geo& g, const Phys& ph, Col& c, Shared& sh, double dtconst,
                                    double dtconsti, const double* denf_zi) {
    const int n = g.n;
    {
        double* divg = c.a[S_DIVG];
        FOR_K(1, n) {
            double d = (k <= n - 1) ? (c.w[k + 1] - c.w[k]) * g.ssdz(k) : 0.0;
            if (ph.iphs == 1) {
                const double ssum = col::box_mean(c.sfgas, g.nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
                d = d - ssum * (ph.den_diff / (ph.denp * ph.denm));
            }
            if (k >= 2) d = d * dtconsti;
            divg[k] = d;
        }
        __syncthreads();
        // POISSON (1d.f:3492-3578)
        double *ak = c.a[S_AK], *bk = c.a[S_BK], *ck = c.a[S_CK], *gk = c.a[S_GK];
        FOR_K(1, n) {
            const double fixkl = (k == 1) ? 1.0 : 0.0;
            const double a = g.vvdz(k) * g.ssdz(k) * denf_zi[k] * (1.0 - fixkl);
            const double cc = g.vvdz(k + 1) * g.ssdz(k) * denf_zi[k + 1];
            ak[k] = a;
            ck[k] = cc;
            bk[k] = -(a + cc);
            gk[k] = divg[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            thomas(ak, bk, ck, gk, c.a[S_GAM], 1, n);
            for (int k = 1; k <= n; ++k) c.p[k] = gk[k];
            c.p[0] = c.p[1];
            c.p[n + 1] = c.p[n];
        }
        __syncthreads();
        // UCALC (1d.f:3582-3627) and the reference shift P -= P(1) (1d.f:3431-3446)
        FOR_K(2, n) c.w[k] = c.w[k] - dtconst * (c.p[k] - c.p[k - 1]) * g.vvdz(k) * denf_zi[k];
        __syncthreads();
        if (threadIdx.x == 0) {
            c.w[1] = 0.0;
            c.w[n + 1] = c.w[n];
            sh.dbuf[0] = c.p[1];
        }
        __syncthreads();
        const double phiref = sh.dbuf[0];
        FOR_K(1, n) c.p[k] = c.p[k] - phiref;
        __syncthreads();
        if (threadIdx.x == 0) c.p[0] = c.p[1];
        __syncthreads();
    }
}

// One time step (1d.f:190-250).  Returns a lica_status.
__device__ int column_step(const Geo& g, const Phys& ph, Col& c, Shared& sh, double L) {
    const int n = g.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m_step = (int)c.scal[2] + 1;
    __syncthreads();
    if (tid == 0) c.scal[2] = c.scal[2] + 1.0;
    if (m_step == 1) FOR_K(0, g.nf + 6) c.mflvs[k] = 0.0;
    // DETERMINE_DT + CFL (1d.f:683-817, 1325-1373)
    {
        const double dt = c.scal[0];
        double dsrc = 1000.0, cfl = 0.0;
        FOR_K(1, n) {
            if (ph.time_st != 0.0 && fabs(c.psi_cn[k] - 0.5) < 0.5) {
                const double dx1 = fmin(1.0, g.sdz(k));
                const double t1 = 0.5 * dx1 / sqrt(ph.time_st / dx1 + ph.time_gv * dx1);
                const double dx2 = fmax(1.0, g.sdz(k));
                const double t2 = 0.5 * dx2 / sqrt(ph.time_st / dx2 + ph.time_gv * dx2);
                dsrc = fmin(dsrc, fmin(t1, t2));
            }
            const double c3 = fabs(c.w[k] + c.w[k + 1]) * g.ssdz(k);
            cfl = fmax(0.5 * ((0.0 + 0.0) + c3) * dt, cfl);
        }
        dsrc = block_min(dsrc, sh);
        cfl = block_max(cfl, sh);
        if (ph.time_st == 0.0) dsrc = 1000000.0;
        __syncthreads();
        if (tid == 0) {
            const double dt_old = dt;
            const double cfl_surf = dt / dsrc;
            const double cfl_sum = 0.5 * (cfl + sqrt(cfl * cfl + 4.0 * cfl_surf));
            double dtn = dt * ph.cflmax / cfl_sum;
            if (dtn / dt_old > 2.0) dtn = dt_old * 1.2;
            c.scal[0] = dtn;
            c.stats[0] = cfl;
        }
        __syncthreads();
    }
    FOR_K(0, n + 1) c.a[S_RK3ZO][k] = 0.0;
    __syncthreads();
    double iters = 0.0, subcycles = 0.0, imass = 0.0, dvmax = 0.0;
    for (int msub = 1; msub <= 3; ++msub) {
        const int it = rhsnlhs(g, ph, c, sh, L, msub, m_step);
        if (it < 0) return -it;
        iters += it;
        // CONVRGE1 (1d.f:3306-3362)
        double dv = 0.0;
        FOR_K(1, n) {
            double d = (c.w[k + 1] - c.w[k]) * g.ssdz(k);
            if (ph.iphs == 1) {
                const double ssum = col::box_mean(c.sfgas, g.nf, g.kcou2(k), g.kcou1(k + 1), g.z(k), g.z(k + 1), g.hf);
                d = d - ssum * (ph.den_diff / ph.denp);
            }
            dv = fmax(fabs(d), dv);
        }
        dvmax = block_max(dv, sh);
        c.mark(PH_CONV);
        // TRANSPORT + GRID_COUPLING(0) on warp 0
        __syncthreads();
        const double dtconst = 2. * (0.5 * (c_gamma[msub] + c_ro[msub])) * c.scal[0];
        if (warp == 0) {
            lvs::Params P{ph.iphs, (m_step == 1 && msub == 1) ? 1 : 0, m_step, ph.mglobal, ph.denr, dtconst};
            double lst[4] = {0, 0, 0, 0};
            double* st4 = c.stats + 4;   // scratch for the transport statistics
            const int st = lvs::transport_column(&sh.win, lane, n, L, c.phi, c.layer, c.psif, c.wo, c.w, c.mflvs,
                                                 &c.scal[3], c.scal[4], c.psi_cn, c.psi_zn, st4, P, g.cg);
            __syncwarp();
            if (lane == 0) {
                for (int q = 0; q < 4; ++q) lst[q] = st4[q];
                sh.ibuf[6] = st;
                sh.dbuf[1] = lst[0];
                sh.dbuf[2] = (lst[0] > 0) ? lst[3] : 0.0;
            }
        }
        __syncthreads();
        c.mark(PH_TRANSPORT);
        if (sh.ibuf[6] != LICA_OK) return sh.ibuf[6];
        subcycles += sh.dbuf[1];
        imass += sh.dbuf[2];
    }
    __syncthreads();
    if (tid == 0) {
        c.scal[1] = c.scal[1] + c.scal[0];
        double zi = 0.0;
        for (int k = 1; k < g.nf; ++k)
            if (c.layer[k + 2] > 0 && c.layer[k + 3] > 0 && c.phi[k + 2] < 0.0 && c.phi[k + 3] >= 0.0) {
                zi = g.zpf(k) - c.phi[k + 2] * (g.zpf(k + 1) - g.zpf(k)) / (c.phi[k + 3] - c.phi[k + 2]);
                break;
            }
        c.stats[1] = dvmax;
        c.stats[2] = iters;
        c.stats[3] = subcycles;
        c.stats[4] = imass;
        c.stats[5] = zi;
        c.stats[6] = c.scal[4];
        c.stats[7] = c.scal[0];
    }
    __syncthreads();
    return LICA_OK;
}

// NTH threads per column; one CTA per SM is enough for the register budget the sequential
// parts want (no spills), more columns per SM come from smaller NTH.
template <int NTH>
// The 64-thread form is bounded for 5 CTAs per SM (about 200 registers): latency-bound
// columns gain more from columns in flight than they lose to a few spilled registers.
__global__ void __launch_bounds__(NTH, NTH == 32 ? 8 : (NTH == 64 ? 5 : 1)) k_column_steps(const __grid_constant__ Args A) {
    __shared__ Shared sh;
    extern __shared__ double dsm[];   // 5 (n+2) doubles when A.tri_smem
    if ((int)blockIdx.x >= A.ncol) return;
    const int col = A.order ? A.order[blockIdx.x] : (int)blockIdx.x;
    int n;
    double L;
    Phys ph;
    size_t of, op, oq, od, oi;
    if (A.desc) {
        const ColDesc& D = A.desc[col];
        n = D.n;
        L = D.L;
        ph = D.ph;
        of = D.off_f;
        op = D.off_p;
        oq = D.off_q;
        od = D.off_d;
        oi = D.off_i;
    } else {
        n = A.n;
        L = A.L;
        ph = A.ph;
        const size_t sf = (size_t)n + 2, sq = 2 * (size_t)n + 2;
        of = col * sf;
        op = col * (2 * (size_t)n + 7);
        oq = col * sq;
        od = col * (NFLOW * sf + sq);
        oi = col * (sf + 2);
    }
    const int nf = 2 * n;
    const size_t sf = (size_t)n + 2;
    Col c;
    c.w = A.w + of;
    c.p = A.p + of;
    c.t = A.t + of;
    c.psi_cn = A.psi_cn + of;
    c.psi_zn = A.psi_zn + of;
    c.wo = A.wo + of;
    c.imask = A.imask + of;
    c.phi = A.phi + op;
    c.layer = A.layer + op;
    c.mflvs = A.mflvs + op;
    c.psif = A.psif + oq;
    c.sfgas = A.sfgas + oq;
    c.sfgas2 = A.sfgas2 + oq;
    c.scal = A.scal + col * 5;
    c.stats = A.stats + col * 8;
    (void)nf;
    double* d = A.dscr + od;
    for (int q = 0; q < NFLOW; ++q) c.a[q] = d + q * sf;
    c.psif_mtp = d + NFLOW * sf;
    if (A.tri_smem && n <= A.tri_cap) {
        // the Thomas coefficient, right-hand-side and elimination arrays: thread 0 walks
        // them sequentially, so they are kept at shared-memory latency
        c.a[S_AK] = dsm;
        c.a[S_BK] = dsm + sf;
        c.a[S_CK] = dsm + 2 * sf;
        c.a[S_GK] = dsm + 3 * sf;
        c.a[S_GAM] = dsm + 4 * sf;
    }
    share_scratch(c);
    c.region = A.iscr + oi;
    c.prof = A.prof ? A.prof + (size_t)col * PH_COUNT : nullptr;
    c.t0 = clock64();
    const Geo g(n, L, A.has_geo ? &A.geo : nullptr);
    int st = LICA_OK;
    double* hist = A.hist ? A.hist + (size_t)col * A.hist_cap * HIST_REC : nullptr;
    for (int s = 0; s < A.nsteps && st == LICA_OK; ++s) {
        // thread 0 alone writes and reads sh.dbuf[5] (place) and the history record
        double time0 = 0.0;
        if (threadIdx.x == 0) {
            sh.dbuf[5] = 0.0;
            time0 = c.scal[1];
        }
        st = column_step(g, ph, c, sh, L);
        if (hist && s < A.hist_cap && threadIdx.x == 0 && st == LICA_OK) {
            double* r = hist + (size_t)s * HIST_REC;
            r[0] = time0;
            r[1] = sh.dbuf[5];
            r[2] = c.scal[4];
            r[3] = c.scal[0];
        }
    }
    if (threadIdx.x == 0) A.status[col] = st;
}

// Single routines of the step on a batch of equal columns, for hosts that call the
// reference's subroutines one at a time: the step kernel's own device code, one CTA per
// column.
enum { RT_TEMP_GRAD = 0, RT_PRESSURE_CORRECTION = 1 };

struct RoutineArgs {
    int ncol, n, routine;
    double L, dtconst;
    Phys ph;
    double *w, *p, *t, *psi_cn, *phi, *mflvs, *sfgas, *sfgas2, *vol;
    const double* denf_zi;
    int *layer, *imask, *status, *iters;
    double* dscr;   // NFLOW (n+2) + 2n+2 doubles per column
};

__global__ void __launch_bounds__(NT_DEFAULT, 1) k_col_routine(const __grid_constant__ RoutineArgs A) {
    __shared__ Shared sh;
    const int col = blockIdx.x;
    if (col >= A.ncol) return;
    const int n = A.n;
    const size_t sf = (size_t)n + 2, sp = 2 * (size_t)n + 7, sq = 2 * (size_t)n + 2;
    Col c{};
    double* d = A.dscr + col * (NFLOW * sf + sq);
    for (int q = 0; q < NFLOW; ++q) c.a[q] = d + q * sf;
    c.psif_mtp = d + NFLOW * sf;
    c.scal = c.a[S_SPARE4];   // VOL_TOT_IPHS in c.scal[4]
    const Geo g(n, A.L);
    if (A.routine == RT_TEMP_GRAD) {
        c.t = A.t + col * sf;
        c.psi_cn = A.psi_cn + col * sf;
        c.phi = A.phi + col * sp;
        c.layer = A.layer + col * sp;
        c.mflvs = A.mflvs + col * sp;
        c.sfgas = A.sfgas + col * sq;
        c.sfgas2 = A.sfgas2 + col * sq;
        c.imask = A.imask + col * sf;
        if (threadIdx.x == 0) {
            c.scal[4] = A.vol[col];
            sh.dbuf[5] = 0.0;
        }
        __syncthreads();
        const int it = temp_grad(g, A.ph, c, sh, A.L, A.dtconst);
        __syncthreads();
        if (threadIdx.x == 0) {
            A.status[col] = it < 0 ? -it : LICA_OK;
            A.iters[col] = it < 0 ? 0 : it;
            A.vol[col] = c.scal[4];
        }
    } else {
        c.w = A.w + col * sf;
        c.p = A.p + col * sf;
        c.sfgas = A.sfgas + col * sq;
        pressure_correction(g, A.ph, c, sh, A.dtconst, 1. / A.dtconst, A.denf_zi + col * sf);
        if (threadIdx.x == 0) A.status[col] = LICA_OK;
    }
}

}  // namespace colk
}  // namespace lica

using namespace lica;

namespace {

colk::Phys make_phys(const lica_col_props* p) {
    colk::Phys ph;
    const double pi = std::acos(-1.0);
    ph.re = p->re;
    ph.rei = 1.0 / ph.re;
    ph.denm = 1.0;
    ph.denp = p->denr;
    ph.den_diff = ph.denp - ph.denm;
    ph.vism = 1.0 * ph.rei;
    ph.visp = p->visr * ph.rei;
    ph.denscm = ph.denm * 1.0;
    ph.denscp = ph.denscm * (p->denr * p->scr);
    ph.densc_diff = ph.denscp - ph.denscm;
    ph.tcm = 1.0;
    ph.tcp = p->tcr;
    ph.tc_diff = ph.tcp - ph.tcm;
    ph.prm = p->prm;
    ph.prai = 1.0 / p->prm;
    ph.surf = (p->weber == 0.0) ? 0.0 : 1.0 / p->weber;
    ph.gravity = (p->fr == 0.0) ? 0.0 : 1.0 / (p->fr * p->fr);
    ph.time_st = ph.surf * pi / (ph.denm + ph.denp);
    ph.time_gv = ph.den_diff / (ph.denm + ph.denp) * ph.gravity / pi;
    ph.denr = p->denr;
    ph.ja = p->jakob;
    ph.t_sat = p->t_sat;
    ph.cflmax = p->cflmax;
    ph.iphs = p->iphs;
    ph.mglobal = p->mglobal;
    return ph;
}

// Library-owned device buffers and streams are kept per device (ordinals 0..63), so a process
// that drives several GPUs gets each one's own.
constexpr int kMaxDevices = 64;
struct ScratchCache {
    std::mutex mu;
    void* ptr = nullptr;
    size_t bytes = 0;
};
int current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
    return dev;
}
ScratchCache& scratch_cache(int dev) {
    static ScratchCache s[kMaxDevices];
    return s[dev];
}

// per-phase cycle profile target (device array of COLUMN_PHASES * ncol int64) or null
long long* g_col_prof = nullptr;
// interface history target (device array of 4 * capacity doubles per column) or null
double* g_col_hist = nullptr;
int g_col_hist_cap = 0;


// Host-side initial state (runs once, before the time loop).
double h_zp(double h, int n, int k) {
    if (k <= 0) return 0.0;
    if (k >= n + 1) return n * h;
    return (k - 1) * h + 0.5 * h;
}

double h_box_mean(const double* f, int nf, int k1, int k2, double z1, double z2, double hf) {
    const double ssdzf = 1.0 / hf;
    double sum = 0.0, volf = 0.0;
    for (int rep = 0; rep < 4; ++rep)
        for (int kk = k1; kk <= k2; ++kk) {
            const double v = f[kk < 1 ? 1 : (kk > nf ? nf : kk)];
            const double za = (kk - 1) * hf, zb = kk * hf;
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
    return sum / volf;
}

}  // namespace

extern "C" {

// MAKEFLD (1d.f:821-946, IPHS = 1), LVSINIT (two_phase.f:116-388) and GRID_COUPLING(1) for
// a planar film.  LVSINIT's band generation from the candidate cells |phi| <= CRI reduces,
// for one plane, to: S-tube = the two cells around the interface, layer m at m-1 cells
// from it (never k = 1 or nf+1), phi = the signed distance ASSIGN_LVS gives; PSIF is
// CAL_PSIF_MTP(1, N_MAX) with the column fill, the vapour volume its (1 - PSIF) sum.
// geo: the flow grid of a stretched column (host arrays), or null for the uniform one.
static int column_init(int32_t n, double length, double z0, const lica_col_props* props,
                       const lica_col_geometry* geo, lica_col_state* st) {
    if (n < 8 || !(length > 0.0) || !props || !st || !st->w || !st->p || !st->t || !st->psi_cn || !st->psi_zn ||
        !st->phi || !st->layer || !st->psif || !st->wo || !st->mflvs || !st->sfgas || !st->sfgas2 || !st->imask ||
        !st->scal || !st->stats)
        return LICA_BAD_ARG;
    const int nf = 2 * n;
    const double h = length / n, hf = length / nf;
    auto zp = [&](int k) { return geo ? geo->zp[k] : h_zp(h, n, k); };
    auto zc = [&](int k) { return geo ? geo->z[k] : (k - 1) * h; };
    for (int k = 0; k <= n + 1; ++k) {
        st->w[k] = st->p[k] = st->t[k] = st->psi_cn[k] = st->psi_zn[k] = st->wo[k] = 0.0;
        st->imask[k] = 0;
    }
    for (int k = 1; k <= n; ++k) {
        const double pbody = (zp(k) - z0) + 1e-12;
        if (pbody > 0.0) {
            st->t[k] = 1.0;
            st->w[k] = 1.0;
            st->w[n + 1] = 1.0;
        } else {
            st->t[k] = 16.47 * zp(k);
            st->t[0] = 0.0;
            st->w[k] = 0.0;
            st->w[1] = 0.0;
        }
    }
    auto assign = [&](int k) { return (((k - 1) * hf + 0.5 * hf) - z0) + 1e-12; };
    // the one crossing among the candidates |phi| <= CRI = 1.2 MAX(SDXF,SDYF,SDZF)
    const double cri = 1.2 * std::max(std::max(0.5, 0.5), hf);
    int ks = -1, ncross = 0;
    for (int k = 1; k < nf; ++k) {
        const double a = assign(k), b = assign(k + 1);
        if (std::fabs(a) <= cri && std::fabs(b) <= cri && a * b < 0.0) {
            ks = k;
            ++ncross;
        }
    }
    if (ncross != 1 || ks < 2) {
        lica_set_last_error("lica_gpu_column_init", "need one interface above the first refined cell", __FILE__,
                            __LINE__);
        return LICA_BAD_ARG;
    }
    for (int q = 0; q < nf + 7; ++q) {
        st->phi[q] = 0.0;
        st->layer[q] = 0;
        st->mflvs[q] = 0.0;
    }
    for (int j = 0; j <= 10; ++j) {
        const int lo = ks - j, hi = ks + 1 + j;
        if (lo >= 2) st->layer[lo + 2] = 1 + j;
        if (hi <= nf) st->layer[hi + 2] = 1 + j;
    }
    for (int k = 1; k <= nf; ++k)
        if (st->layer[k + 2] > 0) st->phi[k + 2] = assign(k);
    auto P = [&](int k) { return st->phi[k + 2]; };
    std::vector<double> ps(nf + 2, 0.0);
    for (int k = 1; k <= nf; ++k) {
        if (st->layer[k + 2] == 0) continue;
        const double e1 = 0.5 * std::fabs(P(k + 1) - P(k - 1));
        double t;
        if (e1 > 1e-8) {
            const double f1 = std::max(0.5 * (e1 + 0.0 + 0.0) - std::fabs(P(k)), 0.0);
            t = f1 / e1;
        } else {
            t = (P(k) != 0.0) ? 0.0 : 0.5;
        }
        double v = (P(k) <= 0.0) ? t : 1.0 - t;
        if (v < 1e-5) v = 0.0;
        else if (v > 0.99999) v = 1.0;
        ps[k] = v;
    }
    const double t1 = (P(ks) < 0.0) ? 0.0 : 1.0, t2 = (P(ks + 1) < 0.0) ? 0.0 : 1.0;
    for (int k = 1; k <= nf; ++k)
        if (st->layer[k + 2] == 0) ps[k] = (k > ks) ? t2 : t1;
    const double dvol = 0.5 * 0.5 * hf;
    double vol = 0.0;
    for (int k = 1; k <= nf; ++k)
        for (int r = 0; r < 4; ++r) vol = vol + (1.0 - ps[k]) * dvol;
    for (int k = 0; k <= nf + 1; ++k) {
        st->psif[k] = (k >= 1 && k <= nf) ? ps[k] : 0.0;
        st->sfgas[k] = 0.0;
        st->sfgas2[k] = 0.0;
    }
    // GRID_COUPLING(1)
    for (int k = 2; k <= n; ++k)
        st->psi_zn[k] = h_box_mean(st->psif, nf, geo ? geo->kcoump2[k] : 2 * k - 2,
                                   geo ? geo->kcoump1[k + 1] : 2 * k - 1, zp(k - 1), zp(k), hf);
    for (int k = 1; k <= n; ++k) {
        if (st->psi_zn[k] < 1e-3) st->psi_zn[k] = 0.0;
        else if (st->psi_zn[k] > 0.999) st->psi_zn[k] = 1.0;
    }
    for (int k = 1; k <= n; ++k)
        st->psi_cn[k] = h_box_mean(st->psif, nf, geo ? geo->kcou2[k + 1] : 2 * k - 1, geo ? geo->kcou1[k + 2] : 2 * k,
                                   zc(k), zc(k + 1), hf);
    for (int k = 1; k <= n; ++k) {
        if (st->psi_cn[k] < 1e-3) st->psi_cn[k] = 0.0;
        else if (st->psi_cn[k] > 0.999) st->psi_cn[k] = 1.0;
    }
    st->psi_cn[0] = st->psi_cn[1];
    st->psi_cn[n + 1] = st->psi_cn[n];
    st->scal[0] = props->dt0;
    st->scal[1] = 0.0;
    st->scal[2] = 0.0;
    st->scal[3] = vol;
    st->scal[4] = vol;
    for (int q = 0; q < 8; ++q) st->stats[q] = 0.0;
    return LICA_OK;
}

// A stretched column's geometry is accepted when its faces rise, span [0, length], no cell
// is narrower than a refined cell (the level-set band's flow-face window assumes it), the
// velocity tables name flow cells and the box tables stay near the refined grid (the box
// sums clamp their reads to it).
static int geometry_ok(int32_t n, double length, const lica_col_geometry* geo) {
    if (!geo || !geo->z || !geo->zp || !geo->sdz || !geo->vdz || !geo->ssdz || !geo->vvdz || !geo->kcou1 ||
        !geo->kcou2 || !geo->kcoump1 || !geo->kcoump2 || !geo->kcou_vel || !geo->kcoump_vel)
        return 0;
    const double hf = length / (2.0 * n);
    if (std::fabs(geo->z[1]) > 1e-12 * length || std::fabs(geo->z[n + 1] - length) > 1e-12 * length) return 0;
    for (int k = 1; k <= n; ++k)
        if (!(geo->z[k + 1] - geo->z[k] >= hf * (1.0 - 1e-12))) return 0;
    for (int k = 1; k <= 2 * n; ++k)
        if (geo->kcou_vel[k] < 1 || geo->kcou_vel[k] > n || geo->kcoump_vel[k] < 1 || geo->kcoump_vel[k] > n + 1)
            return 0;
    for (int k = -1; k <= n + 2; ++k) {
        const int a = geo->kcou1[k + 1], b = geo->kcou2[k + 1];
        if (a < -8 || a > 2 * n + 8 || b < -8 || b > 2 * n + 8) return 0;
    }
    for (int k = -1; k <= n + 1; ++k) {
        const int a = geo->kcoump1[k + 1], b = geo->kcoump2[k + 1];
        if (a < -8 || a > 2 * n + 8 || b < -8 || b > 2 * n + 8) return 0;
    }
    return 1;
}

int lica_gpu_column_init(int32_t n, double length, double z0, const lica_col_props* props, lica_col_state* st) {
    return column_init(n, length, z0, props, nullptr, st);
}

int lica_gpu_column_init_geometry(int32_t n, double length, double z0, const lica_col_props* props,
                                  const lica_col_geometry* geo, lica_col_state* st) {
    if (n < 8 || !(length > 0.0) || !geometry_ok(n, length, geo)) {
        lica_set_last_error("lica_gpu_column_init_geometry", "bad column geometry", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    return column_init(n, length, z0, props, geo, st);
}

int lica_gpu_column_history_device(double* hist, int32_t capacity) {
    if (hist && capacity < 1) return LICA_BAD_ARG;
    g_col_hist = hist;
    g_col_hist_cap = hist ? capacity : 0;
    return LICA_OK;
}

int lica_gpu_column_profile_device(int64_t* prof) {
    g_col_prof = (long long*)prof;
    return LICA_OK;
}

size_t lica_gpu_column_scratch_bytes(int32_t ncol, int32_t n) {
    const size_t sf = (size_t)n + 2, sq = 2 * (size_t)n + 2;
    return (size_t)ncol * ((colk::NFLOW * sf + sq) * sizeof(double) + (sf + 2) * sizeof(int)) + 256;
}

}  // extern "C"

namespace {

void fill_state(colk::Args& A, const lica_col_state* st) {
    A.w = st->w;
    A.p = st->p;
    A.t = st->t;
    A.psi_cn = st->psi_cn;
    A.psi_zn = st->psi_zn;
    A.phi = st->phi;
    A.layer = st->layer;
    A.psif = st->psif;
    A.wo = st->wo;
    A.mflvs = st->mflvs;
    A.sfgas = st->sfgas;
    A.sfgas2 = st->sfgas2;
    A.imask = st->imask;
    A.scal = st->scal;
    A.stats = st->stats;
}

bool state_ok(const lica_col_state* st) {
    return st && st->w && st->p && st->t && st->psi_cn && st->psi_zn && st->phi && st->layer && st->psif && st->wo &&
           st->mflvs && st->sfgas && st->sfgas2 && st->imask && st->scal && st->stats;
}

// Launch A over A.ncol CTAs of `threads` threads; nmax = the largest column, which sizes
// the shared-memory tridiagonal arrays.
template <int NTH>
int column_ctas_by_registers() {
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, colk::k_column_steps<NTH>, NTH, 0);
    return std::max(occ, 1);
}

// The CTA width when the caller leaves it open: 256 threads while the batch has at most one
// column per SM (each column is a latency chain, and a wider CTA finishes its phases sooner),
// 64 beyond that (five columns per SM; on the 4096-column batch 64 threads take 25.6-25.8 ms
// a step, 128 threads 38.7).
int default_width(int ncol) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess || sms < 1)
            sms = 1;
    }
    return ncol <= sms ? 256 : 64;
}

int launch_columns(colk::Args& A, int nmax, int threads, void* stream, int cap_limit = -1) {
    const int nth = (threads == 32 || threads == 64 || threads == 128 || threads == 256) ? threads
                                                                                          : default_width(A.ncol);
    // Shared-memory tridiagonal arrays for columns up to tri_cap cells, sized so that the
    // CTAs the registers allow per SM still fit (longer columns keep them in scratch; the
    // arithmetic is the same either way).
    const int ctas = nth == 32    ? column_ctas_by_registers<32>()
                     : nth == 64  ? column_ctas_by_registers<64>()
                     : nth == 128 ? column_ctas_by_registers<128>()
                                  : column_ctas_by_registers<256>();
    const long budget = (long)(228 * 1024) / ctas - (long)sizeof(colk::Shared) - 2048;
    long cap = std::min<long>(nmax, budget / (5 * (long)sizeof(double)) - 2);
    if (cap_limit >= 0) cap = std::min<long>(cap, cap_limit);   // a caller's (autotuner's) limit
    A.tri_cap = cap >= 64 ? (int)cap : 0;
    A.tri_smem = A.tri_cap > 0 ? 1 : 0;
    const size_t dyn = A.tri_smem ? 5 * ((size_t)A.tri_cap + 2) * sizeof(double) : 0;
    {
        // the attribute is the current device's: kept per device
        static std::mutex mu;
        static size_t set_bytes[kMaxDevices][4] = {};
        std::lock_guard<std::mutex> lk(mu);
        const int dev = current_device();
        if (dev >= kMaxDevices) {
            lica_set_last_error("launch_columns", "device ordinal above 63", __FILE__, __LINE__);
            return LICA_BAD_ARG;
        }
        const int slot = nth == 64 ? 0 : (nth == 128 ? 1 : (nth == 256 ? 2 : 3));
        if (dyn > set_bytes[dev][slot]) {
            cudaError_t e = cudaSuccess;
            if (nth == 32)
                e = cudaFuncSetAttribute(colk::k_column_steps<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            else if (nth == 64)
                e = cudaFuncSetAttribute(colk::k_column_steps<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            else if (nth == 128)
                e = cudaFuncSetAttribute(colk::k_column_steps<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)dyn);
            else
                e = cudaFuncSetAttribute(colk::k_column_steps<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)dyn);
            LICA_CUDA_TRY(e);
            set_bytes[dev][slot] = dyn;
        }
    }
    if (nth == 32) colk::k_column_steps<32><<<A.ncol, 32, dyn, (cudaStream_t)stream>>>(A);
    else if (nth == 64) colk::k_column_steps<64><<<A.ncol, 64, dyn, (cudaStream_t)stream>>>(A);
    else if (nth == 128) colk::k_column_steps<128><<<A.ncol, 128, dyn, (cudaStream_t)stream>>>(A);
    else colk::k_column_steps<256><<<A.ncol, 256, dyn, (cudaStream_t)stream>>>(A);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int column_scratch(size_t need, void** out) {
    const int dev = current_device();
    if (dev >= kMaxDevices) {
        lica_set_last_error("column scratch", "device ordinal above 63", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    ScratchCache& sc = scratch_cache(dev);
    std::lock_guard<std::mutex> lk(sc.mu);
    if (need > sc.bytes) {
        if (sc.ptr) cudaFree(sc.ptr);
        sc.ptr = nullptr;
        sc.bytes = 0;
        LICA_CUDA_TRY(cudaMalloc(&sc.ptr, need));
        sc.bytes = need;
    }
    *out = sc.ptr;
    return LICA_OK;
}

}  // namespace

// A batch of columns of uneven size and properties.
struct lica_col_batch {
    int ncol = 0, nmax = 0;
    std::vector<colk::ColDesc> desc;
    std::vector<int> order;
    colk::ColDesc* d_desc = nullptr;
    int* d_order = nullptr;
    int64_t tot[5] = {0, 0, 0, 0, 0};   // flow, phi-like, psif-like doubles; scratch doubles, scratch ints
    std::mutex mu;
};

extern "C" {

}  // extern "C"

namespace {

int column_steps_device(int32_t ncol, int32_t n, double length, const lica_col_props* props, const lica_col_state* st,
                        int32_t nsteps, int32_t threads, void* scratch, int32_t* status, void* stream,
                        const lica_col_geo* geo) {
    if (ncol < 1 || n < 8 || n > (1 << 20) || !(length > 0.0) || !props || !state_ok(st) || nsteps < 0 || !status) {
        lica_set_last_error("lica_gpu_column_steps_device", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    colk::Args A{};
    A.has_geo = geo ? 1 : 0;
    if (geo) A.geo = geo->dev;
    A.ncol = ncol;
    A.n = n;
    A.nsteps = nsteps;
    A.L = length;
    A.ph = make_phys(props);
    A.desc = nullptr;
    A.order = nullptr;
    fill_state(A, st);
    A.status = status;
    A.prof = g_col_prof;
    A.hist = g_col_hist;
    A.hist_cap = g_col_hist_cap;
    void* scr = scratch;
    if (!scr) {
        const int rc = column_scratch(lica_gpu_column_scratch_bytes(ncol, n), &scr);
        if (rc) return rc;
    }
    const size_t sf = (size_t)n + 2, sq = 2 * (size_t)n + 2;
    A.dscr = (double*)scr;
    A.iscr = (int*)((char*)scr + (size_t)ncol * (colk::NFLOW * sf + sq) * sizeof(double));
    return launch_columns(A, n, threads, stream);
}

}  // namespace

extern "C" {

int lica_gpu_column_steps_device(int32_t ncol, int32_t n, double length, const lica_col_props* props,
                                 const lica_col_state* st, int32_t nsteps, int32_t threads, void* scratch,
                                 int32_t* status, void* stream) {
    return column_steps_device(ncol, n, length, props, st, nsteps, threads, scratch, status, stream, nullptr);
}

int lica_gpu_column_geometry_create(lica_col_geo** out, int32_t n, double length, const lica_col_geometry* host) {
    if (!out) return LICA_BAD_ARG;
    *out = nullptr;
    if (n < 8 || n > (1 << 20) || !(length > 0.0) || !geometry_ok(n, length, host)) {
        lica_set_last_error("lica_gpu_column_geometry_create", "bad column geometry", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    // one device buffer: six double arrays of n+2, then the int tables (n+5, n+5, n+4, n+4,
    // 2n+2, 2n+2), each 256-byte aligned
    const size_t nd = (size_t)n + 2;
    const size_t ni[6] = {(size_t)n + 5, (size_t)n + 5, (size_t)n + 4, (size_t)n + 4, 2 * (size_t)n + 2,
                          2 * (size_t)n + 2};
    const double* hd[6] = {host->z, host->zp, host->sdz, host->vdz, host->ssdz, host->vvdz};
    const int32_t* hi[6] = {host->kcou1, host->kcou2, host->kcoump1, host->kcoump2, host->kcou_vel, host->kcoump_vel};
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t total = 6 * up(nd * sizeof(double));
    for (int q = 0; q < 6; ++q) total += up(ni[q] * sizeof(int32_t));
    auto* g = new lica_col_geo();
    g->n = n;
    g->length = length;
    if (cudaMalloc(&g->buf, total) != cudaSuccess) {
        delete g;
        lica_set_last_error("lica_gpu_column_geometry_create", "cudaMalloc failed", __FILE__, __LINE__);
        return LICA_ERR_CUDA;
    }
    char* p = (char*)g->buf;
    const double* dd[6];
    const int* di[6];
    for (int q = 0; q < 6; ++q) {
        dd[q] = (const double*)p;
        if (cudaMemcpy(p, hd[q], nd * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
            lica_gpu_column_geometry_destroy(g);
            return LICA_ERR_CUDA;
        }
        p += up(nd * sizeof(double));
    }
    for (int q = 0; q < 6; ++q) {
        di[q] = (const int*)p;
        if (cudaMemcpy(p, hi[q], ni[q] * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
            lica_gpu_column_geometry_destroy(g);
            return LICA_ERR_CUDA;
        }
        p += up(ni[q] * sizeof(int32_t));
    }
    g->dev = col::ColGeoDev{dd[0], dd[1], dd[2], dd[3], dd[4], dd[5], di[0], di[1], di[2], di[3], di[4], di[5]};
    *out = g;
    return LICA_OK;
}

int lica_gpu_column_geometry_destroy(lica_col_geo* g) {
    if (!g) return LICA_OK;
    if (g->buf) cudaFree(g->buf);
    delete g;
    return LICA_OK;
}

int lica_gpu_column_steps_geometry_device(const lica_col_geo* geo, int32_t ncol, const lica_col_props* props,
                                          const lica_col_state* st, int32_t nsteps, int32_t threads, void* scratch,
                                          int32_t* status, void* stream) {
    if (!geo) return LICA_BAD_ARG;
    return column_steps_device(ncol, geo->n, geo->length, props, st, nsteps, threads, scratch, status, stream, geo);
}

int lica_gpu_column_batch_create(lica_col_batch** out, int32_t ncol, const int32_t* n, const double* length,
                                 const lica_col_props* props) {
    if (!out || ncol < 1 || !n || !length || !props) return LICA_BAD_ARG;
    auto* b = new lica_col_batch();
    b->ncol = ncol;
    b->desc.resize(ncol);
    int64_t of = 0, op = 0, oq = 0, od = 0, oi = 0;
    for (int c = 0; c < ncol; ++c) {
        if (n[c] < 8 || n[c] > (1 << 20) || !(length[c] > 0.0)) {
            delete b;
            lica_set_last_error("lica_gpu_column_batch_create", "column size < 8 or length <= 0", __FILE__, __LINE__);
            return LICA_BAD_ARG;
        }
        colk::ColDesc& D = b->desc[c];
        D.n = n[c];
        D.pad = 0;
        D.L = length[c];
        D.ph = make_phys(&props[c]);
        const int64_t sf = n[c] + 2, sq = 2 * (int64_t)n[c] + 2;
        D.off_f = of;
        D.off_p = op;
        D.off_q = oq;
        D.off_d = od;
        D.off_i = oi;
        of += sf;
        op += 2 * (int64_t)n[c] + 7;
        oq += sq;
        od += colk::NFLOW * sf + sq;
        oi += sf + 2;
        b->nmax = std::max(b->nmax, (int)n[c]);
    }
    b->tot[0] = of;
    b->tot[1] = op;
    b->tot[2] = oq;
    b->tot[3] = od;
    b->tot[4] = oi;
    // longest columns first, so the last CTAs to start are the short ones
    b->order.resize(ncol);
    for (int c = 0; c < ncol; ++c) b->order[c] = c;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return n[x] > n[y]; });
    *out = b;
    return LICA_OK;
}

int lica_gpu_column_batch_destroy(lica_col_batch* b) {
    if (!b) return LICA_OK;
    if (b->d_desc) cudaFree(b->d_desc);
    if (b->d_order) cudaFree(b->d_order);
    delete b;
    return LICA_OK;
}

int lica_gpu_column_batch_layout(const lica_col_batch* b, int64_t* offsets, int64_t* totals) {
    if (!b) return LICA_BAD_ARG;
    if (offsets)
        for (int c = 0; c < b->ncol; ++c) {
            offsets[3 * c + 0] = b->desc[c].off_f;
            offsets[3 * c + 1] = b->desc[c].off_p;
            offsets[3 * c + 2] = b->desc[c].off_q;
        }
    if (totals) {
        totals[0] = b->tot[0];
        totals[1] = b->tot[1];
        totals[2] = b->tot[2];
        totals[3] = (int64_t)(b->tot[3] * sizeof(double) + b->tot[4] * sizeof(int) + 256);
    }
    return LICA_OK;
}

int lica_gpu_column_batch_steps_device(const lica_col_batch* b, const lica_col_state* st, int32_t nsteps,
                                       int32_t threads, void* scratch, int32_t* status, void* stream) {
    return lica_gpu_column_batch_steps_ex_device(b, st, nsteps, threads, -1, scratch, status, stream);
}

int lica_gpu_column_batch_steps_ex_device(const lica_col_batch* b, const lica_col_state* st, int32_t nsteps,
                                          int32_t threads, int32_t tri_cap, void* scratch, int32_t* status,
                                          void* stream) {
    if (!b || !state_ok(st) || nsteps < 0 || !status) return LICA_BAD_ARG;
    {
        // descriptors and launch order go to the device on first use (the host-side layout
        // and initial state need no GPU)
        lica_col_batch* m = const_cast<lica_col_batch*>(b);
        std::lock_guard<std::mutex> lk(m->mu);
        if (!m->d_desc) {
            LICA_CUDA_TRY(cudaMalloc(&m->d_desc, sizeof(colk::ColDesc) * m->ncol));
            LICA_CUDA_TRY(cudaMalloc(&m->d_order, sizeof(int) * m->ncol));
            LICA_CUDA_TRY(
                cudaMemcpy(m->d_desc, m->desc.data(), sizeof(colk::ColDesc) * m->ncol, cudaMemcpyHostToDevice));
            LICA_CUDA_TRY(cudaMemcpy(m->d_order, m->order.data(), sizeof(int) * m->ncol, cudaMemcpyHostToDevice));
        }
    }
    colk::Args A{};
    A.ncol = b->ncol;
    A.n = b->nmax;
    A.nsteps = nsteps;
    A.L = 1.0;
    A.desc = b->d_desc;
    A.order = b->d_order;
    fill_state(A, st);
    A.status = status;
    A.prof = g_col_prof;
    A.hist = g_col_hist;
    A.hist_cap = g_col_hist_cap;
    void* scr = scratch;
    if (!scr) {
        const int rc = column_scratch((size_t)(b->tot[3] * sizeof(double) + b->tot[4] * sizeof(int) + 256), &scr);
        if (rc) return rc;
    }
    A.dscr = (double*)scr;
    A.iscr = (int*)((char*)scr + (size_t)b->tot[3] * sizeof(double));
    return launch_columns(A, b->nmax, threads, stream, tri_cap);
}

}  // extern "C"

namespace {

int column_steps_host(int32_t ncol, int32_t n, double length, const lica_col_props* props, lica_col_state* st,
                      int32_t nsteps, int32_t* status, const lica_col_geo* geo) {
    if (ncol < 1 || n < 8 || !props || !st || !status) return LICA_BAD_ARG;
    const size_t nc = (size_t)ncol, sf = (size_t)n + 2, sp = 2 * (size_t)n + 7, sq = 2 * (size_t)n + 2;
    struct F {
        void* h;
        size_t bytes;
    };
    const F f[] = {{st->w, 8 * nc * sf},      {st->p, 8 * nc * sf},      {st->t, 8 * nc * sf},
                   {st->psi_cn, 8 * nc * sf}, {st->psi_zn, 8 * nc * sf}, {st->phi, 8 * nc * sp},
                   {st->layer, 4 * nc * sp},  {st->psif, 8 * nc * sq},   {st->wo, 8 * nc * sf},
                   {st->mflvs, 8 * nc * sp},  {st->sfgas, 8 * nc * sq},  {st->sfgas2, 8 * nc * sq},
                   {st->imask, 4 * nc * sf},  {st->scal, 8 * nc * 5},    {st->stats, 8 * nc * 8}};
    const int nfld = (int)(sizeof(f) / sizeof(f[0]));
    for (int q = 0; q < nfld; ++q)
        if (!f[q].h) return LICA_BAD_ARG;
    size_t off[16], total = 0;
    for (int q = 0; q < nfld; ++q) {
        off[q] = total;
        total += (f[q].bytes + 255) & ~(size_t)255;
    }
    const size_t st_off = total;
    total += (4 * nc + 255) & ~(size_t)255;
    // device copies in a grow-only buffer kept by the library per device (one host call at a
    // time)
    const int dev = current_device();
    if (dev >= kMaxDevices) {
        lica_set_last_error("lica_gpu_column_steps", "device ordinal above 63", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    static std::mutex host_mu;
    static char* host_buf[kMaxDevices] = {};
    static size_t host_bytes[kMaxDevices] = {};
    static cudaStream_t host_stream[kMaxDevices] = {};
    std::lock_guard<std::mutex> lk(host_mu);
    if (total > host_bytes[dev]) {
        if (host_buf[dev]) cudaFree(host_buf[dev]);
        host_buf[dev] = nullptr;
        host_bytes[dev] = 0;
        LICA_CUDA_TRY(cudaMalloc(&host_buf[dev], total));
        host_bytes[dev] = total;
    }
    char* base = host_buf[dev];
    // copies and steps go on one stream of the library's, so the call waits once; a blocking
    // stream, so it stays ordered after work a caller left on the legacy default stream that
    // may use the same library scratch
    if (!host_stream[dev]) LICA_CUDA_TRY(cudaStreamCreateWithFlags(&host_stream[dev], cudaStreamDefault));
    cudaStream_t hs = host_stream[dev];
    // Small states (a few columns: the per-step drop-in use) go through one page-locked
    // staging buffer (portable: pinned for every device), one copy each way instead of one
    // per array; large ones copy directly.
    static char* pin_buf = nullptr;
    static size_t pin_bytes = 0;
    const bool packed = total <= ((size_t)64 << 20);
    if (packed && total > pin_bytes) {
        if (pin_buf) cudaFreeHost(pin_buf);
        pin_buf = nullptr;
        pin_bytes = 0;
        LICA_CUDA_TRY(cudaHostAlloc((void**)&pin_buf, total, cudaHostAllocPortable));
        pin_bytes = total;
    }
    if (packed) {
        for (int q = 0; q < nfld; ++q) std::memcpy(pin_buf + off[q], f[q].h, f[q].bytes);
        LICA_CUDA_TRY(cudaMemcpyAsync(base, pin_buf, st_off, cudaMemcpyHostToDevice, hs));
    } else {
        for (int q = 0; q < nfld; ++q)
            LICA_CUDA_TRY(cudaMemcpyAsync(base + off[q], f[q].h, f[q].bytes, cudaMemcpyHostToDevice, hs));
    }
    lica_col_state d;
    d.w = (double*)(base + off[0]);
    d.p = (double*)(base + off[1]);
    d.t = (double*)(base + off[2]);
    d.psi_cn = (double*)(base + off[3]);
    d.psi_zn = (double*)(base + off[4]);
    d.phi = (double*)(base + off[5]);
    d.layer = (int32_t*)(base + off[6]);
    d.psif = (double*)(base + off[7]);
    d.wo = (double*)(base + off[8]);
    d.mflvs = (double*)(base + off[9]);
    d.sfgas = (double*)(base + off[10]);
    d.sfgas2 = (double*)(base + off[11]);
    d.imask = (int32_t*)(base + off[12]);
    d.scal = (double*)(base + off[13]);
    d.stats = (double*)(base + off[14]);
    int32_t* dst = (int32_t*)(base + st_off);
    int rc = column_steps_device(ncol, n, length, props, &d, nsteps, 0, nullptr, dst, hs, geo);
    if (rc) {
        cudaStreamSynchronize(hs);
        return rc;
    }
    if (packed) {
        LICA_CUDA_TRY(cudaMemcpyAsync(pin_buf, base, total, cudaMemcpyDeviceToHost, hs));
        LICA_CUDA_TRY(cudaStreamSynchronize(hs));
        for (int q = 0; q < nfld; ++q) std::memcpy(f[q].h, pin_buf + off[q], f[q].bytes);
        std::memcpy(status, pin_buf + st_off, 4 * nc);
    } else {
        for (int q = 0; q < nfld; ++q)
            LICA_CUDA_TRY(cudaMemcpyAsync(f[q].h, base + off[q], f[q].bytes, cudaMemcpyDeviceToHost, hs));
        LICA_CUDA_TRY(cudaMemcpyAsync(status, dst, 4 * nc, cudaMemcpyDeviceToHost, hs));
        LICA_CUDA_TRY(cudaStreamSynchronize(hs));
    }
    int worst = LICA_OK;
    for (size_t c = 0; c < nc; ++c)
        if (status[c] != LICA_OK) worst = status[c];
    return worst;
}

}  // namespace

extern "C" {

int lica_gpu_column_steps(int32_t ncol, int32_t n, double length, const lica_col_props* props, lica_col_state* st,
                          int32_t nsteps, int32_t* status) {
    return column_steps_host(ncol, n, length, props, st, nsteps, status, nullptr);
}

int lica_gpu_column_steps_geometry(const lica_col_geo* geo, int32_t ncol, const lica_col_props* props,
                                   lica_col_state* st, int32_t nsteps, int32_t* status) {
    if (!geo) return LICA_BAD_ARG;
    return column_steps_host(ncol, geo->n, geo->length, props, st, nsteps, status, geo);
}

// ---- single routines (drop-ins for the reference's subroutines, batches of columns)
}  // extern "C"

namespace {

int routine_launch(colk::RoutineArgs& A, void* scratch, void* stream) {
    void* scr = scratch;
    if (!scr) {
        const int rc = column_scratch(lica_gpu_column_scratch_bytes(A.ncol, A.n), &scr);
        if (rc) return rc;
    }
    A.dscr = (double*)scr;
    colk::k_col_routine<<<A.ncol, colk::NT_DEFAULT, 0, (cudaStream_t)stream>>>(A);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

// Device copies of host arrays for the host-array drop-ins; freed on scope exit.
struct HostCopies {
    std::vector<void*> ptrs;
    ~HostCopies() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int in(T** d, const T* h, size_t n) {
        void* p = nullptr;
        LICA_CUDA_TRY(cudaMalloc(&p, sizeof(T) * n));
        ptrs.push_back(p);
        if (h) LICA_CUDA_TRY(cudaMemcpy(p, h, sizeof(T) * n, cudaMemcpyHostToDevice));
        *d = (T*)p;
        return LICA_OK;
    }
};

template <typename T>
int copy_out(T* h, const T* d, size_t n) {
    LICA_CUDA_TRY(cudaMemcpy(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

int worst_status(const int32_t* status, int32_t ncol) {
    int worst = LICA_OK;
    for (int c = 0; c < ncol; ++c)
        if (status[c] != LICA_OK) worst = status[c];
    return worst;
}

}  // namespace

extern "C" {

int lica_gpu_temp_grad_device(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                              const double* t, const double* psi_cn, const double* phi, const int32_t* layer,
                              double* mflvs, double* sfgas, double* sfgas2, int32_t* imask, double* vol_tot_iphs,
                              int32_t* iterations, int32_t* status, void* scratch, void* stream) {
    if (ncol < 1 || n < 8 || n > (1 << 20) || !(length > 0.0) || !props || !(dtconst > 0.0) || !t || !psi_cn ||
        !phi || !layer || !mflvs || !sfgas || !sfgas2 || !imask || !vol_tot_iphs || !iterations || !status) {
        lica_set_last_error("lica_gpu_temp_grad_device", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    colk::RoutineArgs A{};
    A.ncol = ncol;
    A.n = n;
    A.routine = colk::RT_TEMP_GRAD;
    A.L = length;
    A.dtconst = dtconst;
    A.ph = make_phys(props);
    A.t = const_cast<double*>(t);
    A.psi_cn = const_cast<double*>(psi_cn);
    A.phi = const_cast<double*>(phi);
    A.layer = const_cast<int32_t*>(layer);
    A.mflvs = mflvs;
    A.sfgas = sfgas;
    A.sfgas2 = sfgas2;
    A.imask = imask;
    A.vol = vol_tot_iphs;
    A.iters = iterations;
    A.status = status;
    return routine_launch(A, scratch, stream);
}

int lica_gpu_temp_grad(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                       const double* t, const double* psi_cn, const double* phi, const int32_t* layer, double* mflvs,
                       double* sfgas, double* sfgas2, int32_t* imask, double* vol_tot_iphs, int32_t* iterations,
                       int32_t* status) {
    if (ncol < 1 || n < 8 || n > (1 << 20) || !t || !psi_cn || !phi || !layer || !mflvs || !sfgas || !sfgas2 ||
        !imask || !vol_tot_iphs || !iterations || !status) {
        lica_set_last_error("lica_gpu_temp_grad", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const size_t nc = (size_t)ncol, sf = (size_t)n + 2, sp = 2 * (size_t)n + 7, sq = 2 * (size_t)n + 2;
    HostCopies H;
    double *dt_, *dcn, *dphi, *dmf, *dsf, *dsf2, *dvol;
    int32_t *dlay, *dim, *dit, *dst;
    int rc;
    if ((rc = H.in(&dt_, t, nc * sf)) || (rc = H.in(&dcn, psi_cn, nc * sf)) || (rc = H.in(&dphi, phi, nc * sp)) ||
        (rc = H.in(&dlay, layer, nc * sp)) || (rc = H.in(&dmf, (const double*)nullptr, nc * sp)) ||
        (rc = H.in(&dsf, (const double*)nullptr, nc * sq)) || (rc = H.in(&dsf2, (const double*)nullptr, nc * sq)) ||
        (rc = H.in(&dim, (const int32_t*)nullptr, nc * sf)) || (rc = H.in(&dvol, vol_tot_iphs, nc)) ||
        (rc = H.in(&dit, (const int32_t*)nullptr, nc)) || (rc = H.in(&dst, (const int32_t*)nullptr, nc)))
        return rc;
    if ((rc = lica_gpu_temp_grad_device(ncol, n, length, props, dtconst, dt_, dcn, dphi, dlay, dmf, dsf, dsf2, dim,
                                        dvol, dit, dst, nullptr, nullptr)))
        return rc;
    LICA_CUDA_TRY(cudaDeviceSynchronize());
    if ((rc = copy_out(mflvs, dmf, nc * sp)) || (rc = copy_out(sfgas, dsf, nc * sq)) ||
        (rc = copy_out(sfgas2, dsf2, nc * sq)) || (rc = copy_out(imask, dim, nc * sf)) ||
        (rc = copy_out(vol_tot_iphs, dvol, nc)) || (rc = copy_out(iterations, dit, nc)) ||
        (rc = copy_out(status, dst, nc)))
        return rc;
    return worst_status(status, ncol);
}

int lica_gpu_pressure_correction_device(int32_t ncol, int32_t n, double length, const lica_col_props* props,
                                        double dtconst, double* w, double* p, const double* denf_zi,
                                        const double* sfgas, int32_t* status, void* scratch, void* stream) {
    if (ncol < 1 || n < 8 || n > (1 << 20) || !(length > 0.0) || !props || !(dtconst > 0.0) || !w || !p ||
        !denf_zi || !sfgas || !status) {
        lica_set_last_error("lica_gpu_pressure_correction_device", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    colk::RoutineArgs A{};
    A.ncol = ncol;
    A.n = n;
    A.routine = colk::RT_PRESSURE_CORRECTION;
    A.L = length;
    A.dtconst = dtconst;
    A.ph = make_phys(props);
    A.w = w;
    A.p = p;
    A.denf_zi = denf_zi;
    A.sfgas = const_cast<double*>(sfgas);
    A.status = status;
    return routine_launch(A, scratch, stream);
}

int lica_gpu_pressure_correction(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                                 double* w, double* p, const double* denf_zi, const double* sfgas) {
    if (ncol < 1 || n < 8 || n > (1 << 20) || !w || !p || !denf_zi || !sfgas) {
        lica_set_last_error("lica_gpu_pressure_correction", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const size_t nc = (size_t)ncol, sf = (size_t)n + 2, sq = 2 * (size_t)n + 2;
    HostCopies H;
    double *dw, *dp, *dden, *dsf;
    int32_t* dst;
    int rc;
    if ((rc = H.in(&dw, (const double*)w, nc * sf)) || (rc = H.in(&dp, (const double*)p, nc * sf)) ||
        (rc = H.in(&dden, denf_zi, nc * sf)) || (rc = H.in(&dsf, sfgas, nc * sq)) ||
        (rc = H.in(&dst, (const int32_t*)nullptr, nc)))
        return rc;
    if ((rc = lica_gpu_pressure_correction_device(ncol, n, length, props, dtconst, dw, dp, dden, dsf, dst, nullptr,
                                                  nullptr)))
        return rc;
    LICA_CUDA_TRY(cudaDeviceSynchronize());
    if ((rc = copy_out(w, (const double*)dw, nc * sf)) || (rc = copy_out(p, (const double*)dp, nc * sf))) return rc;
    std::vector<int32_t> st(nc);
    if ((rc = copy_out(st.data(), (const int32_t*)dst, nc))) return rc;
    return worst_status(st.data(), ncol);
}

}  // extern "C"
