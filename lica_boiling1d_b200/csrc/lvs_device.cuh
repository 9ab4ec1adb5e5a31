// Device routines of the 1-D level-set transport (TRANSPORT, two_phase.f:701-984, and the
// routines it calls), shared by the batched level-set kernel (lvs.cu) and the fused
// column-step kernel (column.cu).  See lvs.cu for the parallel layout.
#pragma once
#include "common.cuh"
#include "column_geom.cuh"

#include <cmath>

namespace lica {
namespace lvs {

constexpr int N_MAX = 11;           // M_MAX
constexpr int NN1 = N_MAX - 3;      // two_phase.f:737
constexpr int NN2 = N_MAX - 1;      // two_phase.f:738
constexpr int WIN = 128;            // window cells per column
constexpr int PER = WIN / 32;       // window cells per lane
constexpr int WARPS = 4;            // columns per CTA
constexpr int HALO = 8;             // room kept between the band and the window edge on entry
constexpr int EDGE = 4;             // room the band must keep after a regeneration
constexpr int WTN = 132;            // flow-face window of the time-averaged velocity: the faces
                                    // of 128 refined cells and the stencil margin on any flow
                                    // grid whose cells are at least one refined cell wide

struct Win {
    double phi[WIN];
    double rk3[WIN];
    double alphio[WIN];
    double dp[WIN];
    double nv[WIN];
    double wf[WIN];
    double start[WIN];   // phi at TRANSPORT entry: the phase test of the source, :1470
    double mf[WIN];
    double wt[WTN];
    double ghost[7];     // phi(-2..0), phi(nf+1..nf+4) as last set by ALPHI_BC
    int layer[WIN];
    int mask[WIN];
    int lst[WIN];        // band lists, layer after layer
    int lst2[WIN];
    int lstart[N_MAX + 2];
    int lstart2[N_MAX + 2];
    int fmask[WTN];      // GRID_COUPLING mask of the flow cells kw0..kw0+WTN-1
};

struct Ctx {
    const col::ColGeoDev* cg = nullptr;   // the flow grid's geometry (null: uniform)
    int n, nf, w0, kw0, lane;
    int blo = 0, bhi = -1;   // window slots spanned by the band (per-cell loops run over them)
    int vlo = 0, vhi = -1;   // slots the last VEL_INTP wrote
    double h, hf, ssdzf;
    Win* s;
    __device__ __forceinline__ bool in(int k) const { return k >= w0 && k < w0 + WIN; }
    __device__ __forceinline__ double p(int k) const { return in(k) ? s->phi[k - w0] : 0.0; }
};

// The first flow face of the window's flow range (WT, the GRID_COUPLING mask, TEMP_GRAD's
// flow arrays): band cell k reads faces KCOU_VEL(k)-1..+2.  Uniform column: KCOU_VEL = k/2
// clamped to 1..n, so faces floor(w0/2)-1 .. floor((w0+127)/2)+2 suffice; stretched: from
// KCOU_VEL of the window's first refined cell.
__device__ __forceinline__ int flow_origin(const Ctx& c, int w0) {
    if (!c.cg) return ((w0 >= 0) ? w0 / 2 : -((1 - w0) / 2)) - 2;
    const int k = w0 < 1 ? 1 : (w0 > c.nf ? c.nf : w0);
    return c.cg->kcou_vel[k] - 2;
}

// KCOUMP_VEL(k) of refined cell k: the table, or the uniform column's search
__device__ __forceinline__ int ctx_kcoump_vel(const Ctx& c, int k) {
    return c.cg ? c.cg->kcoump_vel[k] : col::kcoump_vel(c.h, c.hf, c.n, k);
}

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ALPHI_BC, two_phase.f:462-642, z part with IPZ != 1: the wall extrapolation of the
// ghosts (:556-593) followed by the periodic copy (:624-634).  Ghost values are kept in
// s->ghost as well, since the window may not cover both ends of the column.
__device__ inline void alphi_bc(Ctx& c) {
    if (c.lane == 0) {
        Win* s = c.s;
        const int nf = c.nf;
        const double dz = c.hf;
        double* g = s->ghost;   // [0..2] = k -2..0, [3..6] = k nf+1..nf+4
        const double a1 = c.p(1);
        if (fabs(a1) < 1e-8) {
            g[2] = 0.0; g[1] = 0.0; g[0] = 0.0;
        } else if (a1 > 0.0) {
            g[2] = a1 + dz; g[1] = g[2] + dz; g[0] = g[1] + dz;
        } else if (a1 < 0.0) {
            g[2] = a1 - dz; g[1] = g[2] - dz; g[0] = g[1] - dz;
        }
        const double an = c.p(nf);
        if (fabs(an) < 1e-8) {
            g[3] = 0.0; g[4] = 0.0; g[5] = 0.0; g[6] = 0.0;
        } else if (an > 0.0) {
            g[3] = an + dz; g[4] = g[3] + dz; g[5] = g[4] + dz; g[6] = g[5] + dz;
        } else if (an < 0.0) {
            g[3] = an - dz; g[4] = g[3] - dz; g[5] = g[4] - dz; g[6] = g[5] - dz;
        }
        // phi(-k) = phi(nf-k), phi(nf+1+k) = phi(1+k), k = 0..2 (interior sources, nf >= 16)
        for (int k = 0; k <= 2; ++k) {
            g[2 - k] = c.p(nf - k);
            g[3 + k] = c.p(1 + k);
        }
        for (int q = 0; q < 7; ++q) {
            const int k = q < 3 ? q - 2 : nf + q - 2;
            if (c.in(k)) s->phi[k - c.w0] = g[q];
        }
    }
    __syncwarp();
}

// slot range of the band cells; warp-wide
__device__ inline void band_range(Ctx& c) {
    const Win* s = c.s;
    int lo = WIN, hi = -1;
    for (int q = 0; q < PER; ++q) {
        const int i = c.lane + 32 * q, m = s->layer[i];
        if (m >= 1 && m <= N_MAX) {
            lo = min(lo, i);
            hi = max(hi, i);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    c.blo = (hi < 0) ? 0 : lo;
    c.bhi = hi;
}

// per-layer lists in ascending window order from s->layer (the CPU restatement loads a
// column the same way)
__device__ inline void build_lists(Ctx& c) {
    Win* s = c.s;
    int pos = 0;
    const unsigned below = (1u << c.lane) - 1u;
    for (int m = 1; m <= N_MAX; ++m) {
        if (c.lane == 0) s->lstart[m] = pos;
        for (int q = 0; q < PER; ++q) {
            const int i = c.lane + 32 * q;
            const bool pr = (s->layer[i] == m);
            const unsigned b = __ballot_sync(0xffffffffu, pr);
            if (pr) s->lst[pos + __popc(b & below)] = i;
            pos += __popc(b);
        }
    }
    if (c.lane == 0) s->lstart[N_MAX + 1] = pos;
    __syncwarp();
    band_range(c);
}

// layer numbers from the lists
__device__ inline void lists_to_layer(Ctx& c) {
    Win* s = c.s;
    for (int q = 0; q < PER; ++q) s->layer[c.lane + 32 * q] = 0;
    __syncwarp();
    for (int m = 1; m <= N_MAX; ++m)
        for (int j = s->lstart[m] + c.lane; j < s->lstart[m + 1]; j += 32) s->layer[s->lst[j]] = m;
    __syncwarp();
    band_range(c);
}

// Window over the band of a column for work outside TRANSPORT (TEMP_GRAD): the same origin
// rule as TRANSPORT, phi = band values and 0 elsewhere (ghosts included: TEMP_GRAD builds
// ALPHI_EXT from the band alone, chphase.f:121-139), ascending band lists.  Returns
// LICA_OK, LICA_BAD_ARG (band cell outside k = 1..nf) or LICA_BAND_OVERFLOW.
// band_only = false: every window cell takes the caller's phi (the drop-in REINITIALIZATION,
// whose stencils read ALPHI_EXT as the caller holds it).
__device__ inline int load_band_window(Ctx& c, int lane, int n, double length, const double* phi, const int* layer,
                                       bool band_only = true) {
    Win* s = c.s;
    c.n = n;
    c.nf = 2 * n;
    c.h = length / n;
    c.hf = length / c.nf;
    c.ssdzf = 1.0 / c.hf;
    c.lane = lane;
    const int nf = c.nf;
    int kmin = 1 << 30, kmax = -(1 << 30);
    for (int k = -2 + lane; k <= nf + 4; k += 32)
        if (layer[k + 2] > 0) {
            kmin = min(kmin, k);
            kmax = max(kmax, k);
        }
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (kmax >= kmin && (kmin < 1 || kmax > nf)) return LICA_BAD_ARG;
    if (kmax >= kmin && kmax - kmin + 1 > WIN - 2 * HALO) return LICA_BAND_OVERFLOW;
    int w0 = (kmax >= kmin) ? (kmin + kmax + 1) / 2 - WIN / 2 : -2;
    w0 = max(w0, -2);
    w0 = min(w0, max(-2, nf + 4 - (WIN - 1)));
    c.w0 = w0;
    c.kw0 = flow_origin(c, w0);
    for (int q = 0; q < PER; ++q) {
        const int i = lane + 32 * q, k = w0 + i;
        const bool ok = (k >= -2 && k <= nf + 4);
        const int m = ok ? layer[k + 2] : 0;
        s->layer[i] = m;
        s->phi[i] = (ok && (m > 0 || !band_only)) ? phi[k + 2] : 0.0;
    }
    __syncwarp();
    build_lists(c);
    return LICA_OK;
}

// BAND_GENERATION, two_phase.f:1622-2030 (1-D).  Sequential on lane 0, in the reference's
// list order: the S-tube from the old layers 1..NN2 (:1655-1680), then layer m from the
// neighbours of layer m-1, never k = 1 or k = nf+1 (:1704-1735), with phi at a new cell
// (or at any cell from layer NN2 on) set to the parent's phi -/+ the cell distance
// (:1931-1954).  Returns nonzero if the new band left the window.
__device__ inline int band_generation(Ctx& c) {
    Win* s = c.s;
    for (int q = 0; q < PER; ++q) s->mask[c.lane + 32 * q] = 0;
    __syncwarp();
    int ovf = 0;
    if (c.lane == 0) {
        auto P = [&](int i) { return (i >= 0 && i < WIN) ? s->phi[i] : 0.0; };
        int np = 0;
        s->lstart2[1] = 0;
        for (int m = 1; m <= NN2; ++m)
            for (int j = s->lstart[m]; j < s->lstart[m + 1]; ++j) {
                const int i = s->lst[j];
                if (P(i) * P(i + 1) < 0.0 || P(i) * P(i - 1) < 0.0) {
                    s->lst2[np++] = i;
                    s->mask[i] = 1;
                } else {
                    s->mask[i] = 2;
                }
            }
        const double d = sqrt(0.0 + 0.0 + c.hf * c.hf);
        for (int m = 2; m <= N_MAX; ++m) {
            s->lstart2[m] = np;
            for (int j = s->lstart2[m - 1]; j < s->lstart2[m]; ++j) {
                const int i = s->lst2[j];
                for (int i2 = i - 1; i2 <= i + 1; ++i2) {
                    const int k2 = c.w0 + i2;
                    if (k2 == 1 || k2 == c.nf + 1) continue;
                    if (i2 < 0 || i2 >= WIN) { ovf = 1; continue; }
                    if (s->mask[i2] == 1) continue;
                    if (s->mask[i2] == 0 || m >= NN2) s->phi[i2] = (s->phi[i] >= 0.0) ? s->phi[i] + d : s->phi[i] - d;
                    s->lst2[np++] = i2;
                    s->mask[i2] = 1;
                }
            }
        }
        s->lstart2[N_MAX + 1] = np;
        // the new band must keep its stencil halo inside the window, unless the window
        // already ends at the column end on that side
        int lo = WIN, hi = -1;
        for (int j = 0; j < np; ++j) {
            lo = min(lo, s->lst2[j]);
            hi = max(hi, s->lst2[j]);
        }
        if (np > 0 && ((lo < EDGE && c.w0 > -2) || (hi > WIN - 1 - EDGE && c.w0 + WIN - 1 < c.nf + 4))) ovf = 1;
        for (int j = 0; j < np; ++j) s->lst[j] = s->lst2[j];
        for (int m = 1; m <= N_MAX + 1; ++m) s->lstart[m] = s->lstart2[m];
    }
    __syncwarp();
    lists_to_layer(c);
    return __shfl_sync(0xffffffffu, ovf, 0);
}

// HJWENO, two_phase.f:2477-2500.
__device__ __forceinline__ double hjweno(double a, double b, double cc, double dd) {
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

// face differences dp(i) = (phi(i+1) - phi(i)) * SSDZF over the window
__device__ inline void face_diff(Ctx& c) {
    Win* s = c.s;
    // the WENO stencils of band cells read dp over [blo-3, bhi+2]
    for (int i = max(0, c.blo - 3) + c.lane; i <= min(WIN - 1, c.bhi + 3); i += 32) {
        const double b = (i + 1 < WIN) ? s->phi[i + 1] : 0.0;
        s->dp[i] = (b - s->phi[i]) * c.ssdzf;
    }
    __syncwarp();
}

// one-sided WENO5 derivatives at window cell i (two_phase.f:1170-1290, z part)
__device__ __forceinline__ void weno_z(const Win* s, int i, double& dm, double& dpl) {
    {
        const double v1 = s->dp[i - 3], v2 = s->dp[i - 2], v3 = s->dp[i - 1], v4 = s->dp[i], v5 = s->dp[i + 1];
        const double w = hjweno(v2 - v1, v3 - v2, v4 - v3, v5 - v4);
        dm = 1.0 / 12.0 * (-v2 + 7.0 * v3 + 7.0 * v4 - v5) - w;
    }
    {
        const double v1 = s->dp[i + 2], v2 = s->dp[i + 1], v3 = s->dp[i], v4 = s->dp[i - 1], v5 = s->dp[i - 2];
        const double w = hjweno(v1 - v2, v2 - v3, v3 - v4, v4 - v5);
        dpl = 1.0 / 12.0 * (-v5 + 7.0 * v4 + 7.0 * v3 - v2) + w;
    }
}

// TRANSPORT_RK3, two_phase.f:1133-1495 (1-D): one upwind/LLF stage on layers 1..NN1 plus
// the phase-change source, liquid side divided by DENR (:1466-1477).
__device__ inline void transport_rk3(Ctx& c, double dtlvs, int iphs, double denr) {
    Win* s = c.s;
    face_diff(c);
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int m = s->layer[i];
        if (m < 1 || m > NN1) continue;
        const double uu1 = s->wf[i], uu2 = s->wf[i + 1], uu3 = 0.5 * (uu1 + uu2);
        double dm, dpl, az;
        weno_z(s, i, dm, dpl);
        if (uu1 >= 0.0 && uu2 >= 0.0 && uu3 >= 0.0) {
            az = uu3 * dm;
        } else if (uu1 <= 0.0 && uu2 <= 0.0 && uu3 <= 0.0) {
            az = uu3 * dpl;
        } else {
            const double umax = fmax(fmax(fabs(uu1), fabs(uu2)), fabs(uu3));
            az = 0.5 * (uu3 * (dpl + dm) - umax * (dpl - dm));
        }
        double pn = s->phi[i] - dtlvs * ((0.0 + 0.0) + az);
        if (iphs == 1) {
            if (s->start[i] > 0.0) pn = pn - dtlvs * s->mf[i] / denr;
            else pn = pn - dtlvs * s->mf[i];
        }
        s->nv[i] = pn;
    }
    __syncwarp();
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int m = s->layer[i];
        if (m >= 1 && m <= NN1) s->phi[i] = s->nv[i];
    }
    __syncwarp();
}

// GODUNOV, two_phase.f:2448-2474.
__device__ __forceinline__ double godunov(double sg, double ap, double am) {
    const double aplus = sg * ap, aminus = sg * am;
    if (aplus >= 0.0 && aminus >= 0.0) return am;
    if (aplus <= 0.0 && aminus <= 0.0) return ap;
    if (aplus > 0.0 && aminus < 0.0) return 0.0;
    if (aplus + aminus > 0.0) return am;
    return ap;
}

// REINITIALIZATION_RK3, two_phase.f:2174-2445 (1-D): WENO on layers 1..NN1, first-order
// one-sided differences on NN1+1..NN2, Peng's smoothed sign with eps = min(h)^2.
__device__ inline void reinit_rk3(Ctx& c, double redtl) {
    Win* s = c.s;
    const double eps = c.hf * c.hf;
    face_diff(c);
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int m = s->layer[i];
        if (m < 1 || m > NN2) continue;
        const double dz = 0.5 * (s->phi[i + 1] - s->phi[i - 1]) * c.ssdzf;
        const double dal = (0.0 + 0.0) + dz * dz;
        const double a0 = s->alphio[i];
        const double sg = a0 / sqrt(a0 * a0 + dal * eps);
        double dm, dpl;
        if (m <= NN1) {
            weno_z(s, i, dm, dpl);
        } else {
            dm = (s->phi[i] - s->phi[i - 1]) * c.ssdzf;
            dpl = (s->phi[i + 1] - s->phi[i]) * c.ssdzf;
        }
        const double ax = godunov(sg, 0.0, 0.0), ay = godunov(sg, 0.0, 0.0);
        const double az = godunov(sg, dpl, dm);
        const double drhs = sg * (1.0 - sqrt(ax * ax + ay * ay + az * az));
        s->nv[i] = s->phi[i] + redtl * drhs;
    }
    __syncwarp();
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int m = s->layer[i];
        if (m >= 1 && m <= NN2) s->phi[i] = s->nv[i];
    }
    __syncwarp();
}

// REINITIALIZATION, two_phase.f:2033-2170: ILIMIT pseudo-time SSP-RK3 steps, dtau = h/2.
__device__ inline void reinitialization(Ctx& c, int ilimit) {
    Win* s = c.s;
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) s->alphio[i] = s->phi[i];
    __syncwarp();
    const double redtl = 0.5 * c.hf;
    for (int it = 0; it < ilimit; ++it) {
        for (int i = c.blo + c.lane; i <= c.bhi; i += 32) s->rk3[i] = s->phi[i];
        __syncwarp();
        reinit_rk3(c, redtl);
        reinit_rk3(c, redtl);
        for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            if (m >= 1 && m <= NN2) s->phi[i] = 0.75 * s->rk3[i] + 0.25 * s->phi[i];
        }
        __syncwarp();
        reinit_rk3(c, redtl);
        for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            if (m >= 1 && m <= NN2) s->phi[i] = 1.0 / 3.0 * s->rk3[i] + 2.0 / 3.0 * s->phi[i];
        }
        __syncwarp();
    }
}

// REIN_TRIGGER, two_phase.f:646-697: max and min of |grad phi| over layers 1..NN1.
__device__ inline void rein_trigger(Ctx& c, double& dmax, double& dmin) {
    const Win* s = c.s;
    double mx = 0.0, mn = 1.0;
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int m = s->layer[i];
        if (m < 1 || m > NN1) continue;
        const double dz = 0.5 * (s->phi[i + 1] - s->phi[i - 1]) * c.ssdzf;
        const double v = (0.0 + 0.0) + dz * dz;
        mx = fmax(v, mx);
        mn = fmin(v, mn);
    }
    dmax = sqrt(warp_max(mx));
    dmin = sqrt(warp_min(mn));
}

// VEL_INTP / VELASSIGN, two_phase.f:5539-6035 (1-D): 4-point Lagrange interpolation in z of
// the time-averaged face velocity on the flow cell-centre nodes ZP(KK-1..KK+2),
// KK = KCOU_VEL(k); half on layers NN2-1..NN2, zero on layer N_MAX (:5641-5663).
// Returns nonzero if a stencil left the flow-face window (not expected, see the window
// bounds where it is filled).
__device__ inline int vel_intp(Ctx& c) {
    Win* s = c.s;
    const int n = c.n;
    const double h = c.h;
    const col::ColGeoDev* cg = c.cg;
    auto zp = [&](int k) { return cg ? cg->zp[k] : (k - 1) * h + 0.5 * h; };
    auto vdz = [&](int k) { return cg ? cg->vdz[k] : ((k == 1 || k == n + 1) ? 0.5 * h : h); };
    int bad = 0;
    auto wtv = [&](int k) {
        const int j = k - c.kw0;
        if (j < 0 || j >= WTN) {
            bad = 1;
            return 0.0;
        }
        return s->wt[j];
    };
    // the band slots, and the slots the previous call wrote (reset to 0 when they left it)
    const int vlo = min(c.blo, c.vhi >= 0 ? c.vlo : c.blo), vhi = max(c.bhi, c.vhi);
    for (int i = vlo + c.lane; i <= vhi; i += 32) {
        const int k = c.w0 + i, m = s->layer[i];
        double out = 0.0;
        if (m >= 1 && m <= NN2) {
            const double zz = (k - 1) * c.hf;
            // KCOU_VEL by the search of GEOM_COUPLING (1d.f:5130-5240).  Every q below
            // k/2 - 2 has ZP(q) at least 2.5 flow cells under zz and fails all four tests
            // but the two that do not depend on q, so starting there gives the same KK.
            int kk = 1;
            if (cg) {
                kk = cg->kcou_vel[k];   // the same search, tabulated by GEOM_COUPLING
            } else {
                for (int qq = max(1, k / 2 - 2); qq <= n; ++qq) {
                    if (fabs(zz - zp(qq)) <= 1e-10) { kk = qq; break; }
                    if (zp(1) > zz) { kk = 1; break; }
                    if (zp(qq) > zz) { kk = qq - 1; break; }
                    if (zp(n) < zz) { kk = n; break; }
                }
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
            out = (m < NN2 - 1) ? w : w * 0.5;
        }
        s->wf[i] = out;
    }
    __syncwarp();
    c.vlo = c.blo;
    c.vhi = c.bhi;
    return __any_sync(0xffffffffu, bad) ? 1 : 0;
}

// CAL_PSIF_MTP, two_phase.f:2876-2931, at a band cell: the cut-cell volume fraction from
// phi and its central differences (D1 = D2 = 0 in 1-D), snapped at 1e-5 / 0.99999.
__device__ __forceinline__ double psif_band(const Win* s, int i) {
    const double d3 = 0.5 * fabs(s->phi[i + 1] - s->phi[i - 1]);
    const double e1 = d3;
    double t;
    if (e1 > 1e-8) {
        const double f1 = fmax(0.5 * (e1 + 0.0 + 0.0) - fabs(s->phi[i]), 0.0);
        t = f1 / e1;
    } else {
        t = (s->phi[i] != 0.0) ? 0.0 : 0.5;
    }
    double ps = (s->phi[i] <= 0.0) ? t : 1.0 - t;
    if (ps < 1e-5) ps = 0.0;
    else if (ps > 0.99999) ps = 1.0;
    return ps;
}

// Interface crossings of the column fill of CAL_PSIF_MTP(1) (two_phase.f:2936-3049):
// ktop = the largest, kbot = the smallest k in 1..nf with phi(k) phi(k+1) < 0, -1 if none.
// phi is zero outside the window, so only window cells can cross; warp-wide, every lane
// gets the result.
__device__ inline void window_crossings(Ctx& c, int& ktop, int& kbot) {
    const Win* s = c.s;
    int top = -1, bot = 1 << 30;
    // a crossing needs phi != 0 on both cells: band cells (or a band cell next to a ghost)
    for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
        const int k = c.w0 + i;
        if (k >= 1 && k <= c.nf && i + 1 < WIN && s->phi[i] * s->phi[i + 1] < 0.0) {
            top = max(top, k);
            bot = min(bot, k);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
        bot = min(bot, __shfl_xor_sync(0xffffffffu, bot, o));
    }
    ktop = top;
    kbot = (top < 0) ? -1 : bot;
}

// Vapour volume of the whole column, sum over k = 1..nf of four replicas of
// (1 - PSIF) * DVOL in the reference's order (two_phase.f:6230-6290), with PSIF = band_ps on
// the window cells of layers 1..NN1 and the column fill elsewhere.  Outside the window the
// fill is constant below and above it (the crossings lie inside), and adding 0.0 leaves
// the sum unchanged, so only nonzero terms are added.  Lane 0 only.
__device__ inline double column_vapour_volume(Ctx& c, const double* band_ps, int ktop, int kbot, double dvol) {
    const Win* s = c.s;
    double t1 = 1.0, t2 = 1.0;
    if (ktop >= 0) {
        t1 = (c.p(ktop) < 0.0) ? 0.0 : 1.0;
        t2 = (c.p(kbot + 1) < 0.0) ? 0.0 : 1.0;
    }
    auto fill = [&](int k) { return (ktop < 0) ? 1.0 : ((k > kbot) ? t2 : t1); };
    double vt = 0.0;
    const int wlo = max(1, c.w0), whi = min(c.nf, c.w0 + WIN - 1);
    // below the window
    if (wlo > 1) {
        const double d = (1.0 - fill(1)) * dvol;
        if (d != 0.0)
            for (int k = 1; k < wlo; ++k) {
                vt = vt + d;
                vt = vt + d;
                vt = vt + d;
                vt = vt + d;
            }
    }
    for (int k = wlo; k <= whi; ++k) {
        const int i = k - c.w0;
        const double ps = (s->layer[i] >= 1 && s->layer[i] <= NN1) ? band_ps[i] : fill(k);
        const double d = (1.0 - ps) * dvol;
        if (d != 0.0) {
            vt = vt + d;
            vt = vt + d;
            vt = vt + d;
            vt = vt + d;
        }
    }
    if (whi < c.nf) {
        const double d = (1.0 - fill(c.nf)) * dvol;
        if (d != 0.0)
            for (int k = whi + 1; k <= c.nf; ++k) {
                vt = vt + d;
                vt = vt + d;
                vt = vt + d;
                vt = vt + d;
            }
    }
    return vt;
}

// GLOBAL_MASS_CORRECTION, two_phase.f:6196-6318 (1-D, DVOL = SDXF*SDYF*SDZF with
// SDXF = SDYF = 1/2, four (I,J) replicas per z-level): up to 15 uniform shifts of the
// band phi (layers 1..NN1) towards the target vapour volume.  The first pass sums the
// whole column with the column fill of CAL_PSIF_MTP(1) (:2936-3049), later passes only
// the band.  The sums run on lane 0 in the reference's order.
__device__ inline void global_mass_correction(Ctx& c, double& vol_tot_ori, double vol_tot_iphs, int iphs) {
    Win* s = c.s;
    const double recor = fmin(fmin(0.5, 0.5), c.hf) * 1.5;
    const double dvol = 0.5 * 0.5 * c.hf;
    if (iphs == 1) vol_tot_ori = vol_tot_iphs;
    double vol_in = 0.0;
    for (int l = 1; l <= 15; ++l) {
        for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            s->nv[i] = (m >= 1 && m <= NN1) ? psif_band(s, i) : 0.0;
        }
        __syncwarp();
        double vol_tot = 0.0;
        int ktop = -1, kbot = -1;
        if (l == 1) window_crossings(c, ktop, kbot);
        if (c.lane == 0) {
            double vol_band = 0.0;
            for (int j = s->lstart[1]; j < s->lstart[NN1 + 1]; ++j) {
                const double v = (1.0 - s->nv[s->lst[j]]) * dvol;
                vol_band = vol_band + v;
                vol_band = vol_band + v;
                vol_band = vol_band + v;
                vol_band = vol_band + v;
            }
            if (l == 1) {
                vol_tot = column_vapour_volume(c, s->nv, ktop, kbot, dvol);
                vol_in = vol_tot - vol_band;
            } else {
                vol_tot = vol_in + vol_band;
            }
        }
        vol_tot = __shfl_sync(0xffffffffu, vol_tot, 0);
        vol_in = __shfl_sync(0xffffffffu, vol_in, 0);
        if (fabs(vol_tot - vol_tot_ori) >= 1e-5) {
            const double cor = recor * (-(vol_tot_ori - vol_tot) / vol_tot_ori);
            for (int i = c.blo + c.lane; i <= c.bhi; i += 32) {
                const int m = s->layer[i];
                if (m >= 1 && m <= NN1) s->phi[i] = s->phi[i] + cor;
            }
            __syncwarp();
        } else {
            break;
        }
    }
}

struct Params {
    int iphs, first, m_step, mglobal;
    double denr, dtconst;
};

// TRANSPORT for one column (one warp), followed by CAL_PSIF(0) and GRID_COUPLING(0).
// Returns the column's status; on LICA_BAND_OVERFLOW (or LICA_BAD_ARG: a band cell
// outside k = 1..nf) nothing of the column is written.
__device__ inline int transport_column(Win* s, int lane, int n, double length, double* phi, int* layer, double* psif,
                                double* wo, const double* w, const double* mf, double* vol_ori, double vol_iphs,
                                double* psi_cn, double* psi_zn, double* stats, const Params& P,
                                const col::ColGeoDev* cg = nullptr) {
    Ctx c;
    c.cg = cg;
    c.n = n;
    c.nf = 2 * n;
    c.h = length / n;
    c.hf = length / c.nf;
    c.ssdzf = 1.0 / c.hf;
    c.lane = lane;
    c.s = s;
    const int nf = c.nf;

    // band extent -> window origin (the band is centred; the window is clamped to the column).
    // Band cells live on k = 1..nf (BAND_GENERATION never goes past k = 1 or nf); a band
    // cell elsewhere is rejected, which keeps every stencil inside the window.
    int kmin = 1 << 30, kmax = -(1 << 30);
    for (int k = -2 + lane; k <= nf + 4; k += 32)
        if (layer[k + 2] > 0) {
            kmin = min(kmin, k);
            kmax = max(kmax, k);
        }
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (kmax >= kmin && (kmin < 1 || kmax > nf)) return LICA_BAD_ARG;
    if (kmax >= kmin && kmax - kmin + 1 > WIN - 2 * HALO) return LICA_BAND_OVERFLOW;
    int w0 = (kmax >= kmin) ? (kmin + kmax + 1) / 2 - WIN / 2 : -2;
    w0 = max(w0, -2);
    w0 = min(w0, max(-2, nf + 4 - (WIN - 1)));
    c.w0 = w0;
    c.kw0 = flow_origin(c, w0);

    // ALPHI_EXT = 0 outside the band, band phi inside (:750-767); ALPHI at entry for the
    // phase test of the source
    for (int q = 0; q < PER; ++q) {
        const int i = lane + 32 * q, k = w0 + i;
        const bool ok = (k >= -2 && k <= nf + 4);
        const int m = ok ? layer[k + 2] : 0;
        s->layer[i] = m;
        s->phi[i] = (ok && m > 0) ? phi[k + 2] : 0.0;
        s->start[i] = s->phi[i];
        s->mf[i] = ok ? mf[k + 2] : 0.0;
        s->wf[i] = 0.0;
    }
    if (lane < 7) s->ghost[lane] = 0.0;
    // VEL_INTP(2): UT = (U + UO)/2 with UO = U on the first call (:5567-5600); UO = U after
    for (int j = lane; j < WTN; j += 32) {
        const int k = c.kw0 + j;
        double v = 0.0;
        if (k >= 0 && k <= n + 1) v = 0.5 * (w[k] + (P.first ? w[k] : wo[k]));
        s->wt[j] = v;
    }
    __syncwarp();
    build_lists(c);
    alphi_bc(c);
    int ovf = vel_intp(c);
    double time_tran = 0.0, dmax = 0.0, dmin = 0.0, vo = *vol_ori;
    int imass = 0, isub;
    bool skipped = false;
    for (isub = 1; isub <= 10; ++isub) {
        // subcycle step at CFL 1 on layers 1..NN1 (:800-850)
        double cm = 0.0;
        for (int i = c.blo + lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            if (m < 1 || m > NN1) continue;
            const double cz = fabs(0.5 * (s->wf[i - 1] + s->wf[i])) * c.ssdzf;
            cm = fmax(cm, (0.0 + 0.0) + cz);
        }
        cm = warp_max(cm);
        double dtlvs;
        if (cm == 0.0) {
            double uvw = 0.0;
            if (lane == 0)
                for (int j = s->lstart[1]; j < s->lstart[NN1 + 1]; ++j) uvw = uvw + ((0.0 + 0.0) + s->wf[s->lst[j]]);
            uvw = __shfl_sync(0xffffffffu, uvw, 0);
            if (uvw == 0.0) {
                if (P.iphs != 1) {
                    skipped = true;
                    break;
                }
                dtlvs = P.dtconst / 10.0;
            } else {
                dtlvs = 1.0 / cm;
            }
        } else {
            dtlvs = 1.0 / cm;
        }
        if (time_tran + dtlvs >= P.dtconst) dtlvs = P.dtconst - time_tran;
        time_tran = time_tran + dtlvs;
        for (int i = c.blo + lane; i <= c.bhi; i += 32) s->rk3[i] = s->phi[i];
        __syncwarp();
        transport_rk3(c, dtlvs, P.iphs, P.denr);
        transport_rk3(c, dtlvs, P.iphs, P.denr);
        for (int i = c.blo + lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            if (m >= 1 && m <= NN1) s->phi[i] = 0.75 * s->rk3[i] + 0.25 * s->phi[i];
        }
        __syncwarp();
        transport_rk3(c, dtlvs, P.iphs, P.denr);
        for (int i = c.blo + lane; i <= c.bhi; i += 32) {
            const int m = s->layer[i];
            if (m >= 1 && m <= NN1) s->phi[i] = 1.0 / 3.0 * s->rk3[i] + 2.0 / 3.0 * s->phi[i];
        }
        __syncwarp();
        rein_trigger(c, dmax, dmin);
        imass = (dmax > 2.0 || dmin < 1e-4) ? 1 : 0;
        if (P.iphs == 1) {
            reinitialization(c, NN2);
            if (P.m_step % 50 == 0) imass = 1;
        }
        if (dmax > 2.0 || dmin < 1e-4 || imass == 1) {
            if (P.mglobal == 1 && imass == 1) global_mass_correction(c, vo, vol_iphs, P.iphs);
            alphi_bc(c);
            ovf |= band_generation(c);
            if (ovf) break;   // before any stencil touches the new band
            alphi_bc(c);
            reinitialization(c, NN2);
        }
        alphi_bc(c);
        if (time_tran == P.dtconst) break;
        if (dmax > 2.0 || dmin < 1e-4) ovf |= vel_intp(c);
    }
    if (isub > 10) isub = 10;
    if (ovf) return LICA_BAND_OVERFLOW;

    if (!skipped) {
        // CAL_PSIF(0): PSIF = CAL_PSIF_MTP on layers 1..NN1, then the snap of the whole
        // array (:2600-2680)
        for (int k = 1 + lane; k <= nf; k += 32) {
            const int i = k - w0;
            double v;
            if (c.in(k) && s->layer[i] >= 1 && s->layer[i] <= NN1) {
                v = psif_band(s, i);
            } else {
                v = psif[k];
                if (v < 1e-5) v = 0.0;
                else if (v > 0.99999) v = 1.0;
            }
            psif[k] = v;
        }
        if (imass == 0 && P.iphs == 1) vo = vol_iphs;
    }
    // band phi and layers stored (ALPHI = ALPHI_EXT on the band); zero elsewhere except
    // the ghosts ALPHI_BC set
    for (int k = -2 + lane; k <= nf + 4; k += 32) {
        double v;
        int m;
        if (c.in(k)) {
            v = s->phi[k - w0];
            m = s->layer[k - w0];
        } else {
            m = 0;
            v = (k <= 0) ? s->ghost[k + 2] : (k >= nf + 1 ? s->ghost[k - nf + 2] : 0.0);
        }
        phi[k + 2] = v;
        layer[k + 2] = m;
    }
    for (int k = lane; k <= n + 1; k += 32) wo[k] = w[k];
    if (skipped) {
        if (lane == 0) {
            *vol_ori = vo;
            stats[0] = 0.0;
        }
        return LICA_OK;
    }
    __syncwarp();   // psif visible to the whole warp
    // GRID_COUPLING(0) (two_phase.f:4863-5118): the flow cells KCOUMP_VEL(k) of the band
    // cells of layers 1..NN1 on k = 1..nf (MASK_GLOBAL, set by CAL_PSIF) take the box
    // means of PSIF over [ZP(K-1),ZP(K)] (PSI_ZN, K >= 2) and [Z(K),Z(K+1)] (PSI_CN); all
    // cells are snapped at 1e-3 / 0.999 (:5000-5061).
    for (int j = lane; j < WTN; j += 32) s->fmask[j] = 0;
    __syncwarp();
    for (int i = c.blo + lane; i <= c.bhi; i += 32) {
        const int k = w0 + i, m = s->layer[i];
        if (m >= 1 && m <= NN1 && k >= 1 && k <= nf) {
            const int j = ctx_kcoump_vel(c, k) - c.kw0;   // inside the window's face range
            if (j >= 0 && j < WTN) s->fmask[j] = 1;
        }
    }
    __syncwarp();
    for (int kk = 1 + lane; kk <= n; kk += 32) {
        const int j = kk - c.kw0;
        const bool mk = (j >= 0 && j < WTN) && s->fmask[j] != 0;
        double zn = psi_zn[kk];
        const col::ColGeoDev* cg = c.cg;
        // INTER_PSI over the face box [ZP(K-1), ZP(K)], refined cells KCOUMP2(K-1)..KCOUMP1(K)
        if (kk >= 2 && mk)
            zn = col::box_mean(psif, nf, cg ? cg->kcoump2[kk] : 2 * kk - 2, cg ? cg->kcoump1[kk + 1] : 2 * kk - 1,
                               cg ? cg->zp[kk - 1] : col::grid_zp(c.h, n, kk - 1),
                               cg ? cg->zp[kk] : col::grid_zp(c.h, n, kk), c.hf);
        if (zn < 1e-3) zn = 0.0;
        else if (zn > 0.999) zn = 1.0;
        psi_zn[kk] = zn;
        double cn = psi_cn[kk];
        // over the cell box [Z(K), Z(K+1)], refined cells KCOU2(K)..KCOU1(K+1)
        if (mk)
            cn = col::box_mean(psif, nf, cg ? cg->kcou2[kk + 1] : 2 * kk - 1, cg ? cg->kcou1[kk + 2] : 2 * kk,
                               cg ? cg->z[kk] : col::grid_z(c.h, kk), cg ? cg->z[kk + 1] : col::grid_z(c.h, kk + 1),
                               c.hf);
        if (cn < 1e-3) cn = 0.0;
        else if (cn > 0.999) cn = 1.0;
        psi_cn[kk] = cn;
    }
    __syncwarp();
    if (lane == 0) {
        psi_cn[0] = psi_cn[1];
        psi_cn[n + 1] = psi_cn[n];
        *vol_ori = vo;
        stats[0] = isub;
        stats[1] = dmax;
        stats[2] = dmin;
        stats[3] = imass;
    }
    return LICA_OK;
}

}  // namespace lvs
}  // namespace lica
