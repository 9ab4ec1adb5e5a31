// Persistent, TMA-staged forms of the two PCG vector kernels on level 0 (k_cg_tma): the
// same arithmetic as k_pupdate / k_xupdate, cell for cell, with the tiles streamed through a
// CG_STAGES-deep shared-memory ring.  A CTA (one per SM, 512 threads) walks tiles t, t + grid,
// ...; while it computes tile t the TMA copies of tile t + grid are in flight, so the
// per-tile load latency of the one-tile-per-CTA kernels is hidden.
//
// Tile 32 x 32; a box covers global columns gi0 = 32 tx - 4 .. gi0 + 39 (16-byte aligned
// for FP32 and FP64) and rows gj0 = 32 ty - 1 .. gj0 + 33: the tile and the one-cell ring
// the stencil reads.  x is periodic: the first and last tile columns also copy the 4
// columns at the far end of the row.  Rows off the domain are zero-filled by the TMA, as
// the per-tile kernels' loads fill them.
//
// k_pupdate_tma: p_new = z + beta p_old on the tile (and, as the stencil reads them, on its
//   one-cell ring), then p_new.(A p_new) on the tile; the last CTA sets alpha = rz / p.Ap.
// k_xupdate_tma: x_new = x + alpha p likewise, r = f - A x_new on the tile
//   (stored as TR), ||r||^2; the last CTA runs xupdate_finish.
// Every wait is bounded (tc::mbar_wait); one that runs out sets State::kerr.
#pragma once
#include <cuda.h>

#include <type_traits>

#include "tc_sm100.cuh"

namespace lica {
namespace mg {

constexpr int CG_TS = 32;
constexpr int CG_BW = 40;      // box width (columns gi0 .. gi0 + 39)
constexpr int CG_BH = 34;      // box height (rows gj0 .. gj0 + 33)
constexpr int CG_X0 = 4;       // box column of tile column 0
constexpr int CG_WW = 4;       // wrap strip width
constexpr int CG_NT = 512;   // 32 rows x 16 column pairs of a tile
#ifndef LICA_CG_STAGES
#define LICA_CG_STAGES 2
#endif
constexpr int CG_STAGES = LICA_CG_STAGES;   // tiles in flight + 1

struct CgMaps {
    // by iteration parity: p_old / x read from [par], written to [par ^ 1]
    CUtensorMap p[2], pw[2], x[2], xw[2], z, zw, f, ax, axw, ay;
};

struct CgArgs {
    CgMaps m;
    double* pbuf[2];   // the two p buffers (p_new is written to pbuf[par ^ 1])
    double* xbuf[2];   // the two x buffers (x_new to xbuf[par ^ 1])
    void* r_out;       // r (TR) for the preconditioner
    int nx, ny, ntx, nty;
    State* st;
    double* partials;
    cudaGraphConditionalHandle cond;
    int use_cond;
};

// One stage of the ring, boxes A, B, C, AX, AY and the wrap strips of A, B, AX.
//   k_pupdate's: A = p_old, B = z (TB = the V-cycle's type), C unused.
//   k_xupdate's: A = x, B = p (TB = double), C = f.
template <typename TB>
struct CgStage {
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int B8 = al(CG_BW * CG_BH * 8);
    static constexpr int BT = al(CG_BW * CG_BH * (int)sizeof(TB));
    static constexpr int W8 = al(CG_WW * CG_BH * 8);
    static constexpr int WT = al(CG_WW * CG_BH * (int)sizeof(TB));
    static constexpr int A = 0;
    static constexpr int B = A + B8;
    static constexpr int C = B + BT;
    static constexpr int AX = C + B8;
    static constexpr int AY = AX + B8;
    static constexpr int WA = AY + B8;
    static constexpr int WB = WA + W8;
    static constexpr int WAX = WB + WT;
    static constexpr int BYTES = WAX + W8;
};

template <typename TZ, bool XUP>
struct CgLayout {
    using TB = typename std::conditional<XUP, double, TZ>::type;
    using S = CgStage<TB>;
    static constexpr int BYTES = CG_STAGES * S::BYTES + 128;  // + room to align the base
    // transaction bytes of one tile's copies (whole boxes, filled parts included)
    static constexpr uint32_t TX_MAIN =
        (uint32_t)(CG_BW * CG_BH * (3 * 8 + (int)sizeof(TB) + (XUP ? 8 : 0)));
    static constexpr uint32_t TX_WRAP = (uint32_t)(CG_WW * CG_BH * (2 * 8 + (int)sizeof(TB)));
};

// Thread 0: the copies of one tile into stage buffer sb (bar: its barrier).
template <typename TZ, bool XUP>
__device__ __forceinline__ void cg_issue(const CgArgs& A, unsigned char* sb, uint64_t* bar, int tile, int par) {
    using Lay = CgLayout<TZ, XUP>;
    using S = typename Lay::S;
    const int tx = tile % A.ntx, ty = tile / A.ntx;
    const int gi0 = tx * CG_TS - CG_X0, gj0 = ty * CG_TS - 1;
    const bool edge = (tx == 0 || tx == A.ntx - 1);
    tc::mbar_expect_tx(bar, Lay::TX_MAIN + (edge ? Lay::TX_WRAP : 0u));
    if (XUP) {
        tc::tma_load_2d(sb + S::A, &A.m.x[par], bar, gi0, gj0);
        tc::tma_load_2d(sb + S::B, &A.m.p[par ^ 1], bar, gi0, gj0);
        tc::tma_load_2d(sb + S::C, &A.m.f, bar, gi0, gj0);
    } else {
        tc::tma_load_2d(sb + S::A, &A.m.p[par], bar, gi0, gj0);
        tc::tma_load_2d(sb + S::B, &A.m.z, bar, gi0, gj0);
    }
    tc::tma_load_2d(sb + S::AX, &A.m.ax, bar, gi0, gj0);
    tc::tma_load_2d(sb + S::AY, &A.m.ay, bar, gi0, gj0);
    if (edge) {
        const int wx = (tx == 0) ? A.nx - CG_WW : 0;
        if (XUP) {
            tc::tma_load_2d(sb + S::WA, &A.m.xw[par], bar, wx, gj0);
            tc::tma_load_2d(sb + S::WB, &A.m.pw[par ^ 1], bar, wx, gj0);
        } else {
            tc::tma_load_2d(sb + S::WA, &A.m.pw[par], bar, wx, gj0);
            tc::tma_load_2d(sb + S::WB, &A.m.zw, bar, wx, gj0);
        }
        tc::tma_load_2d(sb + S::WAX, &A.m.axw, bar, wx, gj0);
    }
}

// XUP = false: k_pupdate's work (TZ = the V-cycle's type); XUP = true: k_xupdate's (TZ = TR).
template <typename TZ, bool XUP>
__global__ void __launch_bounds__(CG_NT, 1) k_cg_tma(const __grid_constant__ CgArgs A) {
    using Lay = CgLayout<TZ, XUP>;
    using S = typename Lay::S;
    extern __shared__ __align__(16) unsigned char cg_smem_raw[];
    unsigned char* sm = cg_smem_raw + ((128u - (tc::smem_u32(cg_smem_raw) & 127u)) & 127u);
    __shared__ __align__(8) uint64_t bar[CG_STAGES];
    __shared__ double red[32];
    const int ntiles = A.ntx * A.nty;
    const int par = A.st->it & 1;
    const double coef = XUP ? A.st->alpha : A.st->beta;
    if (threadIdx.x == 0) {
        for (int q = 0; q < CG_STAGES; ++q) tc::mbar_init(&bar[q], 1);
        tc::fence_barrier_init();
    }
    __syncthreads();
    // the first CG_STAGES - 1 tiles in flight
    if (threadIdx.x == 0)
        for (int q = 0; q + 1 < CG_STAGES; ++q) {
            const int t = (int)blockIdx.x + q * (int)gridDim.x;
            if (t < ntiles) cg_issue<TZ, XUP>(A, sm + q * S::BYTES, &bar[q], t, par);
        }
    double acc = 0.0;
    bool failed = false;
    int i = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
        const int s = i % CG_STAGES;
        // tile i + CG_STAGES - 1 into the stage tile i - 1 used (its last reader finished
        // before the barrier that closed the previous iteration)
        {
            const int t = tile + (CG_STAGES - 1) * (int)gridDim.x;
            const int sn = (i + CG_STAGES - 1) % CG_STAGES;
            if (threadIdx.x == 0 && t < ntiles) cg_issue<TZ, XUP>(A, sm + sn * S::BYTES, &bar[sn], t, par);
        }
        const int ok = tc::mbar_wait(&bar[s], (uint32_t)((i / CG_STAGES) & 1)) ? 1 : 0;
        if (!__syncthreads_and(ok)) {
            // let the copies still in flight land (bounded) before the CTA leaves
            if (threadIdx.x == 0)
                for (int q = 1; q < CG_STAGES; ++q) {
                    const int t = tile + q * (int)gridDim.x;
                    if (t < ntiles) (void)tc::mbar_wait(&bar[(i + q) % CG_STAGES], (uint32_t)(((i + q) / CG_STAGES) & 1));
                }
            failed = true;
            break;
        }
        unsigned char* sb = sm + s * S::BYTES;
        const int tx = tile % A.ntx, ty = tile / A.ntx;
        // edge tiles: the wrapped column -1 (first tile column) or nx (last) into the boxes,
        // so that the passes below index the boxes alone
        if (tx == 0 || tx == A.ntx - 1) {
            const int bc = (tx == 0) ? CG_X0 - 1 : CG_X0 + CG_TS;   // box column of the wrapped cell
            const int wc = (tx == 0) ? CG_WW - 1 : 0;               // its column in the strip
            for (int r = threadIdx.x; r < CG_BH; r += CG_NT) {
                double* a = reinterpret_cast<double*>(sb + S::A);
                a[r * CG_BW + bc] = reinterpret_cast<const double*>(sb + S::WA)[r * CG_WW + wc];
                typename Lay::TB* b = reinterpret_cast<typename Lay::TB*>(sb + S::B);
                b[r * CG_BW + bc] = reinterpret_cast<const typename Lay::TB*>(sb + S::WB)[r * CG_WW + wc];
                if (tx == A.ntx - 1) {   // the east weight of the last column is ax at nx (= ax at 0)
                    double* ax = reinterpret_cast<double*>(sb + S::AX);
                    ax[r * CG_BW + bc] = reinterpret_cast<const double*>(sb + S::WAX)[r * CG_WW + wc];
                }
            }
            // order these shared-memory writes before the next TMA copy into this stage
            tc::fence_async_smem();
            __syncthreads();
        }
        // the stencil on the tile: thread t owns cells 2 (t % 16) and 2 (t % 16) + 1 of row t / 16
        {
            const int ty_ = threadIdx.x >> 4, tx0 = (threadIdx.x & 15) * 2;
            const int br = ty_ + 1, bc = tx0 + CG_X0;
            const double* axb = reinterpret_cast<const double*>(sb + S::AX) + br * CG_BW + bc;
            const double* ayb = reinterpret_cast<const double*>(sb + S::AY) + br * CG_BW + bc;
            const size_t g = (size_t)(ty * CG_TS + ty_) * A.nx + tx * CG_TS + tx0;
            // the updated vector (p_new or x_new) at a box cell, formed where the stencil reads
            // it: each neighbour is recomputed rather than staged in a separate pass, which
            // saves that pass and one CTA barrier per tile
            const double* av = reinterpret_cast<const double*>(sb + S::A);
            const typename Lay::TB* bv = reinterpret_cast<const typename Lay::TB*>(sb + S::B);
            const int q0 = br * CG_BW + bc;
            auto upd = [&](int e, int off) {   // off: 0 the cell, +-1 east / west, +-CG_BW north / south
                const int q = q0 + e + off;
                return XUP ? av[q] + coef * double(bv[q]) : double(bv[q]) + coef * av[q];
            };
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const double aw = axb[e], ae = axb[e + 1], as = ayb[e], an = ayb[e + CG_BW];
                const double cw = upd(e, -1), ce = upd(e, 1), cs = upd(e, -CG_BW), cn = upd(e, CG_BW);
                double ss = aw * cw;
                ss += ae * ce;
                ss += as * cs;
                ss += an * cn;
                double dd = aw;
                dd += ae;
                dd += as;
                dd += an;
                const double v = upd(e, 0);
                if (XUP) {
                    const double fv = reinterpret_cast<const double*>(sb + S::C)[br * CG_BW + bc + e];
                    const double r = fv - (ss - dd * v);
                    acc += r * r;
                    A.xbuf[par ^ 1][g + e] = v;
                    reinterpret_cast<TZ*>(A.r_out)[g + e] = TZ(r);
                } else {
                    const double q = ss - dd * v;
                    acc += v * q;
                    A.pbuf[par ^ 1][g + e] = v;
                }
            }
        }
        __syncthreads();   // this stage is free again
    }
    if (failed) {
        if (threadIdx.x == 0) atomicExch(&A.st->kerr, 1);
        return;
    }
    const double b = block_sum(acc, red);
    double tot;
    if (XUP) {
        if (grid_sum_last(b, A.partials, &A.st->cnt[2], &tot, red)) xupdate_finish(A.st, tot, 0, A.cond, A.use_cond);
    } else {
        if (grid_sum_last(b, A.partials, &A.st->cnt[1], &tot, red)) A.st->alpha = A.st->rz / tot;
    }
}

}  // namespace mg
}  // namespace lica
