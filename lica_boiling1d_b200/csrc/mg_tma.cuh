// Persistent red-black smoothing kernels of the large multigrid levels, with every tile
// staged into shared memory by the tensor memory accelerator (TMA).
//
// The per-tile kernels k_down / k_up read a tile's f, weights and 1/d with ordinary loads
// at the start of each CTA, so their sweeps wait on global-memory latency once per tile
// and nothing is in flight while a CTA sweeps.  Here a CTA stays resident (two per SM)
// and walks tiles t, t + grid, ...: as soon as its threads have moved tile t's staged
// data into registers, one thread issues the TMA copies of its next tile into the same
// staging buffer, and those copies run while the CTA sweeps, writes and reduces tile t.
// The sweep, residual, restriction and write code is the per-tile kernels' own (down_body,
// up_body), so the results are bit-identical to theirs.
//
// Tile 32 x 32 with the halo of two sweeps (H = 4): region 40 x 40, 416 threads, four
// cells per thread.  Boxes of one tile (row-major, x fastest; outside the domain rows the
// TMA fills zeros, which is what the per-tile loads put there):
//   f, 1/d, u_pre : RX x RY at (gi0, gj0)          ax : 44 x RY (east weight of column 39)
//   ay : RX x (RY + 1) (north weight of row 39)     uc : 24 x 20 coarse at (gi0/2 - 2, gj0/2)
// x is periodic: the first and last tile columns also copy an 8-column strip of the far
// end of the row (4 columns for uc) and read the wrapped columns from it.  Every box
// starts on a 16-byte boundary in FP32 and FP64 (gi0 = 32 tx - 4).
//
// The wait for a tile's copies is bounded (tc::mbar_wait); if it runs out the kernel sets
// State::kerr and returns, and the PCG ends with LICA_ERR_CUDA.
#pragma once
#include <cuda.h>

#include "tc_sm100.cuh"

namespace lica {
namespace mg {

constexpr int TM_TS = 32;
using TmCfg = RBCfg<2, TM_TS, TM_TS, 4>;
constexpr int TM_H = TmCfg::H;
constexpr int TM_RX = TmCfg::RX;
constexpr int TM_RY = TM_TS + 2 * TM_H;
constexpr int TM_AXW = 44;
constexpr int TM_AYH = TM_RY + 1;
constexpr int TM_WW = 8;
constexpr int TM_CW = 24;
constexpr int TM_CH = TM_RY / 2;
constexpr int TM_CWW = 4;
static_assert(TmCfg::RY == TM_RY && TM_RX == 40 && TM_AXW >= TM_RX + 1, "tile geometry");

struct TmMaps {
    CUtensorMap f, fw, d, dw, ax, axw, ay, ayw, u, uw, c, cw;
};

template <typename T>
struct TmArgs {
    TmMaps m;
    T* out;     // k_down: u after pre-smoothing; k_up: u after post-smoothing
    T* fc;      // k_down: the restricted residual (the coarse level's f)
    int nx, ny, ntx, nty;
    State* st;
    double* partials;
};

// Shared-memory layout (byte offsets): the staged boxes, 128-byte aligned, then u.
template <typename T>
struct TmStage {
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int E = (int)sizeof(T);
    static constexpr int F = 0;
    static constexpr int D = F + al(TM_RY * TM_RX * E);
    static constexpr int AX = D + al(TM_RY * TM_RX * E);
    static constexpr int AY = AX + al(TM_RY * TM_AXW * E);
    static constexpr int U = AY + al(TM_AYH * TM_RX * E);
    static constexpr int C = U + al(TM_RY * TM_RX * E);
    static constexpr int WF = C + al(TM_CH * TM_CW * E);
    static constexpr int WD = WF + al(TM_RY * TM_WW * E);
    static constexpr int WAX = WD + al(TM_RY * TM_WW * E);
    static constexpr int WAY = WAX + al(TM_RY * TM_WW * E);
    static constexpr int WU = WAY + al(TM_AYH * TM_WW * E);
    static constexpr int WC = WU + al(TM_RY * TM_WW * E);
    static constexpr int SU = WC + al(TM_CH * TM_CWW * E);
    static constexpr int BYTES = SU + al(TmCfg::WORDS * E) + 128;  // + room to align the base
    // transaction bytes of one tile (the TMA counts whole boxes, filled parts included)
    static constexpr uint32_t MAIN_DOWN = (uint32_t)((2 * TM_RY * TM_RX + TM_RY * TM_AXW + TM_AYH * TM_RX) * E);
    static constexpr uint32_t MAIN_UP = MAIN_DOWN + (uint32_t)((TM_RY * TM_RX + TM_CH * TM_CW) * E);
    static constexpr uint32_t WRAP_DOWN = (uint32_t)((3 * TM_RY * TM_WW + TM_AYH * TM_WW) * E);
    static constexpr uint32_t WRAP_UP = WRAP_DOWN + (uint32_t)((TM_RY * TM_WW + TM_CH * TM_CWW) * E);
};

// Thread 0: the copies of one tile into the staging buffer, completing on bar.
template <typename T, bool UP>
__device__ __forceinline__ void tm_issue(const TmArgs<T>& A, unsigned char* sm, uint64_t* bar, int tile) {
    using S = TmStage<T>;
    const int tx = tile % A.ntx, ty = tile / A.ntx;
    const int gi0 = tx * TM_TS - TM_H, gj0 = ty * TM_TS - TM_H;
    const bool edge = (tx == 0 || tx == A.ntx - 1);
    const uint32_t bytes = (UP ? S::MAIN_UP : S::MAIN_DOWN) + (edge ? (UP ? S::WRAP_UP : S::WRAP_DOWN) : 0u);
    tc::mbar_expect_tx(bar, bytes);
    tc::tma_load_2d(sm + S::F, &A.m.f, bar, gi0, gj0);
    tc::tma_load_2d(sm + S::D, &A.m.d, bar, gi0, gj0);
    tc::tma_load_2d(sm + S::AX, &A.m.ax, bar, gi0, gj0);
    tc::tma_load_2d(sm + S::AY, &A.m.ay, bar, gi0, gj0);
    if (UP) {
        tc::tma_load_2d(sm + S::U, &A.m.u, bar, gi0, gj0);
        tc::tma_load_2d(sm + S::C, &A.m.c, bar, gi0 / 2 - 2, gj0 / 2);
    }
    if (edge) {
        const int wx = (tx == 0) ? A.nx - TM_WW : 0;
        tc::tma_load_2d(sm + S::WF, &A.m.fw, bar, wx, gj0);
        tc::tma_load_2d(sm + S::WD, &A.m.dw, bar, wx, gj0);
        tc::tma_load_2d(sm + S::WAX, &A.m.axw, bar, wx, gj0);
        tc::tma_load_2d(sm + S::WAY, &A.m.ayw, bar, wx, gj0);
        if (UP) {
            tc::tma_load_2d(sm + S::WU, &A.m.uw, bar, wx, gj0);
            tc::tma_load_2d(sm + S::WC, &A.m.cw, bar, (tx == 0) ? A.nx / 2 - TM_CWW : 0, gj0 / 2);
        }
    }
}

// The value of region row rr at global column i (region column x = i - gi0) of a staged
// array: the main box, or for a wrapped column the strip copied from the far end (at
// nx - 8 for the first tile column, at 0 for the last).
template <typename T>
__device__ __forceinline__ T tm_at(const T* __restrict__ box, int bw, const T* __restrict__ wrap, int rr, int x, int i,
                                   int nx) {
    if (i < 0) return wrap[rr * TM_WW + i + TM_WW];
    if (i >= nx) return wrap[rr * TM_WW + i - nx];
    return box[rr * bw + x];
}

// The thread's cells from the staged tile (rb_load's values).
template <typename T>
__device__ __forceinline__ void tm_load(RBCells<T, TmCfg::K>& cl, const RBGeom<TmCfg>& g,
                                        const unsigned char* __restrict__ sm, int nx, int ny, int gi0, int gj0) {
    using S = TmStage<T>;
    const T* sF = reinterpret_cast<const T*>(sm + S::F);
    const T* sD = reinterpret_cast<const T*>(sm + S::D);
    const T* sAX = reinterpret_cast<const T*>(sm + S::AX);
    const T* sAY = reinterpret_cast<const T*>(sm + S::AY);
    const T* wF = reinterpret_cast<const T*>(sm + S::WF);
    const T* wD = reinterpret_cast<const T*>(sm + S::WD);
    const T* wAX = reinterpret_cast<const T*>(sm + S::WAX);
    const T* wAY = reinterpret_cast<const T*>(sm + S::WAY);
    const int i = gi0 + g.x;
    cl.valid = 0u;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int k = 0; k < TmCfg::K; ++k) {
            const int rr = g.row(c, k);
            const int j = gj0 + rr;
            const bool ok = g.used && j >= 0 && j < ny;
            T vf = T(0), vd = T(0), vw = T(0), ve = T(0), vs = T(0), vn = T(0);
            if (ok) {
                vf = tm_at(sF, TM_RX, wF, rr, g.x, i, nx);
                vd = tm_at(sD, TM_RX, wD, rr, g.x, i, nx);
                vw = tm_at(sAX, TM_AXW, wAX, rr, g.x, i, nx);
                ve = tm_at(sAX, TM_AXW, wAX, rr, g.x + 1, i + 1, nx);
                vs = tm_at(sAY, TM_RX, wAY, rr, g.x, i, nx);
                vn = tm_at(sAY, TM_RX, wAY, rr + 1, g.x, i, nx);
            }
            cl.f[c][k] = vf;
            cl.di[c][k] = vd;
            cl.aw[c][k] = vw;
            cl.ae[c][k] = ve;
            cl.as[c][k] = vs;
            cl.an[c][k] = vn;
            cl.valid |= (ok ? 1u : 0u) << (c * TmCfg::K + k);
        }
    }
    cl.sweep = (g.x >= 1 && g.x < TmCfg::RX - 1) ? cl.valid : 0u;
}

// u_pre + P uc of the thread's cells (k_up's values; zero off the domain rows).
template <typename T>
__device__ __forceinline__ void tm_load_u(T (&uv)[2][TmCfg::K], const RBCells<T, TmCfg::K>& cl,
                                          const RBGeom<TmCfg>& g, const unsigned char* __restrict__ sm, int nx,
                                          int gi0) {
    using S = TmStage<T>;
    const T* sU = reinterpret_cast<const T*>(sm + S::U);
    const T* sC = reinterpret_cast<const T*>(sm + S::C);
    const T* wU = reinterpret_cast<const T*>(sm + S::WU);
    const T* wC = reinterpret_cast<const T*>(sm + S::WC);
    const int i = gi0 + g.x;
    // coarse column of the cell in its box: the main box starts 2 coarse cells left of
    // gi0 / 2; the wrapped strips at ncx - 4 (first tile column) or 0 (last)
    const int ncx = nx >> 1;
    const T* cbase;
    int cw, cc;
    if (i < 0) {
        cbase = wC;
        cw = TM_CWW;
        cc = ((i + nx) >> 1) - (ncx - TM_CWW);
    } else if (i >= nx) {
        cbase = wC;
        cw = TM_CWW;
        cc = (i - nx) >> 1;
    } else {
        cbase = sC;
        cw = TM_CW;
        cc = (g.x >> 1) + 2;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int k = 0; k < TmCfg::K; ++k) {
            T v = T(0);
            if (cl.valid & (1u << (c * TmCfg::K + k))) {
                const int rr = g.row(c, k);
                v = tm_at(sU, TM_RX, wU, rr, g.x, i, nx);
                v += cbase[(rr >> 1) * cw + cc];
            }
            uv[c][k] = v;
        }
    }
}

// UP = false: k_down (nu1 = 2 sweeps from zero, residual, restriction) on every tile.
// UP = true : k_up (prolongation + nu2 = 2 sweeps), at level 0 with the CG's r.z.
template <typename T, bool UP, bool LEVEL0>
__global__ void __launch_bounds__(TmCfg::NTH, 2) k_smooth_tma(const __grid_constant__ TmArgs<T> A) {
    using S = TmStage<T>;
    extern __shared__ __align__(16) unsigned char tm_smem_raw[];
    // TMA destinations on 128-byte boundaries (the launch adds 128 bytes of room)
    unsigned char* sm = tm_smem_raw + ((128u - (tc::smem_u32(tm_smem_raw) & 127u)) & 127u);
    __shared__ __align__(8) uint64_t bar;
    __shared__ double red[32];
    T* su = reinterpret_cast<T*>(sm + S::SU);
    const int ntiles = A.ntx * A.nty;
    const RBGeom<TmCfg> g;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) tm_issue<T, UP>(A, sm, &bar, blockIdx.x);
    uint32_t parity = 0u;
    double acc = 0.0;
    bool failed = false;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tx = tile % A.ntx, ty = tile / A.ntx;
        const int gi0 = tx * TM_TS - TM_H, gj0 = ty * TM_TS - TM_H;
        rb_zero<T, TmCfg>(su);
        const int ok = tc::mbar_wait(&bar, parity) ? 1 : 0;
        if (!__syncthreads_and(ok)) {
            failed = true;
            break;
        }
        parity ^= 1u;
        RBCells<T, TmCfg::K> cl;
        tm_load<T>(cl, g, sm, A.nx, A.ny, gi0, gj0);
        T uv[2][TmCfg::K];
        if (UP) tm_load_u<T>(uv, cl, g, sm, A.nx, gi0);
        __syncthreads();  // the staged tile is in registers and u is zero-filled
        if (threadIdx.x == 0 && tile + (int)gridDim.x < ntiles) tm_issue<T, UP>(A, sm, &bar, tile + gridDim.x);
        if (UP)
            acc += up_body<T, 2, TM_TS, TM_TS, 4, LEVEL0>(cl, g, uv, su, A.out, A.nx, tx * TM_TS, ty * TM_TS);
        else
            down_body<T, 2, TM_TS, TM_TS, 4>(cl, g, su, A.out, A.fc, A.nx, tx * TM_TS, ty * TM_TS);
        __syncthreads();  // u read back before the next tile's zero fill
    }
    if (failed) {
        if (threadIdx.x == 0) atomicExch(&A.st->kerr, 1);
        return;
    }
    if (LEVEL0) {
        const double b = block_sum(acc, red);
        double tot;
        if (grid_sum_last(b, A.partials, &A.st->cnt[0], &tot, red)) {
            A.st->beta = (A.st->it == 0) ? 0.0 : tot / A.st->rz;
            A.st->rz = tot;
        }
    }
}

}  // namespace mg
}  // namespace lica
