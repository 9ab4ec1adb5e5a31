// Multigrid-preconditioned CG for the variable-coefficient pressure Poisson equation on
// one B200 (sm_100a).  The reference's POISSON (1d.f:3492-3578) is a 1-D Thomas solve of
// AK p(k-1) + BK p(k) + CK p(k+1) = DIVGSUM with AK/CK built from the face values of
// 1/rho (DENF_ZI); this file solves the 2-D generalisation of that operator (x periodic
// as IPX=1, y the wall-normal direction with the reference's bottom Neumann / top
// p=0-on-the-face boundary) for the 2-D workloads.
//
// Design (HBM/L2-bound stencil work; no tensor cores):
//   * Grid kernels own a TX x TY tile plus a halo staged in shared memory and run every
//     red-black half-sweep of one visit to a level inside the tile (temporal blocking:
//     the halo shrinks by one ring per half-sweep), so a visit reads u, f, beta once.
//     No kernel writes an array it reads a halo of: k_up writes a separate post-smoothing
//     buffer and the CG vectors x, p ping-pong between two buffers by iteration parity.
//       k_down : nu1 sweeps from a zero iterate + residual + 2x2 restriction
//       k_up   : piecewise-constant prolongation + nu2 sweeps (black first), and at
//                level 0 the r.z partial of the CG update
//   * The levels below 64x64 run in one CTA with everything in shared memory
//     (k_cta): remaining outer levels, the coarsest outer level solved in FP64 by inner
//     V-cycles that end in a dense elimination; levels <= 8x8 run in warp 0 alone.
//   * CG vector updates are fused with the stencil they need (k_pupdate: p = z + beta p
//     and p.Ap; k_xupdate: x += alpha p and the true residual f - A x with its norm).
//     Grid-wide sums use a deterministic last-block reduction, which also computes the
//     CG scalars on the device, so the host never reads a scalar inside an iteration.
//   * Optional (LICA_MG_CROSS_LEVEL=1 at create): the grid levels between level 0 and the
//     single-CTA levels run as one cooperative launch per V-cycle leg (k_down_mid,
//     k_up_mid) with grid barriers between levels; bit-identical, but slower on a B200 than
//     one graph node per level, so it is off by default.
//   * With use_graph the whole solve is one CUDA graph: set-up kernels followed by a
//     conditional WHILE node whose body is one PCG iteration; the last block of
//     k_xupdate sets the loop condition.
//   * Every kernel follows the operation order of the oracle and the library is built
//     with -fmad=false, so a preconditioner application is bit-identical to the CPU
//     restatement in FP64 and in FP32; only the dot products differ (summation order).
#include "common.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

extern "C" void lica_count_launches(int64_t n);

namespace lica {
namespace mg {

constexpr int TX = 32;
constexpr int TY = 32;
constexpr int NT = 256;          // threads of a CG / set-up grid-kernel CTA
constexpr int NT_CTA = 512;      // threads of the single-CTA coarse kernel (fewer idle warps per barrier than 1024)
constexpr int kMaxLevels = 16;
constexpr int kSmallCells = 64;  // levels with <= this many cells run in warp 0 alone
constexpr int kMaxDense = 64;    // bottom-level unknowns solved by dense elimination
constexpr double kStallFactor = 1e3;  // a rise of the residual below this x tol ends the PCG (LICA_STALLED)

struct State {
    double fscale;  // ||f||_2 (1 if f = 0)
    double rel;     // ||f - A x||_2 / fscale
    double rz;      // r.z of the latest preconditioner application
    double alpha, beta;
    double tol;
    double sums[2];
    double rel_prev;  // rel of the previous iterate
    int it, max_it;
    int status;     // lica_status
    int cont;       // 1 while the loop should continue
    int back;       // 1: stalled, the answer is the iterate before the last one (it was decremented)
    int kerr;       // 1: a bounded wait inside a kernel ran out (the solve ends with LICA_ERR_CUDA)
    unsigned cnt[4];
    unsigned bar_count, bar_gen;  // grid barrier of the cross-level kernels
};

// ------------------------------------------------------------------------------------
// Coefficient arrays.  Every level stores its stencil weights pre-scaled, so no kernel
// branches on the boundary or multiplies by 1/h^2:
//   AX[j*nx+i] = cx * bx[j*nx+i]                 (west face of cell i; periodic)
//   AY[j*nx+i] = 0                      j = 0    (Neumann wall: FIXKL(1) = 1)
//              = cy * by[j*nx+i]        0 < j < ny
//              = (2*cy) * by[ny*nx+i]   j = ny   (p = 0 on the top face: VVDZ(N3) = 2/h)
// These are the same products the oracle forms at each use, so results stay identical.
// ------------------------------------------------------------------------------------
template <typename T>
struct V2;
template <>
struct V2<double> {
    using type = double2;
};
template <>
struct V2<float> {
    using type = float2;
};

__device__ __forceinline__ void async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ------------------------------------------------------------------------------------
// Register-blocked red-black smoothing kernels (k_down, k_up).
//
// A CTA owns a TXX x TYY tile of one level plus a halo of H = 2*nsw cells and runs every
// half-sweep of one visit inside that region (temporal blocking: the valid part shrinks
// by one ring per half-sweep and one more for the residual; k_down's first half-sweep
// starts from zero and needs no neighbour), so a visit reads f and the weights once.
//
// Thread t owns column x = t % RXP of the region (threads with x >= RX idle) and rows
// [s*R, s*R + R) of strip s = t / RXP.  Its cells are held in colour order: A[k] is the red cell of row pair k
// (row 2k + p with p = x & 1) and B[k] the black one (row 2k + 1 - p).  Their weights,
// f and 1/d stay in registers for the whole visit; only u goes through shared memory, so
// an update is four shared loads at fixed offsets, the oracle's nine FP64 operations and
// one shared store.
//
// Shared layout of u: word(s, r, x) = PAD + s*SSTR + r*RXP + x, RXP = 8 (mod 16) and
// SSTR = R*RXP + 8.  Lanes sit on consecutive x; in every access of a sweep (own cell,
// west, east, south, north, also across a strip boundary) the 16 lanes of a half-warp
// then touch 16 distinct 8-byte bank pairs.
// ------------------------------------------------------------------------------------
template <int NSW, int TXX, int TYY, int R>
struct RBCfg {
    static constexpr int H = 2 * NSW;
    static constexpr int RX = TXX + 2 * H;
    static constexpr int RXP = RX + ((8 - RX % 16) + 16) % 16;
    static constexpr int RY = ((TYY + 2 * H + R - 1) / R) * R;
    static constexpr int NS = RY / R;
    static constexpr int NUSED = RXP * NS;  // threads mapped over the padded pitch
    static constexpr int NTH = (NUSED + 31) / 32 * 32;
    static constexpr int SSTR = R * RXP + 8;
    static constexpr int PAD = RXP + 16;
    static constexpr int WORDS = PAD + NS * SSTR + RXP + 16;
    static constexpr int K = R / 2;
    static_assert(R % 2 == 0 && TXX % 16 == 0 && TYY % 2 == 0, "tile shape");
    static_assert(RXP % 16 == 8 && SSTR % 16 == 8, "bank layout");
};

// The cells of one thread: colour c (0 red = A, 1 black = B), pair k.
template <typename T, int K>
struct RBCells {
    T f[2][K], di[2][K], aw[2][K], ae[2][K], as[2][K], an[2][K];
    unsigned valid;  // bit c*K + k: the cell lies inside the domain (rows 0..ny-1)
    unsigned sweep;  // valid, and not in the region's edge columns x = 0, RX-1
};

template <class C>
struct RBGeom {
    int x, s, p;
    bool used;
    int base[2];  // word of A[0] and B[0]
    int soff[2];  // south offset of A[0], B[0] (a strip boundary adds the 8-word skew)
    int noff[2];  // north offset of A[K-1], B[K-1]
    __device__ __forceinline__ RBGeom() {
        const int t = threadIdx.x;
        s = t / C::RXP;
        x = t - s * C::RXP;
        used = t < C::NUSED && x < C::RX;
        if (!used) s = x = 0;
        p = x & 1;
        base[0] = C::PAD + s * C::SSTR + p * C::RXP + x;
        base[1] = C::PAD + s * C::SSTR + (1 - p) * C::RXP + x;
        soff[0] = -C::RXP - 8 * (1 - p);
        soff[1] = -C::RXP - 8 * p;
        noff[0] = C::RXP + 8 * p;
        noff[1] = C::RXP + 8 * (1 - p);
    }
    // region row of cell (c, k)
    __device__ __forceinline__ int row(int c, int k) const { return s * (C::K * 2) + 2 * k + (c ? 1 - p : p); }
};

// Loads f, 1/d and the four weights of the thread's cells (zero outside the domain rows).
// COH: f was written earlier in the same launch (the cross-level kernels), so it is read
// through L2 (ld.global.cg), never through the non-coherent read-only path.
template <typename T, class C, bool COH = false>
__device__ __forceinline__ void rb_load(RBCells<T, C::K>& cl, const RBGeom<C>& g, const T* __restrict__ f,
                                        const T* __restrict__ ax, const T* __restrict__ ay,
                                        const T* __restrict__ dinv, int nx, int ny, int gi0, int gj0) {
    int i = gi0 + g.x;
    if (i < 0) i += nx; else if (i >= nx) i -= nx;
    const int ip = (i + 1 == nx) ? 0 : i + 1;
    cl.valid = 0u;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int k = 0; k < C::K; ++k) {
            const int j = gj0 + g.row(c, k);
            const bool ok = g.used && j >= 0 && j < ny;
            T vf = T(0), vd = T(0), vw = T(0), ve = T(0), vs = T(0), vn = T(0);
            if (ok) {
                const int o = j * nx;
                vf = COH ? __ldcg(f + o + i) : f[o + i];
                vd = dinv[o + i];
                vw = ax[o + i];
                ve = ax[o + ip];
                vs = ay[o + i];
                vn = ay[o + nx + i];
            }
            cl.f[c][k] = vf;
            cl.di[c][k] = vd;
            cl.aw[c][k] = vw;
            cl.ae[c][k] = ve;
            cl.as[c][k] = vs;
            cl.an[c][k] = vn;
            cl.valid |= (ok ? 1u : 0u) << (c * C::K + k);
        }
    }
    // The west read of column 0 (east read of column RX-1) lands on the previous (next)
    // row's far column, a cell of the same colour: the edge columns, outside the valid
    // part after their first neighbour-dependent update, are never swept.
    cl.sweep = (g.x >= 1 && g.x < C::RX - 1) ? cl.valid : 0u;
}

// Stencil sum of cell (c, k) in the oracle's order: s = aw*uw + ae*ue + as*us + an*un.
template <typename T, class C>
__device__ __forceinline__ T rb_sum(const RBCells<T, C::K>& cl, const RBGeom<C>& g, const T* __restrict__ pc, int c,
                                    int k) {
    const T uw = pc[-1], ue = pc[1];
    const T us = (k == 0) ? pc[g.soff[c]] : pc[-C::RXP];
    const T un = (k == C::K - 1) ? pc[g.noff[c]] : pc[C::RXP];
    T ss = cl.aw[c][k] * uw;
    ss += cl.ae[c][k] * ue;
    ss += cl.as[c][k] * us;
    ss += cl.an[c][k] * un;
    return ss;
}

// One half-sweep of colour c over the thread's cells: u = (s - f) * (1/d).
template <typename T, class C, int c>
__device__ __forceinline__ void rb_half_sweep(const RBCells<T, C::K>& cl, const RBGeom<C>& g, T* __restrict__ su) {
#pragma unroll
    for (int k = 0; k < C::K; ++k) {
        if (cl.sweep & (1u << (c * C::K + k))) {
            T* pc = su + g.base[c] + 2 * k * C::RXP;
            const T ss = rb_sum<T, C>(cl, g, pc, c, k);
            pc[0] = (ss - cl.f[c][k]) * cl.di[c][k];
        }
    }
}

// The first red half-sweep from a zero iterate: every neighbour is zero and every weight
// is >= 0, so the oracle's sum is +0 and u = (0 - f) * (1/d) exactly, on every cell of
// the region (no neighbour read, so the edge columns are valid too).
template <typename T, class C>
__device__ __forceinline__ void rb_first_red(const RBCells<T, C::K>& cl, const RBGeom<C>& g, T* __restrict__ su) {
#pragma unroll
    for (int k = 0; k < C::K; ++k) {
        if (cl.valid & (1u << k)) su[g.base[0] + 2 * k * C::RXP] = (T(0) - cl.f[0][k]) * cl.di[0][k];
    }
}

// Residual f - (s - d*u) of cell (c, k), d = ((aw + ae) + as) + an as in the oracle.
template <typename T, class C>
__device__ __forceinline__ T rb_residual(const RBCells<T, C::K>& cl, const RBGeom<C>& g, const T* __restrict__ su,
                                         int c, int k, T& u) {
    const T* pc = su + g.base[c] + 2 * k * C::RXP;
    const T ss = rb_sum<T, C>(cl, g, pc, c, k);
    T d = cl.aw[c][k];
    d += cl.ae[c][k];
    d += cl.as[c][k];
    d += cl.an[c][k];
    u = pc[0];
    return cl.f[c][k] - (ss - d * u);
}

template <typename T, class C>
__device__ __forceinline__ void rb_zero(T* __restrict__ su) {
    for (int k = threadIdx.x; k < C::WORDS; k += C::NTH) su[k] = T(0);
}

// ------------------------------------------------------------------------------------
// k_down: nu1 red-black sweeps from a zero iterate, the residual and its 2x2 restriction
// (fc = (r00 + r10 + r01 + r11) / 4 in the oracle's order; the east partner of an even
// column is the neighbouring lane).
// ------------------------------------------------------------------------------------
// The part after the loads, for the tile whose first interior cell is (ti0, tj0); su is
// zero-filled and the thread's cells are loaded; every thread calls it.
template <typename T, int NSW, int TXX, int TYY, int R>
__device__ __forceinline__ void down_body(const RBCells<T, RBCfg<NSW, TXX, TYY, R>::K>& cl,
                                          const RBGeom<RBCfg<NSW, TXX, TYY, R>>& g, T* __restrict__ su,
                                          T* __restrict__ u_out, T* __restrict__ fc_out, int nx, int ti0, int tj0) {
    using C = RBCfg<NSW, TXX, TYY, R>;
    rb_first_red<T, C>(cl, g, su);
    __syncthreads();
    rb_half_sweep<T, C, 1>(cl, g, su);
    __syncthreads();
#pragma unroll 1
    for (int q = 1; q < NSW; ++q) {
        rb_half_sweep<T, C, 0>(cl, g, su);
        __syncthreads();
        rb_half_sweep<T, C, 1>(cl, g, su);
        __syncthreads();
    }
    const bool col_in = g.used && g.x >= C::H && g.x < C::H + TXX;
    const int ti = ti0 + g.x - C::H;
    const int ncx = nx >> 1;
#pragma unroll
    for (int k = 0; k < C::K; ++k) {
        T u0, u1;
        const T r0 = rb_residual<T, C>(cl, g, su, 0, k, u0);
        const T r1 = rb_residual<T, C>(cl, g, su, 1, k, u1);
        // rows of the pair: 2k + p (A) and 2k + 1 - p (B); useful rows are [H, H + TYY)
        const int y = g.s * R + 2 * k;
        const bool row_in = col_in && y >= C::H && y < C::H + TYY;
        if (row_in) {
            const int tj = tj0 + y - C::H;
            u_out[(tj + g.p) * nx + ti] = u0;
            u_out[(tj + 1 - g.p) * nx + ti] = u1;
        }
        // even column: A = row 2k, B = row 2k+1; its partner (odd column): A = row 2k+1, B = row 2k
        const T oA = __shfl_xor_sync(0xffffffffu, r0, 1);
        const T oB = __shfl_xor_sync(0xffffffffu, r1, 1);
        if (row_in && g.p == 0) {
            const T fcv = T(0.25) * ((r0 + oB) + (r1 + oA));
            fc_out[((tj0 + y - C::H) >> 1) * ncx + (ti >> 1)] = fcv;
        }
    }
}

template <typename T, int NSW, int TXX, int TYY, int R>
__global__ void __launch_bounds__(RBCfg<NSW, TXX, TYY, R>::NTH, 2)
    k_down(const T* __restrict__ f, const T* __restrict__ ax, const T* __restrict__ ay, const T* __restrict__ dinv,
           T* __restrict__ u_out, T* __restrict__ fc_out, int nx, int ny) {
    using C = RBCfg<NSW, TXX, TYY, R>;
    __shared__ __align__(16) T su[C::WORDS];
    const int gi0 = blockIdx.x * TXX - C::H, gj0 = blockIdx.y * TYY - C::H;
    const RBGeom<C> g;
    RBCells<T, C::K> cl;
    rb_zero<T, C>(su);
    rb_load<T, C>(cl, g, f, ax, ay, dinv, nx, ny, gi0, gj0);
    __syncthreads();  // zero fill done
    down_body<T, NSW, TXX, TYY, R>(cl, g, su, u_out, fc_out, nx, blockIdx.x * TXX, blockIdx.y * TYY);
}

// ------------------------------------------------------------------------------------
// k_up: u = u_pre + P uc (piecewise constant), nu2 sweeps black-then-red, written to
// u_post (out of place: no block reads a tile another block has updated); at level 0
// also the r.z partial (r = f of level 0, z = u) and, in the last block, beta.
// ------------------------------------------------------------------------------------
// The part after the loads: uv holds u_pre + P uc of the thread's cells (0 off the
// domain), su is zero-filled; returns the tile's r.z partial (LEVEL0) or 0.
template <typename T, int NSW, int TXX, int TYY, int R, bool LEVEL0>
__device__ __forceinline__ double up_body(const RBCells<T, RBCfg<NSW, TXX, TYY, R>::K>& cl,
                                          const RBGeom<RBCfg<NSW, TXX, TYY, R>>& g,
                                          const T (&uv)[2][RBCfg<NSW, TXX, TYY, R>::K], T* __restrict__ su,
                                          T* __restrict__ u_post, int nx, int ti0, int tj0) {
    using C = RBCfg<NSW, TXX, TYY, R>;
    if (g.used) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
            for (int k = 0; k < C::K; ++k) su[g.base[c] + 2 * k * C::RXP] = uv[c][k];
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int q = 0; q < NSW; ++q) {
        rb_half_sweep<T, C, 1>(cl, g, su);
        __syncthreads();
        rb_half_sweep<T, C, 0>(cl, g, su);
        __syncthreads();
    }
    const bool col_in = g.used && g.x >= C::H && g.x < C::H + TXX;
    const int ti = ti0 + g.x - C::H;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < C::K; ++k) {
        const int y = g.s * R + 2 * k;
        if (col_in && y >= C::H && y < C::H + TYY) {
            const int tj = tj0 + y - C::H;
            const T u0 = su[g.base[0] + 2 * k * C::RXP];
            const T u1 = su[g.base[1] + 2 * k * C::RXP];
            u_post[(tj + g.p) * nx + ti] = u0;
            u_post[(tj + 1 - g.p) * nx + ti] = u1;
            if (LEVEL0) {
                acc += double(cl.f[0][k]) * double(u0);
                acc += double(cl.f[1][k]) * double(u1);
            }
        }
    }
    return acc;
}

template <typename T, int NSW, int TXX, int TYY, int R, bool LEVEL0>
__global__ void __launch_bounds__(RBCfg<NSW, TXX, TYY, R>::NTH, std::is_same<T, float>::value ? 3 : 2)
    k_up(const T* __restrict__ u_pre, T* __restrict__ u_post, const T* __restrict__ uc, const T* __restrict__ f,
         const T* __restrict__ ax, const T* __restrict__ ay, const T* __restrict__ dinv, int nx, int ny,
         State* __restrict__ st, double* __restrict__ partials) {
    using C = RBCfg<NSW, TXX, TYY, R>;
    __shared__ __align__(16) T su[C::WORDS];
    __shared__ double red[32];
    const int gi0 = blockIdx.x * TXX - C::H, gj0 = blockIdx.y * TYY - C::H;
    const int ncx = nx >> 1;
    const RBGeom<C> g;
    RBCells<T, C::K> cl;
    rb_zero<T, C>(su);
    rb_load<T, C>(cl, g, f, ax, ay, dinv, nx, ny, gi0, gj0);
    T uv[2][C::K];
    {
        int i = gi0 + g.x;
        if (i < 0) i += nx; else if (i >= nx) i -= nx;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
            for (int k = 0; k < C::K; ++k) {
                T v = T(0);
                if (cl.valid & (1u << (c * C::K + k))) {
                    const int j = gj0 + g.row(c, k);
                    v = u_pre[j * nx + i];
                    v += uc[(j >> 1) * ncx + (i >> 1)];
                }
                uv[c][k] = v;
            }
        }
    }
    __syncthreads();  // zero fill done
    const double acc =
        up_body<T, NSW, TXX, TYY, R, LEVEL0>(cl, g, uv, su, u_post, nx, blockIdx.x * TXX, blockIdx.y * TYY);
    if (LEVEL0) {
        const double b = block_sum(acc, red);
        double tot;
        if (grid_sum_last(b, partials, &st->cnt[0], &tot, red)) {
            st->beta = (st->it == 0) ? 0.0 : tot / st->rz;
            st->rz = tot;
        }
    }
}

// ------------------------------------------------------------------------------------
// Cross-level kernels: the grid levels below level 0 (1 .. lcta-1) of one V-cycle leg in one
// cooperative launch.  k_down_mid runs k_down's tile work level after level and k_up_mid
// k_up's (LEVEL0 = false) from the coarsest grid level up to level 1, each block looping
// over the tiles of a level, with a grid barrier between levels in place of a kernel
// boundary.  Arrays written earlier in the launch (a level's restricted residual, the
// coarser level's correction) are read through L2.  Same arithmetic as the per-level
// kernels, so the results are identical.
// ------------------------------------------------------------------------------------
constexpr int RB_TILE_R = 4;  // rows per thread strip of the smoothing tiles

struct MidLevel {
    int nx, ny, big;  // big: 32 x 32 tiles (else 16 x 16)
    const void *f, *ax, *ay, *di, *upre, *uc;
    void *u, *fc, *up;
};

struct MidParams {
    int l0, l1;  // levels l0 .. l1-1
    State* st;
    MidLevel lv[kMaxLevels];
};

constexpr unsigned kBarSpin = 1u << 21;  // bounded wait of a grid barrier (about 0.3 s)

// Grid barrier over all blocks of a cooperative launch; a wait that runs out sets st->kerr
// and lets the block go on (the solve then reports LICA_ERR_CUDA).
__device__ __forceinline__ void grid_barrier(State* __restrict__ st) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &st->bar_gen;
        const unsigned g0 = *vgen;
        __threadfence();
        const unsigned nb = gridDim.x * gridDim.y;
        if (atomicAdd(&st->bar_count, 1u) == nb - 1u) {
            atomicExch(&st->bar_count, 0u);
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else {
            unsigned it = 0;
            while (*vgen == g0) {
                if (++it > kBarSpin) {
                    atomicExch(&st->kerr, 1);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <typename T, int NSW, int TS>
__device__ __forceinline__ void mid_down_level(const MidLevel& L, T* __restrict__ su) {
    using C = RBCfg<NSW, TS, TS, RB_TILE_R>;
    const int ntx = L.nx / TS, nt = ntx * (L.ny / TS);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int bi = t % ntx, bj = t / ntx;
        const RBGeom<C> g;
        RBCells<T, C::K> cl;
        for (int k = threadIdx.x; k < C::WORDS; k += blockDim.x) su[k] = T(0);
        rb_load<T, C, true>(cl, g, (const T*)L.f, (const T*)L.ax, (const T*)L.ay, (const T*)L.di, L.nx, L.ny,
                            bi * TS - C::H, bj * TS - C::H);
        __syncthreads();
        down_body<T, NSW, TS, TS, RB_TILE_R>(cl, g, su, (T*)L.u, (T*)L.fc, L.nx, bi * TS, bj * TS);
        __syncthreads();  // su is reused by the next tile
    }
}

template <typename T, int NSW, int TS>
__device__ __forceinline__ void mid_up_level(const MidLevel& L, T* __restrict__ su) {
    using C = RBCfg<NSW, TS, TS, RB_TILE_R>;
    const int ntx = L.nx / TS, nt = ntx * (L.ny / TS), nx = L.nx, ncx = L.nx >> 1;
    const T* upre = (const T*)L.upre;
    const T* uc = (const T*)L.uc;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int bi = t % ntx, bj = t / ntx;
        const int gi0 = bi * TS - C::H, gj0 = bj * TS - C::H;
        const RBGeom<C> g;
        RBCells<T, C::K> cl;
        for (int k = threadIdx.x; k < C::WORDS; k += blockDim.x) su[k] = T(0);
        rb_load<T, C>(cl, g, (const T*)L.f, (const T*)L.ax, (const T*)L.ay, (const T*)L.di, L.nx, L.ny, gi0, gj0);
        T uv[2][C::K];
        int i = gi0 + g.x;
        if (i < 0) i += nx; else if (i >= nx) i -= nx;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
            for (int k = 0; k < C::K; ++k) {
                T v = T(0);
                if (cl.valid & (1u << (c * C::K + k))) {
                    const int j = gj0 + g.row(c, k);
                    v = upre[j * nx + i];
                    v += __ldcg(uc + (j >> 1) * ncx + (i >> 1));
                }
                uv[c][k] = v;
            }
        }
        __syncthreads();  // zero fill done
        up_body<T, NSW, TS, TS, RB_TILE_R, false>(cl, g, uv, su, (T*)L.up, L.nx, bi * TS, bj * TS);
        __syncthreads();
    }
}

template <typename T, int NSW>
__global__ void __launch_bounds__(RBCfg<NSW, 32, 32, RB_TILE_R>::NTH, 2) k_down_mid(const __grid_constant__ MidParams P) {
    __shared__ __align__(16) T su[RBCfg<NSW, 32, 32, RB_TILE_R>::WORDS];
    for (int l = P.l0; l < P.l1; ++l) {
        if (P.lv[l].big) mid_down_level<T, NSW, 32>(P.lv[l], su);
        else mid_down_level<T, NSW, 16>(P.lv[l], su);
        if (l + 1 < P.l1) grid_barrier(P.st);
    }
}

template <typename T, int NSW>
__global__ void __launch_bounds__(RBCfg<NSW, 32, 32, RB_TILE_R>::NTH, 2) k_up_mid(const __grid_constant__ MidParams P) {
    __shared__ __align__(16) T su[RBCfg<NSW, 32, 32, RB_TILE_R>::WORDS];
    for (int l = P.l1 - 1; l >= P.l0; --l) {
        if (P.lv[l].big) mid_up_level<T, NSW, 32>(P.lv[l], su);
        else mid_up_level<T, NSW, 16>(P.lv[l], su);
        if (l > P.l0) grid_barrier(P.st);
    }
}

// ------------------------------------------------------------------------------------
// CG kernels (FP64 vectors) on TX x TY tiles with a 2-cell halo (one ring is used; the
// second keeps every row segment an aligned vector load).
// ------------------------------------------------------------------------------------
constexpr int PH = 2, PRX = TX + 2 * PH, PRY = TY + 2 * PH;

// Issues the copies of a (PRY x PRX) region of a row-major array into s (x periodic,
// rows outside [0, nrows) zero), one pair of cells (8 or 16 bytes) per copy.
// Completion: async_wait_all + barrier.
template <typename TG>
__device__ __forceinline__ void load_plain(TG* __restrict__ s, const TG* __restrict__ g, int nx, int nrows, int gi0,
                                           int gj0) {
    for (int k = threadIdx.x; k < PRY * (PRX / 2); k += blockDim.x) {
        const int sy = k / (PRX / 2), m = k - sy * (PRX / 2);
        const int j = gj0 + sy;
        int i = gi0 + 2 * m;
        if (i < 0) i += nx; else if (i >= nx) i -= nx;
        const bool ok = (j >= 0 && j < nrows);
        const TG* src = ok ? g + (size_t)j * nx + i : g;
        const unsigned d = (unsigned)__cvta_generic_to_shared(s + sy * PRX + 2 * m);
        if (sizeof(TG) == 8) {
            const int n = ok ? 16 : 0;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
        } else {
            const int n = ok ? 8 : 0;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
        }
    }
}

__device__ __forceinline__ void plain_sums(const double* su, const double* sax, const double* say, int sx, int sy,
                                           double& s, double& d) {
    const int c = sy * PRX + sx;
    const double aw = sax[c], ae = sax[c + 1], as = say[c], an = say[c + PRX];
    double ss = aw * su[c - 1];
    ss += ae * su[c + 1];
    ss += as * su[c - PRX];
    ss += an * su[c + PRX];
    double dd = aw;
    dd += ae;
    dd += as;
    dd += an;
    s = ss;
    d = dd;
}

constexpr int PAREA = PRX * PRY;

// p_new = z + beta*p_old on the tile and a ring, then p_new.(A p_new) over the tile; the
// last block sets alpha = rz / p.Ap.  p ping-pongs between two buffers chosen on the
// device by the iteration parity (p_old = pp[it&1], p_new = pp[(it+1)&1]), so the halo is
// always read from a buffer no block of this launch writes.
template <typename TZ>
__global__ void __launch_bounds__(NT) k_pupdate(double* __restrict__ p0, double* __restrict__ p1,
                                                const TZ* __restrict__ z, const double* __restrict__ ax,
                                                const double* __restrict__ ay, int nx, int ny,
                                                State* __restrict__ st, double* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sp = reinterpret_cast<double*>(smem_raw);
    double* sax = sp + PAREA;
    double* say = sax + PAREA;
    TZ* sz = reinterpret_cast<TZ*>(say + PAREA);
    __shared__ double red[32];
    const int gi0 = blockIdx.x * TX - PH, gj0 = blockIdx.y * TY - PH;
    const int par = st->it & 1;
    const double* __restrict__ p = par ? p1 : p0;
    double* __restrict__ pn = par ? p0 : p1;
    load_plain(sp, p, nx, ny, gi0, gj0);
    load_plain(sz, z, nx, ny, gi0, gj0);
    load_plain(sax, ax, nx, ny, gi0, gj0);
    load_plain(say, ay, nx, ny + 1, gi0, gj0);
    const double beta = st->beta;
    async_wait_all();
    __syncthreads();
    for (int k = threadIdx.x; k < PAREA; k += blockDim.x) sp[k] = double(sz[k]) + beta * sp[k];
    __syncthreads();
    double acc = 0.0;
    for (int k = threadIdx.x; k < TX * TY; k += blockDim.x) {
        const int ty = k / TX, tx = k - ty * TX;
        const int sx = tx + PH, sy = ty + PH;
        double s, d;
        plain_sums(sp, sax, say, sx, sy, s, d);
        const double pv = sp[sy * PRX + sx];
        const double q = s - d * pv;
        acc += pv * q;
        pn[(size_t)(blockIdx.y * TY + ty) * nx + blockIdx.x * TX + tx] = pv;
    }
    const double b = block_sum(acc, red);
    double tot;
    if (grid_sum_last(b, partials, &st->cnt[1], &tot, red)) st->alpha = st->rz / tot;
}

// x_new = x_old + alpha*p on the tile and a ring, r = f - A x_new over the tile (FP64),
// stored as TR; the last block forms rel = ||r||/||f||, advances the iteration count and
// sets the loop condition.  x ping-pongs like p: x_old = xx[it&1], x_new = xx[(it+1)&1]
// (xx[0] is the caller's array); p is the buffer k_pupdate just wrote, pp[(it+1)&1].
// first = 1: the set-up pass, r = f - A x0 and ||f||, nothing written to x.
__device__ __noinline__ void xupdate_finish(State* __restrict__ st, double tot, int first,
                                            cudaGraphConditionalHandle cond, int use_cond);

template <typename TR>
__global__ void __launch_bounds__(NT) k_xupdate(double* __restrict__ x0, double* __restrict__ x1,
                                                const double* __restrict__ p0, const double* __restrict__ p1,
                                                const double* __restrict__ f, const double* __restrict__ ax,
                                                const double* __restrict__ ay, TR* __restrict__ r_out, int nx, int ny,
                                                State* __restrict__ st, double* __restrict__ partials, int first,
                                                cudaGraphConditionalHandle cond, int use_cond) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sxv = reinterpret_cast<double*>(smem_raw);
    double* spv = sxv + PAREA;
    double* sax = spv + PAREA;
    double* say = sax + PAREA;
    double* sf = say + PAREA;
    __shared__ double red[32];
    const int gi0 = blockIdx.x * TX - PH, gj0 = blockIdx.y * TY - PH;
    const int par = first ? 0 : (st->it & 1);
    const double* __restrict__ x = par ? x1 : x0;
    double* __restrict__ xn = par ? x0 : x1;
    const double* __restrict__ p = par ? p0 : p1;
    load_plain(sxv, x, nx, ny, gi0, gj0);
    if (!first) load_plain(spv, p, nx, ny, gi0, gj0);
    load_plain(sax, ax, nx, ny, gi0, gj0);
    load_plain(say, ay, nx, ny + 1, gi0, gj0);
    load_plain(sf, f, nx, ny, gi0, gj0);
    const double alpha = first ? 0.0 : st->alpha;
    async_wait_all();
    __syncthreads();
    if (!first) {
        for (int k = threadIdx.x; k < PAREA; k += blockDim.x) sxv[k] = sxv[k] + alpha * spv[k];
        __syncthreads();
    }
    double acc = 0.0, accf = 0.0;
    for (int k = threadIdx.x; k < TX * TY; k += blockDim.x) {
        const int ty = k / TX, tx = k - ty * TX;
        const int sx = tx + PH, sy = ty + PH;
        const size_t g = (size_t)(blockIdx.y * TY + ty) * nx + blockIdx.x * TX + tx;
        double s, d;
        plain_sums(sxv, sax, say, sx, sy, s, d);
        const double xv = sxv[sy * PRX + sx];
        const double fv = sf[sy * PRX + sx];
        const double r = fv - (s - d * xv);
        acc += r * r;
        if (first) accf += fv * fv;
        if (!first) xn[g] = xv;
        r_out[g] = TR(r);
    }
    const double b = block_sum(acc, red);
    const double bf = first ? block_sum(accf, red) : 0.0;
    double tot;
    // first launch: two sums (||f||^2 through counter 3, then ||r||^2 through counter 2)
    if (first) {
        if (grid_sum_last(bf, partials + gridDim.x * gridDim.y, &st->cnt[3], &tot, red)) st->sums[1] = tot;
    }
    if (grid_sum_last(b, partials, &st->cnt[2], &tot, red)) xupdate_finish(st, tot, first, cond, use_cond);
}

// The last block of k_xupdate: ||f|| on the set-up pass, the iteration count, rel, the
// status and the loop condition.
__device__ __noinline__ void xupdate_finish(State* __restrict__ st, double tot, int first,
                                            cudaGraphConditionalHandle cond, int use_cond) {
    {
        __threadfence();
        if (first) {
            // the ||f|| sum finished in an earlier (or this) block: read it through L2
            const double ff = *((volatile double*)&st->sums[1]);
            const double fn = sqrt(ff);
            st->fscale = (fn > 0.0) ? fn : 1.0;
            st->it = 0;
        } else {
            st->it = st->it + 1;
        }
        const double rel = sqrt(tot) / st->fscale;
        st->rel = rel;
        int cont = 0;
        if (st->kerr) {
            st->status = LICA_ERR_CUDA;
        } else if (!isfinite(rel)) {
            st->status = LICA_NAN;
        } else if (rel <= st->tol) {
            st->status = LICA_OK;
        } else if (!first && rel >= st->rel_prev && st->rel_prev <= kStallFactor * st->tol) {
            // the true residual rose near the tolerance: FP64's attainable accuracy is
            // reached (past it the search directions lose conjugacy and the iteration
            // diverges).  The previous iterate is in the other x buffer: report it.
            st->status = LICA_STALLED;
            st->it = st->it - 1;
            st->back = 1;
            st->rel = st->rel_prev;
        } else if (st->it >= st->max_it) {
            st->status = LICA_NOT_CONVERGED;
        } else {
            cont = 1;
        }
        st->rel_prev = rel;
        st->cont = cont;
        if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
    }
}

}  // namespace mg
}  // namespace lica

#include "mg_cg_tma.cuh"

namespace lica {
namespace mg {

template <typename TZ>
constexpr size_t pupdate_smem() {
    return sizeof(double) * 3 * PAREA + sizeof(TZ) * PAREA;
}
constexpr size_t xupdate_smem() { return sizeof(double) * 5 * PAREA; }

// ------------------------------------------------------------------------------------
// Single-CTA coarse part: outer levels [lcta, lc) in T, the coarsest outer level lc and
// the inner levels in FP64, all in shared memory.
//
// Every level is stored colour-split: cell (i, j) of colour c = (i + j) & 1 sits in X_c at
// [j * half + (i >> 1)], half = nx / 2, for X = u, f, ax (west faces), ay (south faces,
// rows 0..ny) and 1/d.  A red (black) half-sweep then reads and writes consecutive words
// across a warp, and the four children of coarse cell (I, J) are the entries I of rows
// 2J and 2J+1 of both colours.  u has a zero ghost row below row 0 and above row ny-1,
// so the wall neighbours need no branch.  Work items are walked with an incremental
// (row, column) pair: no division per cell.
// ------------------------------------------------------------------------------------
struct CtaLevel {
    int nx, ny, half;
    unsigned mag_h, mag_nx;  // division multipliers for half and nx (t / c = umulhi(t, mag), c > 1)
    unsigned off_u[2], off_f[2], off_ax[2], off_ay[2], off_di[2];  // byte offsets into dynamic smem
    const void* gax;                                                // AX, AY, DINV of this level (T or double)
    const void* gay;
    const void* gdi;
};

struct CtaParams {
    int lcta, lc, bottom;
    int nu1, nu2, ncoarse;
    unsigned off_dense, off_rhs;
    const double* glu; // bottom-level elimination (multipliers below, U on and above the diagonal)
    const void* f_in;  // f of level lcta (T)
    void* u_out;       // u of level lcta (T)
    CtaLevel lv[kMaxLevels];
};

template <typename E>
struct SL {
    E* u[2];  // row 0 of each colour; rows -1 and ny are zero ghosts
    E* f[2];
    E* ax[2];
    E* ay[2];
    E* di[2];
    int nx, ny, h;
    unsigned mag_h, mag_nx;
};

template <typename E>
__device__ __forceinline__ SL<E> make_sl(const CtaParams& P, unsigned char* sm, int l) {
    const CtaLevel& L = P.lv[l];
    SL<E> s;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        s.u[c] = reinterpret_cast<E*>(sm + L.off_u[c]) + L.half;
        s.f[c] = reinterpret_cast<E*>(sm + L.off_f[c]);
        s.ax[c] = reinterpret_cast<E*>(sm + L.off_ax[c]);
        s.ay[c] = reinterpret_cast<E*>(sm + L.off_ay[c]);
        s.di[c] = reinterpret_cast<E*>(sm + L.off_di[c]);
    }
    s.nx = L.nx;
    s.ny = L.ny;
    s.h = L.half;
    s.mag_h = L.mag_h;
    s.mag_nx = L.mag_nx;
    return s;
}

template <bool W>
__device__ __forceinline__ int g_tid() { return W ? (int)(threadIdx.x & 31) : (int)threadIdx.x; }
template <bool W>
__device__ __forceinline__ constexpr int g_nthr() { return W ? 32 : NT_CTA; }
template <bool W>
__device__ __forceinline__ void g_sync() {
    if (W) __syncwarp(); else __syncthreads();
}

// Items it = t, t + G, ... of a (rows x cols) range as an incremental (row, col) pair.
__device__ __forceinline__ int div_mag(int t, int cols, unsigned mag) {
    return cols == 1 ? t : (int)__umulhi((unsigned)t, mag);
}
struct ItemWalk {
    int r, q, dr, dq, cols;
    __device__ __forceinline__ ItemWalk(int t, int G, int cols_, unsigned mag) : cols(cols_) {
        r = div_mag(t, cols, mag);
        q = t - r * cols;
        dr = div_mag(G, cols, mag);
        dq = G - dr * cols;
    }
    __device__ __forceinline__ void next() {
        r += dr;
        q += dq;
        if (q >= cols) { q -= cols; ++r; }
    }
};

// X[c] for a colour c known only at run time, without indexing the pointer pair.
template <typename P2>
__device__ __forceinline__ auto pick(const P2& x, int c) -> decltype(x[0]) { return c ? x[1] : x[0]; }

// The arrays one colour's update touches, selected once (no dynamic indexing of the
// per-colour pointer pairs, which would put them in local memory).
template <typename E>
struct Colour {
    E* uc;
    const E *uo, *axc, *axo, *ayc, *ayo, *fc, *dc;
    int c, h;
    __device__ __forceinline__ Colour(const SL<E>& L, int c_) : c(c_), h(L.h) {
        const bool b = c_ != 0;
        uc = b ? L.u[1] : L.u[0];
        uo = b ? L.u[0] : L.u[1];
        axc = b ? L.ax[1] : L.ax[0];
        axo = b ? L.ax[0] : L.ax[1];
        ayc = b ? L.ay[1] : L.ay[0];
        ayo = b ? L.ay[0] : L.ay[1];
        fc = b ? L.f[1] : L.f[0];
        dc = b ? L.di[1] : L.di[0];
    }
};

// Stencil sums of the colour-c cell (i = 2m + o, j), o = (j + c) & 1, in the oracle's
// order: s = aw*uw + ae*ue + as*us + an*un and d = aw + ae + as + an.  k is its index.
template <typename E>
__device__ __forceinline__ void split_sums(const Colour<E>& V, int j, int m, int k, E& s, E& d) {
    const int h = V.h, o = (j + V.c) & 1;
    int w = m - 1 + o, e = m + o;
    if (w < 0) w += h;
    if (e >= h) e -= h;
    const E aw = V.axc[k], ae = V.axo[j * h + e], as = V.ayc[k], an = V.ayo[k + h];
    const E uw = V.uo[j * h + w], ue = V.uo[j * h + e], us = V.uo[k - h], un = V.uo[k + h];
    E ss = aw * uw;
    ss += ae * ue;
    ss += as * us;
    ss += an * un;
    E dd = aw;
    dd += ae;
    dd += as;
    dd += an;
    s = ss;
    d = dd;
}

template <typename E, bool W>
__device__ void s_sweeps(const SL<E>& L, int nsw, bool reverse) {
    const int items = L.ny * L.h;
    for (int q = 0; q < 2 * nsw; ++q) {
        const Colour<E> V(L, reverse ? 1 - (q & 1) : (q & 1));
        ItemWalk wk(g_tid<W>(), g_nthr<W>(), L.h, L.mag_h);
#pragma unroll 2
        for (int it = g_tid<W>(); it < items; it += g_nthr<W>()) {
            const int k = wk.r * L.h + wk.q;
            E s, d;
            split_sums(V, wk.r, wk.q, k, s, d);
            V.uc[k] = (s - V.fc[k]) * V.dc[k];
            wk.next();
        }
        g_sync<W>();
    }
}

// Residual of the colour-c cell at (j, m), index k: f - (s - d*u).
template <typename E>
__device__ __forceinline__ E split_res(const Colour<E>& V, int j, int m) {
    const int k = j * V.h + m;
    E s, d;
    split_sums(V, j, m, k, s, d);
    return V.fc[k] - (s - d * V.uc[k]);
}

// fc(I, J) = 0.25*((r00 + r10) + (r01 + r11)) of the residual, and uc = 0.
template <typename E, typename EC, bool W>
__device__ void s_restrict(const SL<E>& F, const SL<EC>& C) {
    const int items = C.nx * C.ny;
    const Colour<E> R(F, 0), B(F, 1);
    ItemWalk wk(g_tid<W>(), g_nthr<W>(), C.nx, C.mag_nx);
#pragma unroll 2
    for (int it = g_tid<W>(); it < items; it += g_nthr<W>()) {
        const int J = wk.r, I = wk.q;
        const E r00 = split_res(R, 2 * J, I);
        const E r10 = split_res(B, 2 * J, I);
        const E r01 = split_res(B, 2 * J + 1, I);
        const E r11 = split_res(R, 2 * J + 1, I);
        const E fc = E(0.25) * ((r00 + r10) + (r01 + r11));
        const int cc = (I + J) & 1, kc = J * C.h + (I >> 1);
        pick(C.f, cc)[kc] = EC(fc);
        pick(C.u, cc)[kc] = EC(0);
        wk.next();
    }
    g_sync<W>();
}

// u += P uc (piecewise constant): the four children of coarse cell (I, J).
template <typename E, typename EC, bool W>
__device__ void s_prolong(const SL<EC>& C, const SL<E>& F) {
    const int items = C.nx * C.ny;
    ItemWalk wk(g_tid<W>(), g_nthr<W>(), C.nx, C.mag_nx);
#pragma unroll 2
    for (int it = g_tid<W>(); it < items; it += g_nthr<W>()) {
        const int J = wk.r, I = wk.q;
        const E e = E(pick(C.u, (I + J) & 1)[J * C.h + (I >> 1)]);
        const int k0 = 2 * J * F.h + I, k1 = k0 + F.h;
        F.u[0][k0] += e;
        F.u[1][k0] += e;
        F.u[0][k1] += e;
        F.u[1][k1] += e;
        wk.next();
    }
    g_sync<W>();
}

// Plain-index accessors of a colour-split level (the dense solve's assembly).
template <typename E>
__device__ __forceinline__ int split_index(const SL<E>& L, int i, int j) { return j * L.h + (i >> 1); }

// Dense solve of the bottom level, unknown row = j*nx + i, with the elimination of the
// matrix done once per solve (k_dense_factor): the oracle's b[i] -= m*b[k] in its order,
// then its back substitution s = b[i] - sum_j U[i][j] u[j] (j ascending), u[i] = s / U[i][i].
template <bool W>
__device__ void s_dense(const SL<double>& L, const double* A, double* b) {
    const int nx = L.nx, n = nx * L.ny;
    for (int k = g_tid<W>(); k < n; k += g_nthr<W>()) {
        const int j = k / nx, i = k - j * nx;
        b[k] = pick(L.f, (i + j) & 1)[split_index(L, i, j)];
    }
    g_sync<W>();
    for (int k = 0; k + 1 < n; ++k) {
        const double bk = b[k];
        for (int i = k + 1 + g_tid<W>(); i < n; i += g_nthr<W>()) b[i] -= A[i * n + k] * bk;
        g_sync<W>();
    }
    if (g_tid<W>() == 0) {
        for (int i = n - 1; i >= 0; --i) {
            double s = b[i];
            for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * b[j];
            b[i] = s / A[i * n + i];
        }
    }
    g_sync<W>();
    for (int k = g_tid<W>(); k < n; k += g_nthr<W>()) {
        const int j = k / nx, i = k - j * nx;
        pick(L.u, (i + j) & 1)[split_index(L, i, j)] = b[k];
    }
    g_sync<W>();
}

// First level in [l0, bottom] small enough for warp 0 alone.
__device__ __forceinline__ int first_small(const CtaParams& P, int l0) {
    int l = l0;
    while (l < P.bottom && P.lv[l].nx * P.lv[l].ny > kSmallCells) ++l;
    return l;
}

// Down-and-up over FP64 levels [la, lb] by group W: sweeps + restriction going down to
// lb (dense solve there when lb is the bottom) and prolongation + sweeps coming back.
template <bool W>
__device__ void s_inner_range_down(const CtaParams& P, unsigned char* sm, int la, int lb) {
    for (int l = la; l < lb; ++l) {
        const SL<double> L = make_sl<double>(P, sm, l);
        const SL<double> C = make_sl<double>(P, sm, l + 1);
        s_sweeps<double, W>(L, P.nu1, false);
        s_restrict<double, double, W>(L, C);
    }
}
template <bool W>
__device__ void s_inner_range_up(const CtaParams& P, unsigned char* sm, int la, int lb) {
    for (int l = lb - 1; l >= la; --l) {
        const SL<double> L = make_sl<double>(P, sm, l);
        const SL<double> C = make_sl<double>(P, sm, l + 1);
        s_prolong<double, double, W>(C, L);
        s_sweeps<double, W>(L, P.nu2, true);
    }
}

// One inner V-cycle on the FP64 levels [l0, bottom] starting from the iterate in u(l0).
// Levels above the first small level run block-wide, the rest in warp 0.
__device__ void s_vcycle_inner(const CtaParams& P, unsigned char* sm, int l0) {
    double* A = reinterpret_cast<double*>(sm + P.off_dense);
    double* b = reinterpret_cast<double*>(sm + P.off_rhs);
    const int ls = first_small(P, l0);
    s_inner_range_down<false>(P, sm, l0, ls);
    if (threadIdx.x < 32) {
        s_inner_range_down<true>(P, sm, ls, P.bottom);
        s_dense<true>(make_sl<double>(P, sm, P.bottom), A, b);
        s_inner_range_up<true>(P, sm, ls, P.bottom);
    }
    __syncthreads();
    s_inner_range_up<false>(P, sm, l0, ls);
}

// Levels [lcta, lc) in T, then the coarsest outer level lc (FP64): ncoarse inner
// V-cycles from a zero iterate, or the dense solve when lc is the bottom level.
template <typename T>
__device__ void s_outer(const CtaParams& P, unsigned char* sm) {
    for (int l = P.lcta; l < P.lc; ++l) {
        const SL<T> L = make_sl<T>(P, sm, l);
        s_sweeps<T, false>(L, P.nu1, false);
        if (l + 1 == P.lc) s_restrict<T, double, false>(L, make_sl<double>(P, sm, l + 1));
        else s_restrict<T, T, false>(L, make_sl<T>(P, sm, l + 1));
    }
    {
        const SL<double> L = make_sl<double>(P, sm, P.lc);
        if (P.lcta == P.lc) {  // no restriction wrote u(lc)
            for (int k = threadIdx.x; k < L.ny * L.h; k += NT_CTA) { L.u[0][k] = 0.0; L.u[1][k] = 0.0; }
            __syncthreads();
        }
        if (P.lc == P.bottom) {
            if (threadIdx.x < 32)
                s_dense<true>(L, reinterpret_cast<double*>(sm + P.off_dense), reinterpret_cast<double*>(sm + P.off_rhs));
            __syncthreads();
        } else {
            for (int c = 0; c < P.ncoarse; ++c) s_vcycle_inner(P, sm, P.lc);
        }
    }
    for (int l = P.lc - 1; l >= P.lcta; --l) {
        const SL<T> L = make_sl<T>(P, sm, l);
        if (l + 1 == P.lc) s_prolong<T, double, false>(make_sl<double>(P, sm, l + 1), L);
        else s_prolong<T, T, false>(make_sl<T>(P, sm, l + 1), L);
        s_sweeps<T, false>(L, P.nu2, true);
    }
}

// Asynchronous copy of one 4- or 8-byte element global -> shared (completion:
// async_wait_all + barrier).
template <typename E>
__device__ __forceinline__ void cp_async_elem(E* dst, const E* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(E) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// Global (row-major, nrows x nx) -> colour-split shared (X0, X1), issued as asynchronous
// copies so that every level's arrays are in flight at once.
template <typename E>
__device__ __forceinline__ void stage_split(E* X0, E* X1, const E* __restrict__ g, int nx, int nrows, unsigned mag_h) {
    const int h = nx >> 1, items = nrows * h;
    ItemWalk wk(threadIdx.x, NT_CTA, h, mag_h);
    for (int it = threadIdx.x; it < items; it += NT_CTA) {
        const int j = wk.r, m = wk.q;
        const E* src = g + j * nx + 2 * m;
        const int k = j * h + m;
        cp_async_elem((j & 1) ? X1 + k : X0 + k, src);
        cp_async_elem((j & 1) ? X0 + k : X1 + k, src + 1);
        wk.next();
    }
}

template <typename T>
__global__ void __launch_bounds__(NT_CTA, 1) k_cta(const __grid_constant__ CtaParams P) {
    extern __shared__ __align__(16) unsigned char sm[];
    // stage beta of every level handled here and the bottom elimination, zero the ghost
    // rows of u, stage f(lcta)
    for (int l = P.lcta; l <= P.bottom; ++l) {
        const CtaLevel& L = P.lv[l];
        if (l < P.lc) {
            const SL<T> S = make_sl<T>(P, sm, l);
            stage_split(S.ax[0], S.ax[1], reinterpret_cast<const T*>(L.gax), L.nx, L.ny, L.mag_h);
            stage_split(S.ay[0], S.ay[1], reinterpret_cast<const T*>(L.gay), L.nx, L.ny + 1, L.mag_h);
            stage_split(S.di[0], S.di[1], reinterpret_cast<const T*>(L.gdi), L.nx, L.ny, L.mag_h);
            for (int k = threadIdx.x; k < L.half; k += NT_CTA) {
                S.u[0][k - L.half] = T(0); S.u[1][k - L.half] = T(0);
                S.u[0][L.ny * L.half + k] = T(0); S.u[1][L.ny * L.half + k] = T(0);
            }
        } else {
            const SL<double> S = make_sl<double>(P, sm, l);
            stage_split(S.ax[0], S.ax[1], reinterpret_cast<const double*>(L.gax), L.nx, L.ny, L.mag_h);
            stage_split(S.ay[0], S.ay[1], reinterpret_cast<const double*>(L.gay), L.nx, L.ny + 1, L.mag_h);
            stage_split(S.di[0], S.di[1], reinterpret_cast<const double*>(L.gdi), L.nx, L.ny, L.mag_h);
            for (int k = threadIdx.x; k < L.half; k += NT_CTA) {
                S.u[0][k - L.half] = 0.0; S.u[1][k - L.half] = 0.0;
                S.u[0][L.ny * L.half + k] = 0.0; S.u[1][L.ny * L.half + k] = 0.0;
            }
        }
    }
    {
        const int nb = P.lv[P.bottom].nx * P.lv[P.bottom].ny;
        double* A = reinterpret_cast<double*>(sm + P.off_dense);
        for (int k = threadIdx.x; k < nb * nb; k += NT_CTA) cp_async_elem(A + k, P.glu + k);
    }
    {
        const CtaLevel& L = P.lv[P.lcta];
        const T* fin = reinterpret_cast<const T*>(P.f_in);
        if (P.lcta < P.lc) {
            const SL<T> S = make_sl<T>(P, sm, P.lcta);
            stage_split(S.f[0], S.f[1], fin, L.nx, L.ny, L.mag_h);
            for (int k = threadIdx.x; k < L.ny * L.half; k += NT_CTA) { S.u[0][k] = T(0); S.u[1][k] = T(0); }
        } else {
            const SL<double> S = make_sl<double>(P, sm, P.lcta);
            if (std::is_same<T, double>::value) {
                stage_split(S.f[0], S.f[1], reinterpret_cast<const double*>(fin), L.nx, L.ny, L.mag_h);
            } else {
                const int h = L.half, items = L.ny * h;
                ItemWalk wk(threadIdx.x, NT_CTA, h, L.mag_h);
                for (int it = threadIdx.x; it < items; it += NT_CTA) {
                    const int j = wk.r, m = wk.q, k = j * h + m;
                    const double a = double(fin[j * L.nx + 2 * m]), b = double(fin[j * L.nx + 2 * m + 1]);
                    if (j & 1) { S.f[1][k] = a; S.f[0][k] = b; }
                    else { S.f[0][k] = a; S.f[1][k] = b; }
                    wk.next();
                }
            }
        }
    }
    async_wait_all();
    __syncthreads();
    s_outer<T>(P, sm);
    __syncthreads();
    {
        const CtaLevel& L = P.lv[P.lcta];
        T* uo = reinterpret_cast<T*>(P.u_out);
        const int h = L.half, items = L.ny * h;
        ItemWalk wk(threadIdx.x, NT_CTA, h, L.mag_h);
        for (int it = threadIdx.x; it < items; it += NT_CTA) {
            const int j = wk.r, m = wk.q, k = j * h + m;
            T a, b;
            if (P.lcta < P.lc) {
                const SL<T> S = make_sl<T>(P, sm, P.lcta);
                a = (j & 1) ? S.u[1][k] : S.u[0][k];
                b = (j & 1) ? S.u[0][k] : S.u[1][k];
            } else {
                const SL<double> S = make_sl<double>(P, sm, P.lcta);
                a = T((j & 1) ? S.u[1][k] : S.u[0][k]);
                b = T((j & 1) ? S.u[0][k] : S.u[1][k]);
            }
            uo[j * L.nx + 2 * m] = a;
            uo[j * L.nx + 2 * m + 1] = b;
            wk.next();
        }
    }
}

// ------------------------------------------------------------------------------------
// set-up kernels
// ------------------------------------------------------------------------------------
template <typename T>
__global__ void k_coarsen_beta(const T* __restrict__ bxf, const T* __restrict__ byf, T* __restrict__ bxc,
                               T* __restrict__ byc, int nxc, int nyc) {
    const int nxf = 2 * nxc;
    const int n = nxc * nyc, nb = nxc * (nyc + 1);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n + nb; k += gridDim.x * blockDim.x) {
        if (k < n) {
            const int J = k / nxc, I = k - J * nxc;
            bxc[k] = T(0.5) * (bxf[(size_t)(2 * J) * nxf + 2 * I] + bxf[(size_t)(2 * J + 1) * nxf + 2 * I]);
        } else {
            const int kk = k - n;
            const int J = kk / nxc, I = kk - J * nxc;
            byc[kk] = T(0.5) * (byf[(size_t)(2 * J) * nxf + 2 * I] + byf[(size_t)(2 * J) * nxf + 2 * I + 1]);
        }
    }
}

// AX = cx*bx; AY = cy*by inside, 0 on the bottom wall row, (2*cy)*by on the top wall row;
// DINV = 1/d with d = ((aw + ae) + as) + an, the diagonal the oracle forms per update.
template <typename T>
__global__ void k_scale_beta(const T* __restrict__ bx, const T* __restrict__ by, T* __restrict__ ax,
                             T* __restrict__ ay, T* __restrict__ dinv, int nx, int ny, T cx, T cy) {
    const size_t n = (size_t)nx * ny, nb = n + nx;
    const T cy2 = T(2) * cy;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n + nb; k += (size_t)gridDim.x * blockDim.x) {
        if (k < n) {
            const size_t j = k / nx, i = k - j * nx;
            const size_t ip = (i + 1 == (size_t)nx) ? 0 : i + 1;
            const T aw = cx * bx[k];
            const T ae = cx * bx[j * nx + ip];
            const T as = (j > 0) ? cy * by[k] : T(0);
            const T an = (j + 1 < (size_t)ny) ? cy * by[k + nx] : cy2 * by[k + nx];
            T d = aw;
            d += ae;
            d += as;
            d += an;
            ax[k] = aw;
            dinv[k] = T(1) / d;
        } else {
            const size_t kk = k - n;
            const size_t j = kk / nx;
            ay[kk] = (j == 0) ? T(0) : ((j == (size_t)ny) ? cy2 * by[kk] : cy * by[kk]);
        }
    }
}

// Elimination of the bottom level's dense matrix, done once per solve in shared memory:
// the oracle's dense_solve without its right-hand side (same assembly, pivots and
// products).  Output: U on and above the diagonal, the multipliers A[i][k] / piv below.
__global__ void k_dense_factor(const double* __restrict__ ax, const double* __restrict__ ay,
                               double* __restrict__ out, int nx, int ny) {
    extern __shared__ __align__(16) double A[];
    const int n = nx * ny, t = threadIdx.x, G = blockDim.x;
    for (int k = t; k < n * n; k += G) A[k] = 0.0;
    __syncthreads();
    if (t == 0) {
        for (int row = 0; row < n; ++row) {
            const int j = row / nx, i = row - j * nx;
            const int ip = (i + 1 == nx) ? 0 : i + 1, im = (i == 0) ? nx - 1 : i - 1;
            const double aw = ax[j * nx + i], ae = ax[j * nx + ip], as = ay[j * nx + i], an = ay[(j + 1) * nx + i];
            double d = aw;
            d += ae;
            d += as;
            d += an;
            A[row * n + row] -= d;
            A[row * n + j * nx + im] += aw;
            A[row * n + j * nx + ip] += ae;
            if (j > 0) A[row * n + (j - 1) * nx + i] += as;
            if (j < ny - 1) A[row * n + (j + 1) * nx + i] += an;
        }
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = A[k * n + k];
        const int m = n - k - 1;
        for (int q = t; q < m * m; q += G) {
            const int i = k + 1 + q / m, j = k + 1 + q % m;
            const double mult = A[i * n + k] / piv;
            A[i * n + j] -= mult * A[k * n + j];
        }
        __syncthreads();
        for (int i = k + 1 + t; i < n; i += G) A[i * n + k] = A[i * n + k] / piv;
        __syncthreads();
    }
    for (int k = t; k < n * n; k += G) out[k] = A[k];
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        b[k] = float(a[k]);
}

// After the loop: an odd iteration count leaves the solution in the internal buffer x1.
__global__ void k_finish(double* __restrict__ x0, const double* __restrict__ x1, const State* __restrict__ st,
                         size_t n) {
    if ((st->it & 1) == 0) return;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        x0[k] = x1[k];
}

__global__ void k_widen(const float* __restrict__ a, double* __restrict__ b, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        b[k] = double(a[k]);
}

// out = A u (FP64), the operator of the oracle's apply: out = s - d*u.
__global__ void __launch_bounds__(NT) k_apply(double* __restrict__ out, const double* __restrict__ u,
                                              const double* __restrict__ ax, const double* __restrict__ ay, int nx,
                                              int ny) {
    __shared__ __align__(16) double su[PRX * PRY];
    __shared__ __align__(16) double sax[PRX * PRY];
    __shared__ __align__(16) double say[PRX * PRY];
    const int gi0 = blockIdx.x * TX - PH, gj0 = blockIdx.y * TY - PH;
    load_plain(su, u, nx, ny, gi0, gj0);
    load_plain(sax, ax, nx, ny, gi0, gj0);
    load_plain(say, ay, nx, ny + 1, gi0, gj0);
    async_wait_all();
    __syncthreads();
    for (int k = threadIdx.x; k < TX * TY; k += blockDim.x) {
        const int ty = k / TX, tx = k - ty * TX;
        const int sx = tx + PH, sy = ty + PH;
        double s, d;
        plain_sums(su, sax, say, sx, sy, s, d);
        out[(size_t)(blockIdx.y * TY + ty) * nx + blockIdx.x * TX + tx] = s - d * su[sy * PRX + sx];
    }
}

__global__ void k_init_state(State* st, double tol, int max_it) {
    st->tol = tol;
    st->max_it = max_it;
    st->it = 0;
    st->status = LICA_NOT_CONVERGED;
    st->cont = 0;
    st->rz = 0.0;
    st->alpha = 0.0;
    st->beta = 0.0;
    st->rel = 0.0;
    st->rel_prev = 0.0;
    st->back = 0;
    st->kerr = 0;
    st->sums[0] = st->sums[1] = 0.0;
    for (int k = 0; k < 4; ++k) st->cnt[k] = 0u;
    st->bar_count = 0u;
    st->bar_gen = 0u;
}

__global__ void k_zero(double* __restrict__ a, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        a[k] = 0.0;
}

// ------------------------------------------------------------------------------------
// y-line zebra relaxation (lica_mg_options.smoother = 1, FP64): for strongly anisotropic
// cells (wall-normal stretching), where point relaxation stops smoothing along x.  Every
// level runs plain grid kernels in the oracle's order (oracle/mg2d.cpp, flag MG_YLINE):
// columns of one parity are each solved exactly along y by the Thomas algorithm with the
// x neighbours held, u(j-1) as - d u(j) + an u(j+1) = f - aw uw - ae ue (u = 0 past the
// top face); the residual and its 2x2 restriction; piecewise-constant prolongation; the
// bottom level by the dense elimination.  The pre-scaled weights AX, AY are the same
// products the oracle forms, so a preconditioner application is bit-identical.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_yline_half(double* __restrict__ u, const double* __restrict__ f,
                                                    const double* __restrict__ ax, const double* __restrict__ ay,
                                                    double* __restrict__ cp, double* __restrict__ dp, int nx, int ny,
                                                    int parity) {
    const int i = 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x) + parity;
    if (i >= nx) return;
    const int ip = (i + 1 == nx) ? 0 : i + 1, im = (i == 0) ? nx - 1 : i - 1;
    double prev_c = 0.0, prev_d = 0.0;
    for (int j = 0; j < ny; ++j) {
        const size_t k = (size_t)j * nx;
        const double aw = ax[k + i], ae = ax[k + ip], as = ay[k + i], an = ay[k + nx + i];
        double rhs = f[k + i];
        rhs -= aw * u[k + im];
        rhs -= ae * u[k + ip];
        double d = aw;
        d += ae;
        d += as;
        d += an;
        const double diag = -d;
        const double sup = (j < ny - 1) ? an : 0.0;
        const double den = diag - as * prev_c;  // as = 0 on the bottom row
        const double c = sup / den;
        const double e = (rhs - as * prev_d) / den;
        cp[k + i] = c;
        dp[k + i] = e;
        prev_c = c;
        prev_d = e;
    }
    double x = prev_d;
    u[(size_t)(ny - 1) * nx + i] = x;
    for (int j = ny - 2; j >= 0; --j) {
        const size_t k = (size_t)j * nx + i;
        x = dp[k] - cp[k] * x;
        u[k] = x;
    }
}

// Residual r = f - (s - d u) of the four children of coarse cell (I, J) and their 2x2
// average, fc = (r00 + r01) + (r10 + r11) times 1/4 in the oracle's order.
__global__ void k_resid_restrict(const double* __restrict__ u, const double* __restrict__ f,
                                 const double* __restrict__ ax, const double* __restrict__ ay, double* __restrict__ fc,
                                 int nx, int ny) {
    const int ncx = nx >> 1, ncy = ny >> 1;
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= ncx || J >= ncy) return;
    double r[2][2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const int i = 2 * I + a, j = 2 * J + b;
            const int ip = (i + 1 == nx) ? 0 : i + 1, im = (i == 0) ? nx - 1 : i - 1;
            const size_t k = (size_t)j * nx;
            const double aw = ax[k + i], ae = ax[k + ip], as = ay[k + i], an = ay[k + nx + i];
            const double uw = u[k + im], ue = u[k + ip];
            const double us = (j > 0) ? u[k - nx + i] : 0.0;
            const double un = (j < ny - 1) ? u[k + nx + i] : 0.0;
            double sm = aw * uw;
            sm += ae * ue;
            sm += as * us;
            sm += an * un;
            double d = aw;
            d += ae;
            d += as;
            d += an;
            r[b][a] = f[k + i] - (sm - d * u[k + i]);
        }
    }
    fc[(size_t)J * ncx + I] = 0.25 * ((r[0][0] + r[0][1]) + (r[1][0] + r[1][1]));
}

// u += P uc, piecewise constant.
__global__ void k_prolong_add(double* __restrict__ u, const double* __restrict__ uc, int nx, int ny) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    u[(size_t)j * nx + i] += uc[(size_t)(j >> 1) * (nx >> 1) + (i >> 1)];
}

// The bottom level's dense solve on row-major arrays (unknown row = j*nx + i): the
// elimination factors of k_dense_factor applied to f in the oracle's order, then its back
// substitution by thread 0 (the same arithmetic as s_dense).
__global__ void __launch_bounds__(64) k_dense_solve(const double* __restrict__ lu, const double* __restrict__ f,
                                                    double* __restrict__ u, int n) {
    __shared__ double b[kMaxDense];
    for (int k = threadIdx.x; k < n; k += blockDim.x) b[k] = f[k];
    __syncthreads();
    for (int k = 0; k + 1 < n; ++k) {
        const double bk = b[k];
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) b[i] -= lu[i * n + k] * bk;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int i = n - 1; i >= 0; --i) {
            double sm = b[i];
            for (int j = i + 1; j < n; ++j) sm -= lu[i * n + j] * b[j];
            b[i] = sm / lu[i * n + i];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] = b[k];
}

// r.z of the level-0 preconditioner application and the CG beta (the part of k_up's
// level-0 epilogue the y-line cycle needs).
__global__ void __launch_bounds__(256) k_rz(const double* __restrict__ r, const double* __restrict__ z, size_t n,
                                            State* __restrict__ st, double* __restrict__ partials) {
    __shared__ double red[32];
    double acc = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        acc += r[k] * z[k];
    const double b = block_sum(acc, red);
    double tot;
    if (grid_sum_last(b, partials, &st->cnt[0], &tot, red)) {
        st->beta = (st->it == 0) ? 0.0 : tot / st->rz;
        st->rz = tot;
    }
}

// The oracle's mixed path takes r.z with the FP32 copy of r (the V-cycle input), so the
// CG r.z partial of k_up<float,...,true> uses f (FP32) and z (FP32) -- the same values.

}  // namespace mg
}  // namespace lica

using namespace lica;
using namespace lica::mg;

// ------------------------------------------------------------------------------------
// host context
// ------------------------------------------------------------------------------------
struct LevelBuf {
    int nx = 0, ny = 0;
    double cx = 0, cy = 0;
    void* u = nullptr;      // T: iterate after pre-smoothing (k_down), or the CTA kernel's output
    void* up = nullptr;     // T: iterate after correction and post-smoothing (k_up)
    void* f = nullptr;      // T
    double* bx64 = nullptr;  // FP64 face beta (level 0: the caller's arrays), coarsened level by level
    double* by64 = nullptr;
    float* bx32 = nullptr;   // FP32 face beta (mixed), coarsened in FP32
    float* by32 = nullptr;
    double* ax64 = nullptr;  // pre-scaled stencil weights AX, AY and reciprocal diagonal (k_scale_beta)
    double* ay64 = nullptr;
    double* di64 = nullptr;
    float* ax32 = nullptr;
    float* ay32 = nullptr;
    float* di32 = nullptr;
};

struct lica_mg {
    int nx, ny;
    int nsm = 148;  // SMs of the device (persistent grids)
    // the persistent TMA-staged CG kernels (level 0 with at least one 32 x 32 tile per SM)
    bool cg_tma = false;
    CgMaps cgm{};
    const void* cg_x = nullptr;  // the caller's x and f the maps cgm.x[0], cgm.xw[0], cgm.f describe
    const void* cg_f = nullptr;
    double hx, hy;
    lica_mg_options o;
    int nouter = 0, lcta = 0, bottom = 0;
    bool mid = false;  // levels 1 .. lcta-1 (two or more) run as the cross-level kernels
    bool yline = false;  // y-line zebra relaxation on every level (lica_mg_options.smoother = 1)
    double *ycp = nullptr, *ydp = nullptr;  // the line solves' Thomas scratch (level-0 size)
    std::vector<LevelBuf> lv;  // outer levels then inner levels
    size_t cta_smem = 0;
    CtaParams cp{};
    // level-0 CG vectors
    double* pcg[2] = {nullptr, nullptr};  // p, ping-pong by iteration parity
    double* xb = nullptr;    // second x buffer (the first is the caller's)
    void* r = nullptr;       // r (T): the V-cycle's level-0 f
    void* zpre = nullptr;    // z after pre-smoothing (T)
    void* z = nullptr;       // z (T): the V-cycle's level-0 output
    double* partials = nullptr;
    double* dense_lu = nullptr;  // bottom-level elimination, refreshed by every set-up
    State* st = nullptr;
    State* st_host = nullptr;  // pinned
    // host staging for lica_mg_solve_host
    double *d_p = nullptr, *d_f = nullptr, *d_bx = nullptr, *d_by = nullptr;
    cudaStream_t own_stream = nullptr;
    // lica_mg_solve_host_batch: double-buffered input staging [2] (p0, f, bx, by in one block),
    // output staging [2], upload and download streams and their ordering events
    double* b_in[2] = {nullptr, nullptr};
    double* b_out[2] = {nullptr, nullptr};
    cudaStream_t b_up = nullptr, b_down = nullptr;
    State* b_states = nullptr;  // pinned: each batched solve's final state
    int b_states_cap = 0;
    cudaEvent_t b_ev_in[2] = {nullptr, nullptr}, b_ev_used[2] = {nullptr, nullptr};
    cudaEvent_t b_ev_solved[2] = {nullptr, nullptr}, b_ev_out[2] = {nullptr, nullptr};
    cudaStream_t cap_stream = nullptr;  // graphs are captured here, launched on the caller's stream
    // graph cache
    // the solve's graph for the arrays, stream, tolerance and iteration cap of the last solve,
    // and the one before it (a batch alternates between two staging buffers)
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
        cudaStream_t stream = nullptr;
        double tol = -1.0;
        int max = -1;
    };
    GraphSlot gcur, galt;
    int body_nodes = 0, setup_nodes = 0;
    // optional per-kernel-class timing (non-graph solves only)
    bool profile = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
    double prof_ms[LICA_MG_NCLASS] = {0};
    int64_t prof_n[LICA_MG_NCLASS] = {0};
    std::vector<cudaEvent_t> event_pool;
};

namespace {

bool is_mixed(const lica_mg* m) { return m->o.precision == 1; }

PFN_cuTensorMapEncodeTiled_v12000 mg_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// A 2-D map of a row-major w x h array (FP32 or FP64) with a bw x bh box, zero fill.
int tm_map(CUtensorMap* mp, const void* base, bool f32, int w, int h, int bw, int bh) {
    auto fn = mg_encode_fn();
    if (!fn) {
        lica_set_last_error("cuTensorMapEncodeTiled", "driver entry point unavailable", __FILE__, __LINE__);
        return LICA_ERR_CUDA;
    }
    const cuuint64_t es = f32 ? 4 : 8;
    cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
    cuuint64_t strides[1] = {(cuuint64_t)w * es};
    cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
    cuuint32_t el[2] = {1, 1};
    const CUresult r = fn(mp, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                          const_cast<void*>(base), dims, strides, box, el, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        lica_set_last_error("cuTensorMapEncodeTiled", "multigrid tile map rejected", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    return LICA_OK;
}

// Profiling: bracket one kernel launch with events when profiling is on.
cudaEvent_t pool_event(lica_mg* m) {
    if (!m->event_pool.empty()) {
        cudaEvent_t e = m->event_pool.back();
        m->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
struct ProfScope {
    lica_mg* m;
    int cls;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(lica_mg* m_, int cls_, cudaStream_t s_) : m(m_), cls(cls_), s(s_) {
        if (m->profile) {
            a = pool_event(m);
            b = pool_event(m);
            cudaEventRecord(a, s);
        }
    }
    ~ProfScope() {
        if (m->profile) {
            cudaEventRecord(b, s);
            m->prof_pending.push_back({cls, {a, b}});
        }
    }
};
void prof_collect(lica_mg* m) {
    for (auto& pe : m->prof_pending) {
        float ms = 0.f;
        cudaEventSynchronize(pe.second.second);
        cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
        m->prof_ms[pe.first] += ms;
        m->prof_n[pe.first] += 1;
        m->event_pool.push_back(pe.second.first);
        m->event_pool.push_back(pe.second.second);
    }
    m->prof_pending.clear();
}

template <typename T>
const T* lvl_ax(const LevelBuf& L) {
    return std::is_same<T, float>::value ? (const T*)L.ax32 : (const T*)L.ax64;
}
template <typename T>
const T* lvl_ay(const LevelBuf& L) {
    return std::is_same<T, float>::value ? (const T*)L.ay32 : (const T*)L.ay64;
}
template <typename T>
const T* lvl_di(const LevelBuf& L) {
    return std::is_same<T, float>::value ? (const T*)L.di32 : (const T*)L.di64;
}

// Smoothing tiles: 32 x 32 cells on levels with at least one tile per SM, 16 x 16 below
// (more CTAs in flight where the level is small and each tile's latency is the cost);
// strips of 4 rows per thread.
constexpr int RB_R = RB_TILE_R;
constexpr int kSMs = 148;
bool big_tiles(const LevelBuf& L) { return L.nx % 32 == 0 && L.ny % 32 == 0 && (L.nx / 32) * (L.ny / 32) >= kSMs; }

template <typename T, int NS, int TS>
void down_tile(const LevelBuf& L, const LevelBuf& C, cudaStream_t s) {
    using Cfg = RBCfg<NS, TS, TS, RB_R>;
    dim3 grid(L.nx / TS, L.ny / TS);
    k_down<T, NS, TS, TS, RB_R><<<grid, Cfg::NTH, 0, s>>>((const T*)L.f, lvl_ax<T>(L), lvl_ay<T>(L), lvl_di<T>(L),
                                                          (T*)L.u, (T*)C.f, L.nx, L.ny);
}

template <typename T, int NS>
void down_ns(const LevelBuf& L, const LevelBuf& C, cudaStream_t s) {
    if (big_tiles(L)) down_tile<T, NS, 32>(L, C, s);
    else down_tile<T, NS, 16>(L, C, s);
}

template <typename T>
int launch_down(lica_mg* m, int l, cudaStream_t s) {
    LevelBuf& L = m->lv[l];
    LevelBuf& C = m->lv[l + 1];
    ProfScope ps(m, l == 0 ? LICA_MG_DOWN0 : LICA_MG_DOWN, s);
    switch (m->o.nu1) {
        case 1: down_ns<T, 1>(L, C, s); break;
        case 2: down_ns<T, 2>(L, C, s); break;
        default: down_ns<T, 3>(L, C, s); break;
    }
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

template <typename T, int NS, int TS>
void up_tile(lica_mg* m, const LevelBuf& L, const T* uc, bool level0, cudaStream_t s) {
    using Cfg = RBCfg<NS, TS, TS, RB_R>;
    dim3 grid(L.nx / TS, L.ny / TS);
    if (level0)
        k_up<T, NS, TS, TS, RB_R, true><<<grid, Cfg::NTH, 0, s>>>((const T*)L.u, (T*)L.up, uc, (const T*)L.f,
                                                                  lvl_ax<T>(L), lvl_ay<T>(L), lvl_di<T>(L), L.nx,
                                                                  L.ny, m->st, m->partials);
    else
        k_up<T, NS, TS, TS, RB_R, false><<<grid, Cfg::NTH, 0, s>>>((const T*)L.u, (T*)L.up, uc, (const T*)L.f,
                                                                   lvl_ax<T>(L), lvl_ay<T>(L), lvl_di<T>(L), L.nx,
                                                                   L.ny, m->st, m->partials);
}

template <typename T, int NS>
void up_ns(lica_mg* m, const LevelBuf& L, const T* uc, bool level0, cudaStream_t s) {
    if (big_tiles(L)) up_tile<T, NS, 32>(m, L, uc, level0, s);
    else up_tile<T, NS, 16>(m, L, uc, level0, s);
}

template <typename T>
int launch_up(lica_mg* m, int l, cudaStream_t s) {
    LevelBuf& L = m->lv[l];
    LevelBuf& C = m->lv[l + 1];
    const T* uc = (const T*)((l + 1 == m->lcta) ? C.u : C.up);
    ProfScope ps(m, l == 0 ? LICA_MG_UP0 : LICA_MG_UP, s);
    switch (m->o.nu2) {
        case 1: up_ns<T, 1>(m, L, uc, l == 0, s); break;
        case 2: up_ns<T, 2>(m, L, uc, l == 0, s); break;
        default: up_ns<T, 3>(m, L, uc, l == 0, s); break;
    }
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

// The cross-level kernels for levels 1 .. lcta-1 (two or more of them), one cooperative
// launch per leg; the grid is at most what the device holds at once, so the blocks meet at
// every barrier.
template <typename T>
MidParams mid_params(lica_mg* m) {
    MidParams P{};
    P.l0 = 1;
    P.l1 = m->lcta;
    P.st = m->st;
    for (int l = 1; l < m->lcta; ++l) {
        const LevelBuf& L = m->lv[l];
        const LevelBuf& C = m->lv[l + 1];
        MidLevel& M = P.lv[l];
        M.nx = L.nx;
        M.ny = L.ny;
        M.big = big_tiles(L) ? 1 : 0;
        M.f = L.f;
        M.ax = lvl_ax<T>(L);
        M.ay = lvl_ay<T>(L);
        M.di = lvl_di<T>(L);
        M.u = L.u;
        M.fc = C.f;
        M.upre = L.u;
        M.uc = (l + 1 == m->lcta) ? C.u : C.up;
        M.up = L.up;
    }
    return P;
}

template <typename T, int NS>
int launch_mid_ns(lica_mg* m, bool up, cudaStream_t s) {
    const MidParams P = mid_params<T>(m);
    int tiles = 0;
    for (int l = P.l0; l < P.l1; ++l) {
        const int ts = P.lv[l].big ? 32 : 16;
        tiles = std::max(tiles, (P.lv[l].nx / ts) * (P.lv[l].ny / ts));
    }
    auto kern = up ? k_up_mid<T, NS> : k_down_mid<T, NS>;
    const int nth = RBCfg<NS, 32, 32, RB_R>::NTH;
    int occ = 0;
    LICA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, nth, 0));
    if (occ < 1) return LICA_ERR_CUDA;
    const int grid = std::min(tiles, occ * m->nsm);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(nth);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    LICA_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, P));
    lica_count_launches(1);
    return LICA_OK;
}

template <typename T>
int launch_mid(lica_mg* m, bool up, cudaStream_t s) {
    ProfScope ps(m, up ? LICA_MG_UP : LICA_MG_DOWN, s);
    switch (up ? m->o.nu2 : m->o.nu1) {
        case 1: return launch_mid_ns<T, 1>(m, up, s);
        case 2: return launch_mid_ns<T, 2>(m, up, s);
        default: return launch_mid_ns<T, 3>(m, up, s);
    }
}

template <typename T>
int launch_cta(lica_mg* m, cudaStream_t s) {
    CtaParams P = m->cp;
    P.f_in = m->lv[m->lcta].f;
    P.u_out = m->lv[m->lcta].u;
    ProfScope ps(m, LICA_MG_CTA, s);
    k_cta<T><<<1, NT_CTA, m->cta_smem, s>>>(P);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

// z = M r on the level-0 buffers m->r (input) and m->z (output).
template <typename T>
int vcycle(lica_mg* m, cudaStream_t s) {
    int st;
    if (m->mid) {
        if ((st = launch_down<T>(m, 0, s)) || (st = launch_mid<T>(m, false, s)) || (st = launch_cta<T>(m, s)) ||
            (st = launch_mid<T>(m, true, s)) || (st = launch_up<T>(m, 0, s)))
            return st;
        return LICA_OK;
    }
    for (int l = 0; l < m->lcta; ++l)
        if ((st = launch_down<T>(m, l, s))) return st;
    if ((st = launch_cta<T>(m, s))) return st;
    for (int l = m->lcta - 1; l >= 0; --l)
        if ((st = launch_up<T>(m, l, s))) return st;
    return LICA_OK;
}

// The y-line V-cycle (FP64), z = M r on m->r / m->z; the oracle's vcycle_outer with
// coarse_solve and vcycle_inner.
int yl_smooth(lica_mg* m, int l, double* u, const double* f, int nsw, bool reverse, cudaStream_t s) {
    const LevelBuf& L = m->lv[l];
    const int cols = L.nx / 2;
    for (int q = 0; q < nsw; ++q)
        for (int c = 0; c < 2; ++c) {
            const int parity = reverse ? 1 - c : c;
            k_yline_half<<<(cols + 127) / 128, 128, 0, s>>>(u, f, L.ax64, L.ay64, m->ycp, m->ydp, L.nx, L.ny, parity);
            LICA_CUDA_TRY(cudaGetLastError());
            lica_count_launches(1);
        }
    return LICA_OK;
}

int yl_restrict(lica_mg* m, int l, const double* u, const double* f, cudaStream_t s) {
    const LevelBuf& L = m->lv[l];
    const dim3 blk(32, 8), grid((L.nx / 2 + 31) / 32, (L.ny / 2 + 7) / 8);
    k_resid_restrict<<<grid, blk, 0, s>>>(u, f, L.ax64, L.ay64, (double*)m->lv[l + 1].f, L.nx, L.ny);
    LICA_CUDA_TRY(cudaGetLastError());
    LICA_CUDA_TRY(cudaMemsetAsync(m->lv[l + 1].u, 0, sizeof(double) * (size_t)m->lv[l + 1].nx * m->lv[l + 1].ny, s));
    lica_count_launches(1);
    return LICA_OK;
}

int yl_prolong(lica_mg* m, int l, double* u, cudaStream_t s) {
    const LevelBuf& L = m->lv[l];
    const dim3 blk(32, 8), grid((L.nx + 31) / 32, (L.ny + 7) / 8);
    k_prolong_add<<<grid, blk, 0, s>>>(u, (const double*)m->lv[l + 1].u, L.nx, L.ny);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int yl_dense(lica_mg* m, cudaStream_t s) {
    const LevelBuf& B = m->lv[m->bottom];
    k_dense_solve<<<1, 64, 0, s>>>(m->dense_lu, (const double*)B.f, (double*)B.u, B.nx * B.ny);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int yl_inner(lica_mg* m, int l, cudaStream_t s) {
    if (l == m->bottom) return yl_dense(m, s);
    double* u = (double*)m->lv[l].u;
    const double* f = (const double*)m->lv[l].f;
    int st;
    if ((st = yl_smooth(m, l, u, f, m->o.nu1, false, s)) || (st = yl_restrict(m, l, u, f, s)) ||
        (st = yl_inner(m, l + 1, s)) || (st = yl_prolong(m, l, u, s)) || (st = yl_smooth(m, l, u, f, m->o.nu2, true, s)))
        return st;
    return LICA_OK;
}

int vcycle_yline(lica_mg* m, cudaStream_t s) {
    const int lc = m->nouter - 1;
    int st;
    LICA_CUDA_TRY(cudaMemsetAsync(m->z, 0, sizeof(double) * (size_t)m->nx * m->ny, s));
    {
        ProfScope ps(m, LICA_MG_DOWN, s);
        for (int l = 0; l < lc; ++l) {
            double* u = l == 0 ? (double*)m->z : (double*)m->lv[l].u;
            const double* f = l == 0 ? (const double*)m->r : (const double*)m->lv[l].f;
            if ((st = yl_smooth(m, l, u, f, m->o.nu1, false, s)) || (st = yl_restrict(m, l, u, f, s))) return st;
        }
    }
    {
        ProfScope ps(m, LICA_MG_CTA, s);
        if (lc == 0) return LICA_BAD_ARG;
        if (lc == m->bottom) {
            if ((st = yl_dense(m, s))) return st;
        } else {
            for (int c = 0; c < m->o.ncoarse; ++c)
                if ((st = yl_inner(m, lc, s))) return st;
        }
    }
    {
        ProfScope ps(m, LICA_MG_UP, s);
        for (int l = lc - 1; l >= 0; --l) {
            double* u = l == 0 ? (double*)m->z : (double*)m->lv[l].u;
            const double* f = l == 0 ? (const double*)m->r : (const double*)m->lv[l].f;
            if ((st = yl_prolong(m, l, u, s)) || (st = yl_smooth(m, l, u, f, m->o.nu2, true, s))) return st;
        }
    }
    const size_t n0 = (size_t)m->nx * m->ny;
    const int nb = (int)std::min<size_t>(148, (n0 + 255) / 256);
    k_rz<<<nb, 256, 0, s>>>((const double*)m->r, (const double*)m->z, n0, m->st, m->partials);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int run_vcycle(lica_mg* m, cudaStream_t s) {
    if (m->yline) return vcycle_yline(m, s);
    return is_mixed(m) ? vcycle<float>(m, s) : vcycle<double>(m, s);
}

// Beta hierarchy for the caller's level-0 faces bx, by: FP64 faces coarsened level by
// level, and every level's pre-scaled weights AX, AY; in the mixed path also the FP32
// faces (FP32 copy of level 0, coarsened in FP32) and their FP32 weights.
int setup_beta(lica_mg* m, const double* bx, const double* by, cudaStream_t s) {
    ProfScope ps(m, LICA_MG_SETUP, s);
    m->lv[0].bx64 = const_cast<double*>(bx);
    m->lv[0].by64 = const_cast<double*>(by);
    const int nlev = (int)m->lv.size();
    auto blocks_for = [](size_t work) { return (int)std::min<size_t>(1184, (work + 255) / 256); };
    for (int l = 0; l < nlev; ++l) {
        LevelBuf& C = m->lv[l];
        const size_t work = (size_t)C.nx * C.ny * 2 + C.nx;
        if (l > 0) {
            LevelBuf& F = m->lv[l - 1];
            k_coarsen_beta<double><<<blocks_for(work), 256, 0, s>>>(F.bx64, F.by64, C.bx64, C.by64, C.nx, C.ny);
            LICA_CUDA_TRY(cudaGetLastError());
            lica_count_launches(1);
        }
        k_scale_beta<double><<<blocks_for(work), 256, 0, s>>>(C.bx64, C.by64, C.ax64, C.ay64, C.di64, C.nx, C.ny,
                                                               C.cx, C.cy);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(1);
    }
    if (is_mixed(m)) {
        LevelBuf& L0 = m->lv[0];
        const size_t n = (size_t)L0.nx * L0.ny;
        k_to_float<<<1184, 256, 0, s>>>(bx, L0.bx32, n);
        k_to_float<<<1184, 256, 0, s>>>(by, L0.by32, n + L0.nx);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(2);
        for (int l = 0; l < m->nouter - 1; ++l) {
            LevelBuf& C = m->lv[l];
            const size_t work = (size_t)C.nx * C.ny * 2 + C.nx;
            if (l > 0) {
                LevelBuf& F = m->lv[l - 1];
                k_coarsen_beta<float><<<blocks_for(work), 256, 0, s>>>(F.bx32, F.by32, C.bx32, C.by32, C.nx, C.ny);
                LICA_CUDA_TRY(cudaGetLastError());
                lica_count_launches(1);
            }
            k_scale_beta<float><<<blocks_for(work), 256, 0, s>>>(C.bx32, C.by32, C.ax32, C.ay32, C.di32, C.nx, C.ny,
                                                                  float(C.cx), float(C.cy));
            LICA_CUDA_TRY(cudaGetLastError());
            lica_count_launches(1);
        }
    }
    {
        const LevelBuf& B = m->lv[m->bottom];
        const int nb = B.nx * B.ny;
        k_dense_factor<<<1, 256, sizeof(double) * nb * nb, s>>>(B.ax64, B.ay64, m->dense_lu, B.nx, B.ny);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(1);
    }
    // weights of the levels staged by the single-CTA kernel
    for (int l = m->lcta; l <= m->bottom; ++l) {
        if (l < m->nouter - 1 && is_mixed(m)) {
            m->cp.lv[l].gax = m->lv[l].ax32;
            m->cp.lv[l].gay = m->lv[l].ay32;
            m->cp.lv[l].gdi = m->lv[l].di32;
        } else {
            m->cp.lv[l].gax = m->lv[l].ax64;
            m->cp.lv[l].gay = m->lv[l].ay64;
            m->cp.lv[l].gdi = m->lv[l].di64;
        }
    }
    return LICA_OK;
}

// Maps of the caller's x (the first x buffer) and f for the TMA CG kernels, re-encoded when
// the pointers change.
int cg_maps_for(lica_mg* m, const double* x, const double* f) {
    if (m->cg_x == x && m->cg_f == f) return LICA_OK;
    const int nx = m->nx, ny = m->ny;
    int st;
    if ((st = tm_map(&m->cgm.x[0], x, false, nx, ny, CG_BW, CG_BH)) ||
        (st = tm_map(&m->cgm.xw[0], x, false, nx, ny, CG_WW, CG_BH)) ||
        (st = tm_map(&m->cgm.f, f, false, nx, ny, CG_BW, CG_BH)))
        return st;
    m->cg_x = x;
    m->cg_f = f;
    return LICA_OK;
}

template <typename TZ, bool XUP>
int launch_cg_tma(lica_mg* m, double* x, cudaGraphConditionalHandle h, int use_cond, cudaStream_t s) {
    LevelBuf& L = m->lv[0];
    CgArgs A;
    A.m = m->cgm;
    A.pbuf[0] = m->pcg[0];
    A.pbuf[1] = m->pcg[1];
    A.xbuf[0] = x;
    A.xbuf[1] = m->xb;
    A.r_out = m->r;
    A.nx = L.nx;
    A.ny = L.ny;
    A.ntx = L.nx / CG_TS;
    A.nty = L.ny / CG_TS;
    A.st = m->st;
    A.partials = m->partials;
    A.cond = h;
    A.use_cond = use_cond;
    const int grid = std::min(A.ntx * A.nty, m->nsm);
    k_cg_tma<TZ, XUP><<<grid, CG_NT, CgLayout<TZ, XUP>::BYTES, s>>>(A);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

template <typename TR>
int launch_xupdate(lica_mg* m, double* x, const double* f, int first, cudaGraphConditionalHandle h, int use_cond,
                   cudaStream_t s) {
    LevelBuf& L = m->lv[0];
    if (m->cg_tma && !first) {
        ProfScope ps(m, LICA_MG_XUPDATE, s);
        int st = cg_maps_for(m, x, f);
        if (st) return st;
        return launch_cg_tma<TR, true>(m, x, h, use_cond, s);
    }
    dim3 grid(L.nx / TX, L.ny / TY);
    ProfScope ps(m, LICA_MG_XUPDATE, s);
    k_xupdate<TR><<<grid, NT, xupdate_smem(), s>>>(x, m->xb, m->pcg[0], m->pcg[1], f, L.ax64, L.ay64, (TR*)m->r, L.nx, L.ny,
                                      m->st, m->partials, first, h, use_cond);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

template <typename TZ>
int launch_pupdate(lica_mg* m, cudaStream_t s) {
    LevelBuf& L = m->lv[0];
    if (m->cg_tma) {
        ProfScope ps(m, LICA_MG_PUPDATE, s);
        return launch_cg_tma<TZ, false>(m, nullptr, cudaGraphConditionalHandle{}, 0, s);
    }
    dim3 grid(L.nx / TX, L.ny / TY);
    ProfScope ps(m, LICA_MG_PUPDATE, s);
    k_pupdate<TZ><<<grid, NT, pupdate_smem<TZ>(), s>>>(m->pcg[0], m->pcg[1], (const TZ*)m->z, L.ax64, L.ay64, L.nx, L.ny, m->st,
                                      m->partials);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

// Set-up part of a solve: state, beta hierarchy, p = 0, r = f - A x, ||f||, rel.
int enqueue_setup(lica_mg* m, double* x, const double* f, const double* bx, const double* by, double rtol,
                  int max_it, cudaGraphConditionalHandle h, int use_cond, cudaStream_t s) {
    int st;
    k_init_state<<<1, 1, 0, s>>>(m->st, rtol, max_it);
    LICA_CUDA_TRY(cudaGetLastError());
    const size_t n = (size_t)m->nx * m->ny;
    k_zero<<<1184, 256, 0, s>>>(m->pcg[0], n);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(2);
    if ((st = setup_beta(m, bx, by, s))) return st;
    return is_mixed(m) ? launch_xupdate<float>(m, x, f, 1, h, use_cond, s)
                       : launch_xupdate<double>(m, x, f, 1, h, use_cond, s);
}

// One PCG iteration: z = M r; beta; p = z + beta p; alpha; x += alpha p; r = f - A x.
int enqueue_iteration(lica_mg* m, double* x, const double* f, cudaGraphConditionalHandle h, int use_cond,
                      cudaStream_t s) {
    int st;
    m->lv[0].u = m->zpre;
    m->lv[0].up = m->z;
    m->lv[0].f = m->r;
    if ((st = run_vcycle(m, s))) return st;
    if (is_mixed(m)) {
        if ((st = launch_pupdate<float>(m, s))) return st;
        return launch_xupdate<float>(m, x, f, 0, h, use_cond, s);
    }
    if ((st = launch_pupdate<double>(m, s))) return st;
    return launch_xupdate<double>(m, x, f, 0, h, use_cond, s);
}

int enqueue_finish(lica_mg* m, double* x, cudaStream_t s) {
    k_finish<<<1184, 256, 0, s>>>(x, m->xb, m->st, (size_t)m->nx * m->ny);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int read_state(lica_mg* m, cudaStream_t s) {
    LICA_CUDA_TRY(cudaMemcpyAsync(m->st_host, m->st, sizeof(State), cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    return LICA_OK;
}

int build_graph(lica_mg* m, double* x, const double* f, const double* bx, const double* by, double rtol,
                int max_it, cudaStream_t launch_stream) {
    (void)launch_stream;
    if (!m->cap_stream) LICA_CUDA_TRY(cudaStreamCreateWithFlags(&m->cap_stream, cudaStreamNonBlocking));
    cudaStream_t s = m->cap_stream;
    const bool prof = m->profile;
    m->profile = false;
    struct Restore {
        lica_mg* m;
        bool p;
        ~Restore() { m->profile = p; }
    } restore{m, prof};
    if (m->gcur.exec) {
        cudaGraphExecDestroy(m->gcur.exec);
        m->gcur = lica_mg::GraphSlot{};
    }
    cudaGraph_t g;
    LICA_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    LICA_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    // set-up part, captured into g
    int64_t before = lica_kernel_launch_count();
    LICA_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_setup(m, x, f, bx, by, rtol, max_it, h, 1, s);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &captured);
    if (st) { cudaGraphDestroy(g); return st; }
    LICA_CUDA_TRY(e);
    m->setup_nodes = (int)(lica_kernel_launch_count() - before);
    // conditional WHILE node after the set-up nodes
    size_t nleaf = 0;
    LICA_CUDA_TRY(cudaGraphGetNodes(g, nullptr, &nleaf));
    std::vector<cudaGraphNode_t> nodes(nleaf);
    LICA_CUDA_TRY(cudaGraphGetNodes(g, nodes.data(), &nleaf));
    // the set-up was captured on one stream: its sink is the last node added
    std::vector<cudaGraphNode_t> sinks;
    for (auto nd : nodes) {
        size_t nout = 0;
        LICA_CUDA_TRY(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
        if (nout == 0) sinks.push_back(nd);
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    LICA_CUDA_TRY(cudaGraphAddNode(&wnode, g, sinks.data(), sinks.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    before = lica_kernel_launch_count();
    LICA_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    st = enqueue_iteration(m, x, f, h, 1, s);
    e = cudaStreamEndCapture(s, &captured);
    if (st) { cudaGraphDestroy(g); return st; }
    LICA_CUDA_TRY(e);
    m->body_nodes = (int)(lica_kernel_launch_count() - before);
    // finishing copy after the WHILE node, captured into g
    {
        cudaGraph_t fin;
        LICA_CUDA_TRY(cudaGraphCreate(&fin, 0));
        LICA_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, fin, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        st = enqueue_finish(m, x, s);
        e = cudaStreamEndCapture(s, &captured);
        if (st) { cudaGraphDestroy(fin); cudaGraphDestroy(g); return st; }
        LICA_CUDA_TRY(e);
        cudaGraphNode_t child;
        e = cudaGraphAddChildGraphNode(&child, g, &wnode, 1, fin);
        cudaGraphDestroy(fin);
        LICA_CUDA_TRY(e);
        m->setup_nodes += 1;
    }
    // the captures counted as launches; undo that (replays are counted per run)
    lica_count_launches(-(int64_t)(m->setup_nodes + m->body_nodes));
    e = cudaGraphInstantiate(&m->gcur.exec, g, 0);
    cudaGraphDestroy(g);
    LICA_CUDA_TRY(e);
    m->gcur.key[0] = x; m->gcur.key[1] = f; m->gcur.key[2] = bx; m->gcur.key[3] = by;
    m->gcur.stream = launch_stream;
    return LICA_OK;
}

// The kernels read two cells per 16-byte vector load: caller arrays must be 16-byte aligned.
bool aligned16(const void* a, const void* b, const void* c, const void* d) {
    const uintptr_t u = (uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)d;
    if (u & 15u) {
        lica_set_last_error("lica_mg", "device arrays must be 16-byte aligned", __FILE__, __LINE__);
        return false;
    }
    return true;
}

// Launch the solve's graph (built, or rebuilt for new arrays, tolerance or stream) on s.
int graph_launch(lica_mg* m, double* x, const double* f, const double* bx, const double* by, double rtol, int max_it,
                 cudaStream_t s) {
    int st;
    // rtol/max_it live in the graph's k_init_state node: a graph serves only its own
    auto match = [&](const lica_mg::GraphSlot& g) {
        return g.exec && g.key[0] == x && g.key[1] == f && g.key[2] == bx && g.key[3] == by && g.stream == s &&
               g.tol == rtol && g.max == max_it;
    };
    if (!match(m->gcur)) {
        // keep the current graph as the alternate; use the alternate if it fits, else build
        std::swap(m->gcur, m->galt);
        if (!match(m->gcur)) {
            if ((st = build_graph(m, x, f, bx, by, rtol, max_it, s))) return st;
            m->gcur.tol = rtol;
            m->gcur.max = max_it;
        }
    }
    LICA_CUDA_TRY(cudaGraphLaunch(m->gcur.exec, s));
    return LICA_OK;
}

int solve_impl(lica_mg* m, double* x, const double* f, const double* bx, const double* by, double rtol, int max_it,
               lica_mg_result* res, cudaStream_t s) {
    if (!m || !x || !f || !bx || !by || !(rtol >= 0.0) || max_it < 0) return LICA_BAD_ARG;
    if (!aligned16(x, f, bx, by)) return LICA_BAD_ARG;
    int st;
    if (m->o.use_graph && !m->profile) {
        if ((st = graph_launch(m, x, f, bx, by, rtol, max_it, s))) return st;
        if ((st = read_state(m, s))) return st;
        lica_count_launches(m->setup_nodes + (int64_t)(m->st_host->it + m->st_host->back) * m->body_nodes);
    } else {
        cudaGraphConditionalHandle h{};
        if ((st = enqueue_setup(m, x, f, bx, by, rtol, max_it, h, 0, s))) return st;
        if ((st = read_state(m, s))) return st;
        while (m->st_host->cont) {
            if ((st = enqueue_iteration(m, x, f, h, 0, s))) return st;
            if ((st = read_state(m, s))) return st;
        }
        if ((st = enqueue_finish(m, x, s))) return st;
        if ((st = read_state(m, s))) return st;
        if (m->profile) prof_collect(m);
    }
    if (res) {
        res->iterations = m->st_host->it;
        res->status = m->st_host->status;
        res->rel_residual = m->st_host->rel;
    }
    return m->st_host->status;
}

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" {

int lica_mg_create(lica_mg** out, int32_t nx, int32_t ny, double hx, double hy, const lica_mg_options* opt) {
    if (!out || !opt) return LICA_BAD_ARG;
    *out = nullptr;
    const lica_mg_options o = *opt;
    if (nx < TX || ny < TY || nx % TX || ny % TY || !(hx > 0) || !(hy > 0) || o.nlevels < 2 ||
        o.nlevels > 12 || o.nu1 < 1 || o.nu1 > 3 || o.nu2 < 1 || o.nu2 > 3 || o.ncoarse < 1 ||
        (o.precision != 0 && o.precision != 1) || (o.smoother != 0 && o.smoother != 1) ||
        (o.smoother == 1 && o.precision != 0)) {
        lica_set_last_error("lica_mg_create", "unsupported sizes or options", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    lica_mg* m = new lica_mg();
    m->nx = nx; m->ny = ny; m->hx = hx; m->hy = hy; m->o = o;
    // outer levels
    int cx = nx, cy = ny;
    double chx = hx, chy = hy;
    for (int l = 0; l < o.nlevels; ++l) {
        if (l > 0) {
            if ((cx & 1) || (cy & 1) || cx < 4 || cy < 2) { delete m; return LICA_BAD_ARG; }
            cx /= 2; cy /= 2; chx *= 2; chy *= 2;
        }
        LevelBuf L;
        L.nx = cx; L.ny = cy; L.cx = 1.0 / (chx * chx); L.cy = 1.0 / (chy * chy);
        m->lv.push_back(L);
    }
    m->nouter = o.nlevels;
    while (!(cx & 1) && !(cy & 1) && cx / 2 >= 2 && cy / 2 >= 2) {
        cx /= 2; cy /= 2; chx *= 2; chy *= 2;
        LevelBuf L;
        L.nx = cx; L.ny = cy; L.cx = 1.0 / (chx * chx); L.cy = 1.0 / (chy * chy);
        m->lv.push_back(L);
    }
    m->bottom = (int)m->lv.size() - 1;
    if (m->lv[m->bottom].nx * m->lv[m->bottom].ny > kMaxDense || (int)m->lv.size() > kMaxLevels) {
        delete m;
        lica_set_last_error("lica_mg_create", "coarsest level too large for the dense solve", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const bool mixed = o.precision == 1;
    const size_t tsz = mixed ? sizeof(float) : sizeof(double);
    // single-CTA levels: from the first level >= 1 whose remaining hierarchy fits in
    // shared memory and has <= 32*32 cells, or that cannot be tiled
    // per level: u (two colours, each (ny+2) x nx/2 with zero ghost rows), f, ax, 1/d
    // (ny x nx/2 each) and ay ((ny+1) x nx/2), 16-byte aligned arrays
    auto level_arrays = [&](int l, auto&& take) {
        const size_t e = (l < m->nouter - 1) ? tsz : sizeof(double);
        const size_t h = (size_t)m->lv[l].nx / 2, ny = m->lv[l].ny;
        CtaLevel C{};
        for (int c = 0; c < 2; ++c) {
            C.off_u[c] = take(e * (ny + 2) * h);
            C.off_f[c] = take(e * ny * h);
            C.off_ax[c] = take(e * ny * h);
            C.off_ay[c] = take(e * (ny + 1) * h);
            C.off_di[c] = take(e * ny * h);
        }
        return C;
    };
    auto cta_bytes = [&](int from) {
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t r = off; off = (off + bytes + 15) & ~(size_t)15; return (unsigned)r; };
        for (int l = from; l <= m->bottom; ++l) level_arrays(l, take);
        const size_t nb = (size_t)m->lv[m->bottom].nx * m->lv[m->bottom].ny;
        take(sizeof(double) * nb * nb);
        take(sizeof(double) * nb);
        return off;
    };
    int lcta = m->nouter - 1;
    for (int l = 1; l < m->nouter; ++l) {
        const bool tileable = m->lv[l].nx % 16 == 0 && m->lv[l].ny % 16 == 0;
        const size_t n = (size_t)m->lv[l].nx * m->lv[l].ny;
        if (!tileable || (n <= 32 * 32 && cta_bytes(l) <= 226 * 1024)) { lcta = l; break; }
    }
    if (cta_bytes(lcta) > 227 * 1024) {
        delete m;
        lica_set_last_error("lica_mg_create", "coarse levels do not fit in shared memory; use more levels",
                            __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    for (int l = 0; l < lcta; ++l) {
        if (m->lv[l].nx % 16 || m->lv[l].ny % 16) { delete m; return LICA_BAD_ARG; }
    }
    m->lcta = lcta;
    {
        // the cross-level kernels where two or more grid levels lie between level 0 and the
        // single-CTA levels (LICA_MG_CROSS_LEVEL=0 keeps one launch per level)
        const char* ev = std::getenv("LICA_MG_CROSS_LEVEL");
        m->mid = lcta >= 3 && ev && ev[0] == '1' && o.smoother == 0;
        m->yline = o.smoother == 1;
    }
    // shared-memory layout of the single-CTA kernel
    CtaParams& P = m->cp;
    std::memset(&P, 0, sizeof(P));
    P.lcta = lcta; P.lc = m->nouter - 1; P.bottom = m->bottom;
    P.nu1 = o.nu1; P.nu2 = o.nu2; P.ncoarse = o.ncoarse;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off = (off + bytes + 15) & ~(size_t)15; return (unsigned)r; };
    for (int l = lcta; l <= m->bottom; ++l) {
        CtaLevel& C = P.lv[l];
        C = level_arrays(l, take);
        C.nx = m->lv[l].nx; C.ny = m->lv[l].ny; C.half = m->lv[l].nx / 2;
        auto mag = [](unsigned c) { return c > 1 ? (unsigned)((1ull << 32) / c + 1) : 0u; };
        C.mag_h = mag((unsigned)C.half);
        C.mag_nx = mag((unsigned)C.nx);
    }
    const size_t nb = (size_t)m->lv[m->bottom].nx * m->lv[m->bottom].ny;
    P.off_dense = take(sizeof(double) * nb * nb);
    P.off_rhs = take(sizeof(double) * nb);
    m->cta_smem = off;

    auto fail = [&](int code) { lica_mg_destroy(m); return code; };
#define TRY_ALLOC(ptr, bytes)                                                        \
    do {                                                                             \
        cudaError_t _e = cudaMalloc((void**)&(ptr), (bytes));                        \
        if (_e != cudaSuccess) {                                                     \
            lica_set_last_error("cudaMalloc", cudaGetErrorString(_e), __FILE__, __LINE__); \
            return fail(LICA_ERR_NOMEM);                                             \
        }                                                                            \
    } while (0)
    const size_t n0 = (size_t)nx * ny;
    TRY_ALLOC(m->pcg[0], sizeof(double) * n0);
    TRY_ALLOC(m->pcg[1], sizeof(double) * n0);
    TRY_ALLOC(m->xb, sizeof(double) * n0);
    TRY_ALLOC(m->r, tsz * n0);
    TRY_ALLOC(m->zpre, tsz * n0);
    TRY_ALLOC(m->z, tsz * n0);
    if (m->yline) {
        TRY_ALLOC(m->ycp, sizeof(double) * n0);
        TRY_ALLOC(m->ydp, sizeof(double) * n0);
    }
    for (int l = 1; l <= m->bottom; ++l) {
        LevelBuf& L = m->lv[l];
        const size_t n = (size_t)L.nx * L.ny;
        if (l <= lcta || m->yline) {  // the y-line cycle keeps every level in global memory
            TRY_ALLOC(L.u, tsz * n);
            TRY_ALLOC(L.f, tsz * n);
        }
        if (l < lcta) TRY_ALLOC(L.up, tsz * n);
        TRY_ALLOC(L.bx64, sizeof(double) * n);
        TRY_ALLOC(L.by64, sizeof(double) * (n + L.nx));
    }
    for (int l = 0; l <= m->bottom; ++l) {
        LevelBuf& L = m->lv[l];
        const size_t n = (size_t)L.nx * L.ny;
        TRY_ALLOC(L.ax64, sizeof(double) * n);
        TRY_ALLOC(L.ay64, sizeof(double) * (n + L.nx));
        TRY_ALLOC(L.di64, sizeof(double) * n);
    }
    if (mixed) {
        for (int l = 0; l < m->nouter - 1; ++l) {
            LevelBuf& L = m->lv[l];
            const size_t n = (size_t)L.nx * L.ny;
            TRY_ALLOC(L.bx32, sizeof(float) * n);
            TRY_ALLOC(L.by32, sizeof(float) * (n + L.nx));
            TRY_ALLOC(L.ax32, sizeof(float) * n);
            TRY_ALLOC(L.ay32, sizeof(float) * (n + L.nx));
            TRY_ALLOC(L.di32, sizeof(float) * n);
        }
    }
    const size_t ntiles = (size_t)(nx / 16) * (ny / 16);  // the most blocks of any level-0 grid kernel
    TRY_ALLOC(m->partials, sizeof(double) * 2 * ntiles);
    TRY_ALLOC(m->st, sizeof(State));
    {
        const size_t nb = (size_t)m->lv[m->bottom].nx * m->lv[m->bottom].ny;
        TRY_ALLOC(m->dense_lu, sizeof(double) * nb * nb);
        P.glu = m->dense_lu;
    }
    {
        cudaError_t e = cudaMallocHost((void**)&m->st_host, sizeof(State));
        if (e != cudaSuccess) return fail(LICA_ERR_NOMEM);
    }
#undef TRY_ALLOC
    {
        cudaError_t e1 = cudaFuncSetAttribute(k_xupdate<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)xupdate_smem());
        cudaError_t e2 = cudaFuncSetAttribute(k_xupdate<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)xupdate_smem());
        cudaError_t e3 = cudaFuncSetAttribute(k_pupdate<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)pupdate_smem<double>());
        cudaError_t e4 = cudaFuncSetAttribute(k_pupdate<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)pupdate_smem<float>());
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess) {
            lica_set_last_error("cudaFuncSetAttribute(CG kernels)", "failed", __FILE__, __LINE__);
            return fail(LICA_ERR_CUDA);
        }
    }
    // The dynamic shared-memory cap is per function, shared by every solver instance: set it
    // to the device's opt-in maximum (an instance with a smaller coarse level must not lower
    // it under another instance's launches), and check this instance's need against it.
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess && m->cta_smem > (size_t)optin) {
        lica_set_last_error("lica_mg_create", "coarse levels exceed the shared memory of one CTA", __FILE__, __LINE__);
        return fail(LICA_BAD_ARG);
    }
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_cta<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_cta<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) {
        lica_set_last_error("cudaFuncSetAttribute(k_cta)", cudaGetErrorString(e), __FILE__, __LINE__);
        return fail(LICA_ERR_CUDA);
    }
    e = cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        lica_set_last_error("cudaDeviceGetAttribute", cudaGetErrorString(e), __FILE__, __LINE__);
        return fail(LICA_ERR_CUDA);
    }
    m->lv[0].u = m->zpre;
    m->lv[0].up = m->z;
    m->lv[0].f = m->r;
    {
        // the TMA CG kernels: level 0 in 32 x 32 tiles, two tile columns, a tile per SM
        const int ntx = nx / CG_TS, nty = ny / CG_TS;
        if (nx % CG_TS == 0 && ny % CG_TS == 0 && ntx >= 2 && ntx * nty >= m->nsm) {
            LevelBuf& L0 = m->lv[0];
            const bool f32 = is_mixed(m);
            int st;
            CgMaps& M = m->cgm;
            if ((st = tm_map(&M.p[0], m->pcg[0], false, nx, ny, CG_BW, CG_BH)) ||
                (st = tm_map(&M.pw[0], m->pcg[0], false, nx, ny, CG_WW, CG_BH)) ||
                (st = tm_map(&M.p[1], m->pcg[1], false, nx, ny, CG_BW, CG_BH)) ||
                (st = tm_map(&M.pw[1], m->pcg[1], false, nx, ny, CG_WW, CG_BH)) ||
                (st = tm_map(&M.x[1], m->xb, false, nx, ny, CG_BW, CG_BH)) ||
                (st = tm_map(&M.xw[1], m->xb, false, nx, ny, CG_WW, CG_BH)) ||
                (st = tm_map(&M.z, m->z, f32, nx, ny, CG_BW, CG_BH)) ||
                (st = tm_map(&M.zw, m->z, f32, nx, ny, CG_WW, CG_BH)) ||
                (st = tm_map(&M.ax, L0.ax64, false, nx, ny, CG_BW, CG_BH)) ||
                (st = tm_map(&M.axw, L0.ax64, false, nx, ny, CG_WW, CG_BH)) ||
                (st = tm_map(&M.ay, L0.ay64, false, nx, ny + 1, CG_BW, CG_BH)))
                return fail(st);
            cudaError_t ce = cudaFuncSetAttribute(k_cg_tma<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  CgLayout<double, false>::BYTES);
            if (ce == cudaSuccess) ce = cudaFuncSetAttribute(k_cg_tma<float, false>,
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             CgLayout<float, false>::BYTES);
            if (ce == cudaSuccess) ce = cudaFuncSetAttribute(k_cg_tma<double, true>,
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             CgLayout<double, true>::BYTES);
            if (ce == cudaSuccess) ce = cudaFuncSetAttribute(k_cg_tma<float, true>,
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             CgLayout<float, true>::BYTES);
            if (ce != cudaSuccess) {
                lica_set_last_error("cudaFuncSetAttribute(k_cg_tma)", cudaGetErrorString(ce), __FILE__, __LINE__);
                return fail(LICA_ERR_CUDA);
            }
            m->cg_tma = true;
        }
    }
    *out = m;
    return LICA_OK;
}

int lica_mg_destroy(lica_mg* m) {
    if (!m) return LICA_OK;
    if (m->gcur.exec) cudaGraphExecDestroy(m->gcur.exec);
    if (m->galt.exec) cudaGraphExecDestroy(m->galt.exec);
    for (auto& pe : m->prof_pending) {
        cudaEventDestroy(pe.second.first);
        cudaEventDestroy(pe.second.second);
    }
    for (auto e : m->event_pool) cudaEventDestroy(e);
    for (size_t l = 1; l < m->lv.size(); ++l) {
        cudaFree(m->lv[l].u);
        cudaFree(m->lv[l].up);
        cudaFree(m->lv[l].f);
        cudaFree(m->lv[l].bx64);
        cudaFree(m->lv[l].by64);
    }
    for (auto& L : m->lv) {
        cudaFree(L.bx32);
        cudaFree(L.by32);
        cudaFree(L.ax32);
        cudaFree(L.ay32);
        cudaFree(L.ax64);
        cudaFree(L.ay64);
        cudaFree(L.di64);
        cudaFree(L.di32);
    }
    cudaFree(m->pcg[0]);
    cudaFree(m->pcg[1]);
    cudaFree(m->xb);
    cudaFree(m->r);
    cudaFree(m->dense_lu);
    cudaFree(m->zpre);
    cudaFree(m->z);
    cudaFree(m->ycp);
    cudaFree(m->ydp);
    cudaFree(m->partials);
    cudaFree(m->st);
    if (m->st_host) cudaFreeHost(m->st_host);
    if (m->b_states) cudaFreeHost(m->b_states);
    cudaFree(m->d_p);
    cudaFree(m->d_f);
    cudaFree(m->d_bx);
    cudaFree(m->d_by);
    for (int b = 0; b < 2; ++b) {
        cudaFree(m->b_in[b]);
        cudaFree(m->b_out[b]);
        cudaEvent_t evs[] = {m->b_ev_in[b], m->b_ev_used[b], m->b_ev_solved[b], m->b_ev_out[b]};
        for (cudaEvent_t e : evs)
            if (e) cudaEventDestroy(e);
    }
    if (m->b_up) cudaStreamDestroy(m->b_up);
    if (m->b_down) cudaStreamDestroy(m->b_down);
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
    if (m->cap_stream) cudaStreamDestroy(m->cap_stream);
    delete m;
    return LICA_OK;
}

int lica_mg_solve_device(lica_mg* m, double* p, const double* f, const double* bx, const double* by, double rtol,
                         int32_t max_iters, lica_mg_result* res, void* stream) {
    return solve_impl(m, p, f, bx, by, rtol, max_iters, res, (cudaStream_t)stream);
}

int lica_mg_solve_host(lica_mg* m, double* p, const double* f, const double* bx, const double* by, double rtol,
                       int32_t max_iters, lica_mg_result* res, void* stream) {
    if (!m || !p || !f || !bx || !by) return LICA_BAD_ARG;
    const size_t n = (size_t)m->nx * m->ny, nb = n + m->nx;
    if (!stream && !m->own_stream) LICA_CUDA_TRY(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking));
    if (!m->d_p) {
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_p, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_f, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_bx, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_by, sizeof(double) * nb));
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : m->own_stream;
    LICA_CUDA_TRY(cudaMemcpyAsync(m->d_p, p, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(m->d_f, f, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(m->d_bx, bx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(m->d_by, by, sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    int st = solve_impl(m, m->d_p, m->d_f, m->d_bx, m->d_by, rtol, max_iters, res, s);
    if (st == LICA_ERR_CUDA || st == LICA_BAD_ARG) return st;
    LICA_CUDA_TRY(cudaMemcpyAsync(p, m->d_p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    return st;
}

int lica_mg_solve_host_batch(lica_mg* m, int32_t count, double* const* p, const double* const* f,
                             const double* const* bx, const double* const* by, double rtol, int32_t max_iters,
                             lica_mg_result* res) {
    if (!m || count < 0 || (count > 0 && (!p || !f || !bx || !by || !res))) return LICA_BAD_ARG;
    for (int32_t k = 0; k < count; ++k)
        if (!p[k] || !f[k] || !bx[k] || !by[k]) return LICA_BAD_ARG;
    if (count == 0) return LICA_OK;
    const size_t n = (size_t)m->nx * m->ny, nb = n + m->nx, nin = 3 * n + nb;
    if (!m->own_stream) LICA_CUDA_TRY(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking));
    if (!m->d_p) {
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_p, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_f, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_bx, sizeof(double) * n));
        LICA_CUDA_TRY(cudaMalloc((void**)&m->d_by, sizeof(double) * nb));
    }
    if (!m->b_up) {
        LICA_CUDA_TRY(cudaStreamCreateWithFlags(&m->b_up, cudaStreamNonBlocking));
        LICA_CUDA_TRY(cudaStreamCreateWithFlags(&m->b_down, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            LICA_CUDA_TRY(cudaMalloc((void**)&m->b_in[b], sizeof(double) * nin));
            LICA_CUDA_TRY(cudaMalloc((void**)&m->b_out[b], sizeof(double) * n));
            cudaEvent_t* evs[] = {&m->b_ev_in[b], &m->b_ev_used[b], &m->b_ev_solved[b], &m->b_ev_out[b]};
            for (cudaEvent_t* e : evs) LICA_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            // nothing in flight yet: the first waits on these events pass
            LICA_CUDA_TRY(cudaEventRecord(m->b_ev_used[b], m->b_up));
            LICA_CUDA_TRY(cudaEventRecord(m->b_ev_out[b], m->b_down));
        }
    }
    cudaStream_t s = m->own_stream;
    // With graphs the host never waits inside the loop: each solve's final state is copied to
    // its own pinned slot and read after the last download.
    const bool async = m->o.use_graph && !m->profile;
    if (async && m->b_states_cap < count) {
        if (m->b_states) cudaFreeHost(m->b_states);
        m->b_states = nullptr;
        m->b_states_cap = 0;
        LICA_CUDA_TRY(cudaMallocHost((void**)&m->b_states, sizeof(State) * (size_t)count));
        m->b_states_cap = count;
    }
    if (!(rtol >= 0.0) || max_iters < 0) return LICA_BAD_ARG;
    // upload of system k into input staging k % 2 once the solve of k - 2 has consumed it
    auto upload = [&](int32_t k) -> int {
        const int b = k & 1;
        double* in = m->b_in[b];
        LICA_CUDA_TRY(cudaStreamWaitEvent(m->b_up, m->b_ev_used[b], 0));
        LICA_CUDA_TRY(cudaMemcpyAsync(in, p[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
        LICA_CUDA_TRY(cudaMemcpyAsync(in + n, f[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
        LICA_CUDA_TRY(cudaMemcpyAsync(in + 2 * n, bx[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
        LICA_CUDA_TRY(cudaMemcpyAsync(in + 3 * n, by[k], sizeof(double) * nb, cudaMemcpyHostToDevice, m->b_up));
        LICA_CUDA_TRY(cudaEventRecord(m->b_ev_in[b], m->b_up));
        return LICA_OK;
    };
    int st, worst = LICA_OK;
    if (async) {
        // Each system is solved where it was uploaded (its staging buffer holds p, f, bx, by;
        // the solve's graph is cached for both buffers) and downloaded from there: no copies
        // between buffers on the device, which would also push the solver's working set out
        // of L2.  Upload k waits for the download of k - 2 from the same buffer, which follows
        // its solve.
        auto upload_in_place = [&](int32_t k) -> int {
            const int b = k & 1;
            double* in = m->b_in[b];
            LICA_CUDA_TRY(cudaStreamWaitEvent(m->b_up, m->b_ev_out[b], 0));
            LICA_CUDA_TRY(cudaMemcpyAsync(in, p[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
            LICA_CUDA_TRY(cudaMemcpyAsync(in + n, f[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
            LICA_CUDA_TRY(cudaMemcpyAsync(in + 2 * n, bx[k], sizeof(double) * n, cudaMemcpyHostToDevice, m->b_up));
            LICA_CUDA_TRY(cudaMemcpyAsync(in + 3 * n, by[k], sizeof(double) * nb, cudaMemcpyHostToDevice, m->b_up));
            LICA_CUDA_TRY(cudaEventRecord(m->b_ev_in[b], m->b_up));
            return LICA_OK;
        };
        if ((st = upload_in_place(0))) return st;
        for (int32_t k = 0; k < count; ++k) {
            const int b = k & 1;
            if (k + 1 < count && (st = upload_in_place(k + 1))) return st;
            double* in = m->b_in[b];
            LICA_CUDA_TRY(cudaStreamWaitEvent(s, m->b_ev_in[b], 0));
            if ((st = graph_launch(m, in, in + n, in + 2 * n, in + 3 * n, rtol, max_iters, s))) return st;
            LICA_CUDA_TRY(cudaMemcpyAsync(&m->b_states[k], m->st, sizeof(State), cudaMemcpyDeviceToHost, s));
            LICA_CUDA_TRY(cudaEventRecord(m->b_ev_solved[b], s));
            LICA_CUDA_TRY(cudaStreamWaitEvent(m->b_down, m->b_ev_solved[b], 0));
            LICA_CUDA_TRY(cudaMemcpyAsync(p[k], in, sizeof(double) * n, cudaMemcpyDeviceToHost, m->b_down));
            LICA_CUDA_TRY(cudaEventRecord(m->b_ev_out[b], m->b_down));
        }
    } else {
    if ((st = upload(0))) return st;
    for (int32_t k = 0; k < count; ++k) {
        const int b = k & 1;
        // the next system's upload runs during this solve
        if (k + 1 < count && (st = upload(k + 1))) return st;
        double* in = m->b_in[b];
        LICA_CUDA_TRY(cudaStreamWaitEvent(s, m->b_ev_in[b], 0));
        LICA_CUDA_TRY(cudaMemcpyAsync(m->d_p, in, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        LICA_CUDA_TRY(cudaMemcpyAsync(m->d_f, in + n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        LICA_CUDA_TRY(cudaMemcpyAsync(m->d_bx, in + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        LICA_CUDA_TRY(cudaMemcpyAsync(m->d_by, in + 3 * n, sizeof(double) * nb, cudaMemcpyDeviceToDevice, s));
        LICA_CUDA_TRY(cudaEventRecord(m->b_ev_used[b], s));
        if (async) {
            if ((st = graph_launch(m, m->d_p, m->d_f, m->d_bx, m->d_by, rtol, max_iters, s))) return st;
            LICA_CUDA_TRY(cudaMemcpyAsync(&m->b_states[k], m->st, sizeof(State), cudaMemcpyDeviceToHost, s));
        } else {
            st = solve_impl(m, m->d_p, m->d_f, m->d_bx, m->d_by, rtol, max_iters, &res[k], s);
            if (st == LICA_ERR_CUDA || st == LICA_BAD_ARG) return st;
            if (st != LICA_OK && worst == LICA_OK) worst = st;
        }
        // the result leaves through output staging k % 2 (free once the download of k - 2 ended)
        LICA_CUDA_TRY(cudaStreamWaitEvent(s, m->b_ev_out[b], 0));
        LICA_CUDA_TRY(cudaMemcpyAsync(m->b_out[b], m->d_p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        LICA_CUDA_TRY(cudaEventRecord(m->b_ev_solved[b], s));
        LICA_CUDA_TRY(cudaStreamWaitEvent(m->b_down, m->b_ev_solved[b], 0));
        LICA_CUDA_TRY(cudaMemcpyAsync(p[k], m->b_out[b], sizeof(double) * n, cudaMemcpyDeviceToHost, m->b_down));
        LICA_CUDA_TRY(cudaEventRecord(m->b_ev_out[b], m->b_down));
    }
    }
    LICA_CUDA_TRY(cudaStreamSynchronize(m->b_down));
    LICA_CUDA_TRY(cudaStreamSynchronize(m->b_up));
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    if (async) {
        for (int32_t k = 0; k < count; ++k) {
            const State& S = m->b_states[k];
            if (S.kerr) {
                lica_set_last_error("lica_mg_solve_host_batch", "a bounded wait inside a kernel ran out", __FILE__,
                                    __LINE__);
                return LICA_ERR_CUDA;
            }
            res[k].iterations = S.it;
            res[k].status = S.status;
            res[k].rel_residual = S.rel;
            lica_count_launches(m->setup_nodes + (int64_t)(S.it + S.back) * m->body_nodes);
            if (S.status != LICA_OK && worst == LICA_OK) worst = S.status;
        }
    }
    return worst;
}

int lica_mg_precond_device(lica_mg* m, double* z, const double* r, const double* bx, const double* by,
                           void* stream) {
    if (!m || !z || !r || !bx || !by) return LICA_BAD_ARG;
    if (!aligned16(z, r, bx, by)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = setup_beta(m, bx, by, s))) return st;
    const size_t n = (size_t)m->nx * m->ny;
    m->lv[0].u = m->zpre;
    m->lv[0].up = m->z;
    m->lv[0].f = m->r;
    k_init_state<<<1, 1, 0, s>>>(m->st, 0.0, 0);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    if (is_mixed(m)) {
        k_to_float<<<1184, 256, 0, s>>>(r, (float*)m->r, n);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(1);
        if ((st = vcycle<float>(m, s))) return st;
        k_widen<<<1184, 256, 0, s>>>((const float*)m->z, z, n);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(1);
    } else {
        LICA_CUDA_TRY(cudaMemcpyAsync(m->r, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        if ((st = run_vcycle(m, s))) return st;
        LICA_CUDA_TRY(cudaMemcpyAsync(z, m->z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    return LICA_OK;
}

int lica_mg_profile(lica_mg* m, int32_t enable) {
    if (!m) return LICA_BAD_ARG;
    m->profile = enable != 0;
    for (int k = 0; k < LICA_MG_NCLASS; ++k) {
        m->prof_ms[k] = 0.0;
        m->prof_n[k] = 0;
    }
    return LICA_OK;
}

int lica_mg_profile_read(lica_mg* m, int32_t kernel_class, double* total_ms, int64_t* launches) {
    if (!m || kernel_class < 0 || kernel_class >= LICA_MG_NCLASS || !total_ms || !launches) return LICA_BAD_ARG;
    *total_ms = m->prof_ms[kernel_class];
    *launches = m->prof_n[kernel_class];
    return LICA_OK;
}

int lica_mg_apply_device(lica_mg* m, double* out, const double* u, const double* bx, const double* by,
                         void* stream) {
    if (!m || !out || !u || !bx || !by || out == u) return LICA_BAD_ARG;  // out must not alias u (halo reads)
    if (!aligned16(out, u, bx, by)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = setup_beta(m, bx, by, s))) return st;
    const LevelBuf& L = m->lv[0];
    k_apply<<<dim3(L.nx / TX, L.ny / TY), NT, 0, s>>>(out, u, L.ax64, L.ay64, L.nx, L.ny);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    return LICA_OK;
}

}  // extern "C"
