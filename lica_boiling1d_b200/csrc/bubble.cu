// Bubble statistics of several level sets on a 3-D grid: BUBBLE_TRACKING (two_phase.f:
// 6321-6555), BUBBLE_EIGENV (6558-6705) and Jacobi_bub (two_phase.f:19-97).
//
// The reference sums each level set twice over the whole field -- once for the volume,
// centroid and velocity, once more for the second moment about the centroid.  Here one
// pass reads each PSI_TMP field once: every gas cell (PSI_TMP != 1) enters a weighted
// Welford update of the running centroid and co-moments, and the per-thread states are
// merged by Chan's pairwise rule (warp tree, block tree, then the blocks in index order by
// the last block to finish), so the result is the same on every run.  Velocity is read
// only at gas cells.  The z coordinate is carried both as ZP and as the periodic shift
// (ZP + ZL for ZP <= ZL/2) because IZ_PERIODIC -- gas in the top plane -- is known only
// at the end; the finish picks one.
#include "common.cuh"

#include <algorithm>
#include <cmath>

extern "C" void lica_count_launches(int64_t n);

namespace {

constexpr int kBubThreads = 256;
constexpr int kBubWarps = kBubThreads / 32;
constexpr int kBubMaxBlocks = 148 * 2;  // one wave of a level set at two blocks per SM

// Running state of one level set's gas volume: weight W, means of x, y, z and the shifted
// z (s), co-moments sum w (a - mean_a)(b - mean_b), velocity sums, IZ_PERIODIC.
struct Mom {
    double w, mx, my, mz, ms;
    double cxx, cyy, cxy, czz, cyz, czx, css, cys, csx;
    double su, sv, sw;
    double iz;
};
constexpr int kMomN = 18;

__device__ __forceinline__ void mom_zero(Mom& a) {
    double* p = &a.w;
#pragma unroll
    for (int q = 0; q < kMomN; ++q) p[q] = 0.0;
}

// Weighted Welford update with one cell of weight vf at (x, y, z, s).
__device__ __forceinline__ void mom_add(Mom& a, double vf, double x, double y, double z, double s) {
    const double wn = a.w + vf;
    const double r = (wn != 0.0) ? vf / wn : 0.0;
    const double dx = x - a.mx, dy = y - a.my, dz = z - a.mz, ds = s - a.ms;
    a.mx += dx * r;
    a.my += dy * r;
    a.mz += dz * r;
    a.ms += ds * r;
    const double ex = x - a.mx, ey = y - a.my, ez = z - a.mz, es = s - a.ms;
    a.cxx += vf * dx * ex;
    a.cyy += vf * dy * ey;
    a.cxy += vf * dx * ey;
    a.czz += vf * dz * ez;
    a.cyz += vf * dy * ez;
    a.czx += vf * dz * ex;
    a.css += vf * ds * es;
    a.cys += vf * dy * es;
    a.csx += vf * ds * ex;
    a.w = wn;
}

// Chan's rule: a <- a merged with b.
__device__ __forceinline__ void mom_merge(Mom& a, const Mom& b) {
    if (b.w != 0.0) {
        if (a.w == 0.0) {
            const double su = a.su + b.su, sv = a.sv + b.sv, sw = a.sw + b.sw, iz = fmax(a.iz, b.iz);
            a = b;
            a.su = su;
            a.sv = sv;
            a.sw = sw;
            a.iz = iz;
            return;
        }
        const double wn = a.w + b.w;
        const double f = b.w / wn, g = a.w * f;
        const double dx = b.mx - a.mx, dy = b.my - a.my, dz = b.mz - a.mz, ds = b.ms - a.ms;
        a.cxx += b.cxx + dx * dx * g;
        a.cyy += b.cyy + dy * dy * g;
        a.cxy += b.cxy + dx * dy * g;
        a.czz += b.czz + dz * dz * g;
        a.cyz += b.cyz + dy * dz * g;
        a.czx += b.czx + dz * dx * g;
        a.css += b.css + ds * ds * g;
        a.cys += b.cys + dy * ds * g;
        a.csx += b.csx + ds * dx * g;
        a.mx += dx * f;
        a.my += dy * f;
        a.mz += dz * f;
        a.ms += ds * f;
        a.w = wn;
    }
    a.su += b.su;
    a.sv += b.sv;
    a.sw += b.sw;
    a.iz = fmax(a.iz, b.iz);
}

__device__ __forceinline__ void mom_shfl_down(Mom& dst, const Mom& src, int off) {
    const double* s = &src.w;
    double* d = &dst.w;
#pragma unroll
    for (int q = 0; q < kMomN; ++q) d[q] = __shfl_down_sync(0xffffffffu, s[q], off);
}

// Jacobi_bub (two_phase.f:19-97), cyclic Jacobi rotations of a symmetric 3x3 matrix with
// the threshold bar = b2 / 2n^2 on the squared off-diagonal entries; a[r][c] is the
// Fortran A(r+1, c+1), the eigenvalues end on the diagonal, column i of x is the
// eigenvector of a[i][i].  The steps are those of the published method, kept in its order
// so the eigenvectors come out with the same signs and order as the reference's.
__device__ void jacobi3(double a[3][3], double x[3][3], double abserr) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) x[i][j] = (i == j) ? 1.0 : 0.0;
    double b2 = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (i != j) b2 = b2 + a[i][j] * a[i][j];
    if (b2 <= abserr) return;
    double bar = 0.5 * b2 / 9.0;
    for (int it = 0; it < 500; ++it) {
        for (int i = 0; i < 2; ++i) {
            for (int j = i + 1; j < 3; ++j) {
                if (a[j][i] * a[j][i] <= bar) continue;
                b2 = b2 - 2.0 * a[j][i] * a[j][i];
                bar = 0.5 * b2 / 9.0;
                const double beta = (a[j][j] - a[i][i]) / (2.0 * a[j][i]);
                const double coeff = 0.5 * beta / sqrt(1.0 + beta * beta);
                const double s = sqrt(fmax(0.5 + coeff, 0.0));
                const double c = sqrt(fmax(0.5 - coeff, 0.0));
                for (int k = 0; k < 3; ++k) {
                    const double cs = c * a[i][k] + s * a[j][k];
                    const double sc = -s * a[i][k] + c * a[j][k];
                    a[i][k] = cs;
                    a[j][k] = sc;
                }
                for (int k = 0; k < 3; ++k) {
                    double cs = c * a[k][i] + s * a[k][j];
                    double sc = -s * a[k][i] + c * a[k][j];
                    a[k][i] = cs;
                    a[k][j] = sc;
                    cs = c * x[k][i] + s * x[k][j];
                    sc = -s * x[k][i] + c * x[k][j];
                    x[k][i] = cs;
                    x[k][j] = sc;
                }
            }
        }
        if (b2 <= abserr) return;
    }
}

struct BubArgs {
    int n1m, n2m, n3m, ipx, ipy, ipz;
    double zl;
    const double *sdx, *sdy, *sdz, *xp, *yp, *zp;
    const double *psi, *u, *v, *w;
    long long fsize;  // doubles per field, (n1m+2)(n2m+2)(n3m+2)
    int llvs0, icacy;
    double time;
    double* part;        // [nlvs][gridDim.x][kMomN]
    unsigned* counters;  // [nlvs], zero before the launch, reset by the last block
    lica_bub_record* out;
};

// The end of BUBBLE_TRACKING and BUBBLE_EIGENV for one level set from its merged state.
__device__ void bub_finish(const BubArgs& A, const Mom& m, int l) {
    const bool shift = A.ipz == 1 && m.iz != 0.0;
    const double vol = m.w;
    double xx = 0.0, yy = 0.0, zz = 0.0, uu = 0.0, vv = 0.0, ww = 0.0;
    if (vol != 0.0) {
        const double voli = 1.0 / vol;
        xx = m.mx;
        yy = m.my;
        zz = shift ? m.ms : m.mz;
        uu = m.su * voli;
        vv = m.sv * voli;
        ww = m.sw * voli;
    }
    lica_bub_record r;
    r.time = A.time;
    r.llvs = A.llvs0 + l;
    double xc = xx, yc = yy, zc = zz;
    if (A.icacy == 2) {
        const double pi = acos(-1.0);
        const double rr = sqrt(xx * xx + yy * yy);
        double tt = atan(yy / xx);
        if (xx <= 0.0 && yy >= 0.0)
            tt = tt + pi;
        else if (xx <= 0.0 && yy <= 0.0)
            tt = tt + pi;
        else if (xx >= 0.0 && yy <= 0.0)
            tt = tt + 2.0 * pi;
        const double ur = uu * cos(tt) + vv * sin(tt);
        const double ut = -uu * sin(tt) + vv * cos(tt);
        xc = rr * cos(tt);
        yc = rr * sin(tt);
        r.col[0] = rr;
        r.col[1] = tt;
        r.col[3] = ur;
        r.col[4] = ut;
    } else {
        r.col[0] = xx;
        r.col[1] = yy;
        r.col[3] = uu;
        r.col[4] = vv;
    }
    r.col[2] = zz;
    r.col[5] = ww;
    // second moment about (xc, yc, zc): the co-moments about the mean plus W (mean - c)^2
    double a[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    if (vol != 0.0) {
        const double voli = 1.0 / vol;
        const double mz = shift ? m.ms : m.mz;
        const double czz = shift ? m.css : m.czz, cyz = shift ? m.cys : m.cyz, czx = shift ? m.csx : m.czx;
        const double dx = m.mx - xc, dy = m.my - yc, dz = mz - zc;
        a[0][0] = (m.cxx + vol * dx * dx) * voli;
        a[1][1] = (m.cyy + vol * dy * dy) * voli;
        a[2][2] = (czz + vol * dz * dz) * voli;
        a[0][1] = (m.cxy + vol * dx * dy) * voli;
        a[1][2] = (cyz + vol * dy * dz) * voli;
        a[2][0] = (czx + vol * dz * dx) * voli;
    }
    a[1][0] = a[0][1];
    a[2][1] = a[1][2];
    a[0][2] = a[2][0];
    double e[3][3];
    jacobi3(a, e, 1.0e-12);
    double ar;
    int small;
    if (a[0][0] >= a[1][1]) {
        if (a[0][0] >= a[2][2]) {
            if (a[1][1] >= a[2][2]) {
                ar = sqrt(a[0][0] / a[2][2]);
                small = 2;
            } else {
                ar = sqrt(a[0][0] / a[1][1]);
                small = 1;
            }
        } else {
            ar = sqrt(a[2][2] / a[1][1]);
            small = 1;
        }
    } else {
        if (a[1][1] >= a[2][2]) {
            if (a[0][0] >= a[2][2]) {
                ar = sqrt(a[1][1] / a[2][2]);
                small = 2;
            } else {
                ar = sqrt(a[1][1] / a[0][0]);
                small = 0;
            }
        } else {
            ar = sqrt(a[2][2] / a[0][0]);
            small = 0;
        }
    }
    const double denom = 1.0 / sqrt(e[0][small] * e[0][small] + e[1][small] * e[1][small] +
                                    e[2][small] * e[2][small]);
    double ang1 = acos(e[0][small] * denom) * 57.295779513082321;
    double ang2 = acos(e[2][small] * denom) * 57.295779513082321;
    if (ang1 >= 90.0) ang1 = 180.0 - ang1;
    if (ang2 >= 90.0) ang2 = 180.0 - ang2;
    r.col[6] = ar;
    r.col[7] = ang1;
    r.col[8] = ang2;
    r.vel[0] = uu;
    r.vel[1] = vv;
    r.vel[2] = ww;
    r.vol = vol;
    r.ami[0] = a[0][0];
    r.ami[1] = a[1][1];
    r.ami[2] = a[2][2];
    r.iz_periodic = m.iz != 0.0 ? 1 : 0;
    A.out[l] = r;
}

// One block row of gridDim.x blocks per level set (blockIdx.y).  The level set's field is
// read as one flat stream, ghost cells included, in 16-byte pairs aligned to the address:
// thread t of the block row takes pairs t, t + T, t + 2T, ... (T threads in the row), sixteen
// at a time, so a warp's loads are contiguous and a lane keeps sixteen 16-byte loads in flight.
// Only a value other than 1 -- a gas cell, or a ghost cell the caller left unset -- is located
// (two divisions) and, if it is inside the grid, entered; a lone element left at either end
// of the stream is a corner ghost cell.
constexpr int kPairsInFlight = 16;

__device__ __forceinline__ void bub_cell(const BubArgs& A, Mom& m, int i, int j, int k, double ps) {
    const long long p1 = A.n1m + 2, p2 = (long long)(A.n2m + 2) * p1;
    const long long base = j * p1 + k * p2, c = base + i;
    const double z = A.zp[k];
    const double s = (z <= 0.5 * A.zl) ? z + A.zl : z;
    const int in = (i == A.n1m) ? (A.ipx ? 1 : A.n1m + 1) : i + 1;
    const int jn = (j == A.n2m) ? (A.ipy ? 1 : A.n2m + 1) : j + 1;
    const int kn = (k == A.n3m) ? (A.ipz ? 1 : A.n3m + 1) : k + 1;
    const double vf = (1.0 - ps) * A.sdx[i] * A.sdy[j] * A.sdz[k];
    mom_add(m, vf, A.xp[i], A.yp[j], z, s);
    m.su += 0.5 * (A.u[c] + A.u[base + in]) * vf;
    m.sv += 0.5 * (A.v[c] + A.v[i + jn * p1 + k * p2]) * vf;
    m.sw += 0.5 * (A.w[c] + A.w[i + j * p1 + kn * p2]) * vf;
    if (k == A.n3m) m.iz = 1.0;
}

__device__ __forceinline__ void mom_load(Mom& a, const double* src) {
    double* p = &a.w;
#pragma unroll
    for (int q = 0; q < kMomN; ++q) p[q] = src[q];
}

__device__ __forceinline__ void mom_store(double* dst, const Mom& a) {
    const double* p = &a.w;
#pragma unroll
    for (int q = 0; q < kMomN; ++q) dst[q] = p[q];
}

// Merge of the block's threads in a fixed order: the warp trees, then warp 0's tree over the
// warps' results; valid in thread 0.
__device__ __forceinline__ void block_merge(Mom& m, double (*sh)[kMomN]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Mom o;
    for (int off = 16; off > 0; off >>= 1) {
        mom_shfl_down(o, m, off);
        if (lane + off < 32) mom_merge(m, o);
    }
    __syncthreads();
    if (lane == 0) mom_store(sh[warp], m);
    __syncthreads();
    if (warp == 0) {
        if (lane < kBubWarps)
            mom_load(m, sh[lane]);
        else
            mom_zero(m);
        for (int off = kBubWarps / 2; off > 0; off >>= 1) {
            mom_shfl_down(o, m, off);
            if (lane + off < kBubWarps) mom_merge(m, o);
        }
    }
}

constexpr size_t kBubSmem = (size_t)2 * kPairsInFlight * kBubThreads * sizeof(double);

__global__ void __launch_bounds__(kBubThreads, 2) k_bubble(const __grid_constant__ BubArgs A) {
    const int l = blockIdx.y;
    const double* __restrict__ psi = A.psi + (long long)l * A.fsize;
    // elements e with (e + par) even start a 16-byte aligned pair (psi is 8-byte aligned)
    const int par = (int)((reinterpret_cast<uintptr_t>(psi) >> 3) & 1);
    Mom m;
    mom_zero(m);
    const int p1 = A.n1m + 2, p2 = (A.n2m + 2) * p1;
    const int npairs = (int)((A.fsize - par) >> 1);
    const int T = gridDim.x * kBubThreads;
    extern __shared__ double dyn[];  // kBubSmem: a pair batch's values while its gas cells are entered
    double (*gv)[kBubThreads] = reinterpret_cast<double (*)[kBubThreads]>(dyn);
    for (int p0 = blockIdx.x * kBubThreads + threadIdx.x; p0 < npairs; p0 += T * kPairsInFlight) {
        double2 ps[kPairsInFlight];
#pragma unroll
        for (int q = 0; q < kPairsInFlight; ++q) {
            const int p = p0 + q * T;
            ps[q] = (p < npairs) ? __ldcs(reinterpret_cast<const double2*>(psi + par + 2 * p))
                                 : make_double2(1.0, 1.0);
        }
        unsigned hit = 0;  // bit 2q (+1): the first (second) value of pair q is not 1
#pragma unroll
        for (int q = 0; q < kPairsInFlight; ++q) {
            if (ps[q].x != 1.0) hit |= 1u << (2 * q);
            if (ps[q].y != 1.0) hit |= 2u << (2 * q);
        }
        if (hit) {
            // park the values in shared memory, so that the loads' registers are free while
            // the gas cells update the running state
#pragma unroll
            for (int q = 0; q < kPairsInFlight; ++q) {
                gv[2 * q][threadIdx.x] = ps[q].x;
                gv[2 * q + 1][threadIdx.x] = ps[q].y;
            }
            do {
                const int bit = __ffs(hit) - 1;
                hit &= hit - 1;
                const int e = par + 2 * (p0 + (bit >> 1) * T) + (bit & 1);
                const int k = e / p2, r = e - k * p2, j = r / p1, i = r - j * p1;
                if (i >= 1 && i <= A.n1m && j >= 1 && j <= A.n2m && k >= 1 && k <= A.n3m)
                    bub_cell(A, m, i, j, k, gv[bit][threadIdx.x]);
            } while (hit);
        }
    }
    __shared__ double sh[kBubWarps][kMomN];
    __shared__ bool last;
    block_merge(m, sh);
    double* part = A.part + (long long)l * gridDim.x * kMomN;
    if (threadIdx.x == 0) {
        mom_store(part + blockIdx.x * kMomN, m);
        __threadfence();
        last = atomicAdd(&A.counters[l], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block: thread t merges blocks t, t + kBubThreads, ... in order, then the block tree
    mom_zero(m);
    for (unsigned b = threadIdx.x; b < gridDim.x; b += kBubThreads) {
        Mom t;
        const volatile double* src = part + b * kMomN;
        double* d = &t.w;
        for (int q = 0; q < kMomN; ++q) d[q] = src[q];
        mom_merge(m, t);
    }
    block_merge(m, sh);
    if (threadIdx.x == 0) {
        A.counters[l] = 0u;
        bub_finish(A, m, l);
    }
}

}  // namespace

struct lica_bub_geo {
    int n1m, n2m, n3m, ipx, ipy, ipz;
    double zl;
    int max_lvs, nblk;
    bool smem_set;       // k_bubble's dynamic shared-memory limit raised
    double* geom;        // sdx | sdy | sdz | xp | yp | zp, each direction's n+2 entries
    double* part;        // [max_lvs][nblk][kMomN]
    unsigned* counters;  // [max_lvs]
};

extern "C" {

int lica_gpu_bubble_grid_create(lica_bub_geo** out, const lica_bub_grid* g, int32_t max_lvs) {
    if (!out || !g || g->n1m < 1 || g->n2m < 1 || g->n3m < 1 || max_lvs < 1 || max_lvs > 65535 || !g->sdx || !g->sdy || !g->sdz ||
        !g->xp || !g->yp || !g->zp ||
        (long long)(g->n1m + 2) * (g->n2m + 2) * (g->n3m + 2) >= (1ll << 31)) {
        lica_set_last_error("lica_gpu_bubble_grid_create", "bad grid", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const int n[3] = {g->n1m, g->n2m, g->n3m};
    const double* sd[3] = {g->sdx, g->sdy, g->sdz};
    for (int d = 0; d < 3; ++d)
        for (int i = 1; i <= n[d]; ++i)
            if (!(sd[d][i] > 0.0)) {
                lica_set_last_error("lica_gpu_bubble_grid_create", "cell width not positive", __FILE__, __LINE__);
                return LICA_BAD_ARG;
            }
    lica_bub_geo* b = new lica_bub_geo();
    b->n1m = g->n1m;
    b->n2m = g->n2m;
    b->n3m = g->n3m;
    b->ipx = g->ipx != 0;
    b->ipy = g->ipy != 0;
    b->ipz = g->ipz != 0;
    b->zl = g->zl;
    b->max_lvs = max_lvs;
    const long long pairs = (long long)(g->n1m + 2) * (g->n2m + 2) * (g->n3m + 2) / 2;
    b->nblk = (int)std::min<long long>((pairs + kBubThreads * kPairsInFlight - 1) / (kBubThreads * kPairsInFlight),
                                       kBubMaxBlocks);
    const size_t ng = 2 * (size_t)(g->n1m + 2) + 2 * (size_t)(g->n2m + 2) + 2 * (size_t)(g->n3m + 2);
    double* host = new double[ng];
    size_t o = 0;
    const double* src[6] = {g->sdx, g->sdy, g->sdz, g->xp, g->yp, g->zp};
    for (int q = 0; q < 6; ++q) {
        const int len = n[q % 3] + 2;
        for (int i = 0; i < len; ++i) host[o + i] = src[q][i];
        o += len;
    }
    cudaError_t e = cudaMalloc(&b->geom, ng * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(b->geom, host, ng * sizeof(double), cudaMemcpyHostToDevice);
    delete[] host;
    if (e == cudaSuccess) e = cudaMalloc(&b->part, (size_t)max_lvs * b->nblk * kMomN * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->counters, (size_t)max_lvs * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(b->counters, 0, (size_t)max_lvs * sizeof(unsigned));
    if (e != cudaSuccess) {
        lica_set_last_error("lica_gpu_bubble_grid_create", cudaGetErrorString(e), __FILE__, __LINE__);
        cudaFree(b->geom);
        cudaFree(b->part);
        cudaFree(b->counters);
        delete b;
        return e == cudaErrorMemoryAllocation ? LICA_ERR_NOMEM : LICA_ERR_CUDA;
    }
    *out = b;
    return LICA_OK;
}

int lica_gpu_bubble_grid_destroy(lica_bub_geo* b) {
    if (!b) return LICA_OK;
    cudaFree(b->geom);
    cudaFree(b->part);
    cudaFree(b->counters);
    delete b;
    return LICA_OK;
}

int lica_gpu_bubble_tracking_device(lica_bub_geo* b, int32_t nlvs, int32_t llvs0, const double* psi_tmp,
                                    const double* u, const double* v, const double* w, double time, int32_t icacy,
                                    void* out, void* stream) {
    if (!b || nlvs < 0 || nlvs > b->max_lvs || (icacy != 1 && icacy != 2) ||
        (nlvs > 0 && (!psi_tmp || !u || !v || !w || !out)) || (reinterpret_cast<uintptr_t>(psi_tmp) & 7) ||
        (reinterpret_cast<uintptr_t>(out) & 7)) {
        lica_set_last_error("lica_gpu_bubble_tracking_device", "bad argument", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    if (nlvs == 0) return LICA_OK;
    BubArgs A;
    A.n1m = b->n1m;
    A.n2m = b->n2m;
    A.n3m = b->n3m;
    A.ipx = b->ipx;
    A.ipy = b->ipy;
    A.ipz = b->ipz;
    A.zl = b->zl;
    A.sdx = b->geom;
    A.sdy = A.sdx + (b->n1m + 2);
    A.sdz = A.sdy + (b->n2m + 2);
    A.xp = A.sdz + (b->n3m + 2);
    A.yp = A.xp + (b->n1m + 2);
    A.zp = A.yp + (b->n2m + 2);
    A.psi = psi_tmp;
    A.u = u;
    A.v = v;
    A.w = w;
    A.fsize = (long long)(b->n1m + 2) * (b->n2m + 2) * (b->n3m + 2);
    A.llvs0 = llvs0;
    A.icacy = icacy;
    A.time = time;
    A.part = b->part;
    A.counters = b->counters;
    A.out = static_cast<lica_bub_record*>(out);
    if (!b->smem_set) {
        LICA_CUDA_TRY(cudaFuncSetAttribute(k_bubble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBubSmem));
        b->smem_set = true;
    }
    k_bubble<<<dim3(b->nblk, nlvs), kBubThreads, kBubSmem, (cudaStream_t)stream>>>(A);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int lica_gpu_bubble_tracking(const lica_bub_grid* g, int32_t nlvs, int32_t llvs0, const double* psi_tmp,
                             const double* u, const double* v, const double* w, double time, int32_t icacy,
                             lica_bub_record* out) {
    if (nlvs < 0 || (nlvs > 0 && (!psi_tmp || !u || !v || !w || !out))) {
        lica_set_last_error("lica_gpu_bubble_tracking", "bad argument", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    if (nlvs == 0) return LICA_OK;
    lica_bub_geo* b = nullptr;
    int rc = lica_gpu_bubble_grid_create(&b, g, nlvs);
    if (rc != LICA_OK) return rc;
    const size_t fsize = (size_t)(g->n1m + 2) * (g->n2m + 2) * (g->n3m + 2) * sizeof(double);
    double *dpsi = nullptr, *du = nullptr, *dv = nullptr, *dw = nullptr;
    lica_bub_record* dout = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&dpsi, fsize * nlvs);
    if (e == cudaSuccess) e = cudaMalloc(&du, fsize);
    if (e == cudaSuccess) e = cudaMalloc(&dv, fsize);
    if (e == cudaSuccess) e = cudaMalloc(&dw, fsize);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(lica_bub_record) * nlvs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dpsi, psi_tmp, fsize * nlvs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du, u, fsize, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, v, fsize, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dw, w, fsize, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        rc = lica_gpu_bubble_tracking_device(b, nlvs, llvs0, dpsi, du, dv, dw, time, icacy, dout, st);
        if (rc == LICA_OK)
            e = cudaMemcpyAsync(out, dout, sizeof(lica_bub_record) * nlvs, cudaMemcpyDeviceToHost, st);
        if (rc == LICA_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        lica_set_last_error("lica_gpu_bubble_tracking", cudaGetErrorString(e), __FILE__, __LINE__);
        rc = e == cudaErrorMemoryAllocation ? LICA_ERR_NOMEM : LICA_ERR_CUDA;
    }
    if (st) cudaStreamSynchronize(st);
    cudaFree(dpsi);
    cudaFree(du);
    cudaFree(dv);
    cudaFree(dw);
    cudaFree(dout);
    if (st) cudaStreamDestroy(st);
    lica_gpu_bubble_grid_destroy(b);
    return rc;
}

}  // extern "C"
