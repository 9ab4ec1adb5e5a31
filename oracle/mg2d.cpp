// ORACLE (test infrastructure only) -- CPU restatement of the variable-coefficient
// pressure-Poisson multigrid.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs may load this code; the product never does.
//
// Parity status: the reference (Fortran/OpenMP, no test suite, no golden vectors,
// not compilable without a Fortran compiler) has NO multigrid.  Its POISSON
// (1d.f:3492-3578) is a single Thomas sweep along z.  This file generalises that
// discrete operator to 2-D and solves it with a V(nu1,nu2) red-black Gauss-Seidel
// multigrid.  It is pinned by known-answer tests (scipy direct solve, the exact 1-D
// Thomas solution), not by reference outputs: parity unpinned against the reference.
//
// Discrete operator (one level, cell-centred, uniform hx, hy), the 2-D analogue of
// 1d.f:3535-3541 (AK/CK/BK):
//   x: periodic (IPX=1, lica.in:16); bx[j*nx+i] = beta on the face between cell
//      (i-1 mod nx) and cell i.
//   y: wall-normal (the reference's z).  by[j*nx+i], j=0..ny, = beta on the face
//      below cell row j.  Bottom face j=0 is a Neumann wall (FIXKL(1)=1 kills AK(1),
//      1d.f:3537, INDICES 1d.f:5021-5026).  Top face j=ny carries p=0 ON THE FACE:
//      the reference uses VVDZ(N3)=1/(0.5*SDZ(N3M)) (GEOMETRIC 1d.f:4852) with the
//      FIXKU factor commented out (1d.f:3538), so the top coefficient is
//      2*beta/h^2 against a zero ghost.
//   (A u)_ij = aw*uw + ae*ue + as*us + an*un - (aw+ae+as+an)*u_ij,
//   aw = cx*bx(i), ae = cx*bx(i+1), as = cy*by(j) (0 at j=0),
//   an = cy*by(j+1) (2*cy*by(ny) at the top row, un = 0 there), cx=1/hx^2, cy=1/hy^2.
//
// Operation order (the CUDA kernels follow it exactly, compiled without FMA
// contraction, so FP64 and FP32 iterates agree bit for bit):
//   s = aw*uw; s += ae*ue; s += as*us; s += an*un;   d = aw; d += ae; d += as; d += an;
//   Gauss-Seidel update: u = (s - f) * dinv with dinv = 1 / d;  residual: r = f - (s - d*u).
//
// Multigrid (new build; no counterpart in the reference):
//   restriction      fc(I,J) = 0.25*((r00 + r10) + (r01 + r11))  (2x2 average)
//   beta coarsening  bxc(I,J) = 0.5*(bx(2I,2J) + bx(2I,2J+1)),
//                    byc(I,J) = 0.5*(by(2I,2J) + by(2I+1,2J))  (faces in parallel)
//   prolongation     bilinear, cell-centred weights 9/16,3/16,3/16,1/16;
//                    ghosts: x periodic, bottom mirror (Neumann), top -e (p=0 on face)
//   smoother         red (i+j even) then black, nu sweeps
//   coarsest outer level: ncoarse inner V(nu1,nu2) cycles over an inner hierarchy
//                    that halves while both sizes stay even and >= 2, ending in a
//                    dense Gaussian elimination (no pivoting; A is negative definite).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

template <typename T>
struct Level {
    int nx = 0, ny = 0;
    T cx = 0, cy = 0;
    std::vector<T> u, f, r, bx, by;
};

template <typename T>
inline void coeffs(const Level<T>& L, int i, int j, T& aw, T& ae, T& as, T& an) {
    const int nx = L.nx, ny = L.ny;
    const int ip = (i + 1 == nx) ? 0 : i + 1;
    aw = L.cx * L.bx[(size_t)j * nx + i];
    ae = L.cx * L.bx[(size_t)j * nx + ip];
    as = (j > 0) ? L.cy * L.by[(size_t)j * nx + i] : T(0);
    if (j < ny - 1) an = L.cy * L.by[(size_t)(j + 1) * nx + i];
    else            an = T(2) * L.cy * L.by[(size_t)ny * nx + i];
}

template <typename T>
inline void stencil_sums(const Level<T>& L, const T* u, int i, int j, T& s, T& d) {
    const int nx = L.nx, ny = L.ny;
    const int ip = (i + 1 == nx) ? 0 : i + 1;
    const int im = (i == 0) ? nx - 1 : i - 1;
    T aw, ae, as, an;
    coeffs(L, i, j, aw, ae, as, an);
    const T uw = u[(size_t)j * nx + im];
    const T ue = u[(size_t)j * nx + ip];
    const T us = (j > 0) ? u[(size_t)(j - 1) * nx + i] : T(0);
    const T un = (j < ny - 1) ? u[(size_t)(j + 1) * nx + i] : T(0);
    s = aw * uw; s += ae * ue; s += as * us; s += an * un;
    d = aw; d += ae; d += as; d += an;
}

template <typename T>
void rb_sweep(Level<T>& L, int nsweeps, bool reverse) {
    for (int s = 0; s < nsweeps; ++s)
        for (int c = 0; c < 2; ++c) {
            const int colour = reverse ? 1 - c : c;
#pragma omp parallel for schedule(static) if ((size_t)L.nx * L.ny > 65536)
            for (int j = 0; j < L.ny; ++j)
                for (int i = (j + colour) & 1; i < L.nx; i += 2) {
                    T sm, d;
                    stencil_sums(L, L.u.data(), i, j, sm, d);
                    const T dinv = T(1) / d;
                    L.u[(size_t)j * L.nx + i] = (sm - L.f[(size_t)j * L.nx + i]) * dinv;
                }
        }
}

// y-line zebra relaxation (flag MG_YLINE; no counterpart in the reference): columns of
// one parity (i even, then i odd; the reverse order when `reverse`) are each solved
// exactly along y -- as u(j-1) - d u(j) + an u(j+1) = f - aw uw - ae ue, with u = 0 past the
// top face -- by the Thomas algorithm, the x neighbours held at their current values.
// It keeps the multigrid rate on cells much finer in y than in x (stretched wall grids),
// where point relaxation does not smooth along x.
template <typename T>
void yline_sweep(Level<T>& L, int nsweeps, bool reverse) {
    const int nx = L.nx, ny = L.ny;
    for (int s = 0; s < nsweeps; ++s)
        for (int c = 0; c < 2; ++c) {
            const int parity = reverse ? 1 - c : c;
#pragma omp parallel for schedule(static) if ((size_t)nx * ny > 65536)
            for (int i = parity; i < nx; i += 2) {
                const int ip = (i + 1 == nx) ? 0 : i + 1;
                const int im = (i == 0) ? nx - 1 : i - 1;
                std::vector<T> cp(ny), dp(ny);
                T prev_c = T(0), prev_d = T(0);
                for (int j = 0; j < ny; ++j) {
                    T aw, ae, as, an;
                    coeffs(L, i, j, aw, ae, as, an);
                    T rhs = L.f[(size_t)j * nx + i];
                    rhs -= aw * L.u[(size_t)j * nx + im];
                    rhs -= ae * L.u[(size_t)j * nx + ip];
                    T d = aw; d += ae; d += as; d += an;
                    const T diag = -d;
                    const T sup = (j < ny - 1) ? an : T(0);
                    // forward elimination: as is the sub-diagonal (0 at the bottom wall)
                    const T den = diag - as * prev_c;
                    cp[j] = sup / den;
                    dp[j] = (rhs - as * prev_d) / den;
                    prev_c = cp[j];
                    prev_d = dp[j];
                }
                T x = dp[ny - 1];
                L.u[(size_t)(ny - 1) * nx + i] = x;
                for (int j = ny - 2; j >= 0; --j) {
                    x = dp[j] - cp[j] * x;
                    L.u[(size_t)j * nx + i] = x;
                }
            }
        }
}

template <typename T>
void residual(Level<T>& L) {
#pragma omp parallel for schedule(static) if ((size_t)L.nx * L.ny > 65536)
    for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
            T sm, d;
            stencil_sums(L, L.u.data(), i, j, sm, d);
            const size_t k = (size_t)j * L.nx + i;
            L.r[k] = L.f[k] - (sm - d * L.u[k]);
        }
}

// 1-D prolongation weights along y, with the boundary ghosts folded in.
// Fine row j takes from coarse rows J=j>>1 (weight 3/4) and Jn (1/4); Jn=J-1 for even j,
// J+1 for odd j.  Bottom ghost (Jn=-1) mirrors row 0: weight moves onto J=0 (total 1).
// Top ghost (Jn=ncy) is -e(ncy-1): the weight becomes 3/4-1/4 = 1/2 on J=ncy-1.
// For the restriction (the transpose) wy(J, j) returns the weight of fine row j in coarse row J.
template <typename T>
inline T wy(int J, int j, int ncy, int ny) {
    const int Jj = j >> 1;
    if (j < 0 || j >= ny) return T(0);
    if (Jj == J) {
        if (j == 0) return T(1);
        if (j == ny - 1) return T(0.5);
        return T(0.75);
    }
    const int Jn = (j & 1) ? Jj + 1 : Jj - 1;
    if (Jn == J && Jn >= 0 && Jn < ncy) return T(0.25);
    return T(0);
}

// Restriction.  sym=false: 2x2 average fc = 0.25*((r00 + r10) + (r01 + r11)).
// sym=true : R = P^T/4 (the transpose of bilinear prolongation), summed over the 4x4
//            fine neighbourhood i = 2I-1..2I+2 (periodic), j = 2J-1..2J+2, in the order
//            acc_row(j) = ((w0*r0 + w1*r1) + w2*r2) + w3*r3 with x weights 1/4,3/4,3/4,1/4,
//            fc = 0.25 * (((wy0*acc0 + wy1*acc1) + wy2*acc2) + wy3*acc3).
template <typename T>
void restrict_to(const Level<T>& F, Level<T>& C, bool sym) {
#pragma omp parallel for schedule(static) if ((size_t)F.nx * F.ny > 65536)
    for (int J = 0; J < C.ny; ++J)
        for (int I = 0; I < C.nx; ++I) {
            if (!sym) {
                const size_t a = (size_t)(2 * J) * F.nx + 2 * I;
                const size_t b = a + F.nx;
                C.f[(size_t)J * C.nx + I] = T(0.25) * ((F.r[a] + F.r[a + 1]) + (F.r[b] + F.r[b + 1]));
                continue;
            }
            const int i0 = (2 * I - 1 + F.nx) % F.nx, i1 = 2 * I, i2 = 2 * I + 1, i3 = (2 * I + 2) % F.nx;
            T acc[4];
            for (int q = 0; q < 4; ++q) {
                const int j = 2 * J - 1 + q;
                if (j < 0 || j >= F.ny) { acc[q] = T(0); continue; }
                const T* row = F.r.data() + (size_t)j * F.nx;
                T a = T(0.25) * row[i0];
                a += T(0.75) * row[i1];
                a += T(0.75) * row[i2];
                a += T(0.25) * row[i3];
                acc[q] = a;
            }
            T s = wy<T>(J, 2 * J - 1, C.ny, F.ny) * acc[0];
            s += wy<T>(J, 2 * J, C.ny, F.ny) * acc[1];
            s += wy<T>(J, 2 * J + 1, C.ny, F.ny) * acc[2];
            s += wy<T>(J, 2 * J + 2, C.ny, F.ny) * acc[3];
            C.f[(size_t)J * C.nx + I] = T(0.25) * s;
        }
}

// Bilinear cell-centred prolongation added to the fine iterate:
// e = 0.0625*((9*e00 + 3*e10) + (3*e01 + e11)), e10 = x-neighbour, e01 = y-neighbour,
// e11 = diagonal; ghosts: x periodic, bottom mirror (Neumann), top -e (p=0 on the face).
template <typename T>
void prolong_add(const Level<T>& C, Level<T>& F, bool pconst) {
    const int ncx = C.nx, ncy = C.ny;
#pragma omp parallel for schedule(static) if ((size_t)F.nx * F.ny > 65536)
    for (int j = 0; j < F.ny; ++j)
        for (int i = 0; i < F.nx; ++i) {
            const int I = i >> 1, J = j >> 1;
            if (pconst) { F.u[(size_t)j * F.nx + i] += C.u[(size_t)J * ncx + I]; continue; }
            const int In = (i & 1) ? ((I + 1 == ncx) ? 0 : I + 1) : ((I == 0) ? ncx - 1 : I - 1);
            const int Jn = (j & 1) ? J + 1 : J - 1;
            auto ec = [&](int ii, int jj) -> T {
                if (jj < 0) jj = 0;
                if (jj >= ncy) return -C.u[(size_t)(ncy - 1) * ncx + ii];
                return C.u[(size_t)jj * ncx + ii];
            };
            const T e00 = ec(I, J), e10 = ec(In, J), e01 = ec(I, Jn), e11 = ec(In, Jn);
            const T e = T(0.0625) * ((T(9) * e00 + T(3) * e10) + (T(3) * e01 + e11));
            F.u[(size_t)j * F.nx + i] += e;
        }
}

template <typename T>
void coarsen_beta(const Level<T>& F, Level<T>& C) {
    for (int J = 0; J < C.ny; ++J)
        for (int I = 0; I < C.nx; ++I)
            C.bx[(size_t)J * C.nx + I] =
                T(0.5) * (F.bx[(size_t)(2 * J) * F.nx + 2 * I] + F.bx[(size_t)(2 * J + 1) * F.nx + 2 * I]);
    for (int J = 0; J <= C.ny; ++J)
        for (int I = 0; I < C.nx; ++I)
            C.by[(size_t)J * C.nx + I] =
                T(0.5) * (F.by[(size_t)(2 * J) * F.nx + 2 * I] + F.by[(size_t)(2 * J) * F.nx + 2 * I + 1]);
}

template <typename T>
void alloc_level(Level<T>& L, int nx, int ny, double hx, double hy) {
    L.nx = nx; L.ny = ny;
    L.cx = T(1.0 / (hx * hx));
    L.cy = T(1.0 / (hy * hy));
    const size_t n = (size_t)nx * ny;
    L.u.assign(n, T(0)); L.f.assign(n, T(0)); L.r.assign(n, T(0));
    L.bx.assign(n, T(0)); L.by.assign(n + nx, T(0));
}

// Dense Gaussian elimination on the bottom level (row-major n x n, no pivoting).
// Order: for k: for i>k: m = A[i][k]/A[k][k]; A[i][j] -= m*A[k][j] (j>k); b[i] -= m*b[k];
// back substitution x[i] = (b[i] - sum_{j>i} A[i][j]*x[j]) / A[i][i], sum in increasing j.
template <typename T>
void dense_solve(Level<T>& L) {
    const int nx = L.nx, ny = L.ny, n = nx * ny;
    std::vector<T> A((size_t)n * n, T(0)), b(L.f);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            T aw, ae, as, an;
            coeffs(L, i, j, aw, ae, as, an);
            const int row = j * nx + i;
            const int ip = (i + 1 == nx) ? 0 : i + 1, im = (i == 0) ? nx - 1 : i - 1;
            T d = aw; d += ae; d += as; d += an;
            A[(size_t)row * n + row] -= d;
            A[(size_t)row * n + j * nx + im] += aw;
            A[(size_t)row * n + j * nx + ip] += ae;
            if (j > 0) A[(size_t)row * n + (j - 1) * nx + i] += as;
            if (j < ny - 1) A[(size_t)row * n + (j + 1) * nx + i] += an;
        }
    for (int k = 0; k < n; ++k) {
        const T piv = A[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) {
            const T m = A[(size_t)i * n + k] / piv;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= m * A[(size_t)k * n + j];
            b[i] -= m * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        T s = b[i];
        for (int j = i + 1; j < n; ++j) s -= A[(size_t)i * n + j] * L.u[j];
        L.u[i] = s / A[(size_t)i * n + i];
    }
}


// Cycle options (flags): MG_SYM_SMOOTH post-smoothing black-then-red; MG_RT restriction
// R = P^T/4 of bilinear P (else the 2x2 average); MG_PCONST piecewise-constant P (whose
// transpose/4 is the 2x2 average); MG_YLINE y-line zebra relaxation instead of red-black
// points (post-smoothing in the reverse parity order when MG_SYM_SMOOTH).
enum { MG_SYM_SMOOTH = 1, MG_RT = 2, MG_PCONST = 4, MG_YLINE = 8 };
struct Opts {
    int nu1, nu2, ncoarse;
    int flags;
    bool sym() const { return flags & MG_SYM_SMOOTH; }
    bool rt() const { return (flags & MG_RT) && !(flags & MG_PCONST); }
    bool pconst() const { return flags & MG_PCONST; }
    bool yline() const { return flags & MG_YLINE; }
};

template <typename T>
void smooth(Level<T>& L, int nsweeps, bool reverse, const Opts& o) {
    if (o.yline()) yline_sweep(L, nsweeps, reverse);
    else rb_sweep(L, nsweeps, reverse);
}

template <typename T>
struct Hierarchy {
    std::vector<Level<T>> lv;   // outer levels 0..nouter-1, then the inner levels
    int nouter = 0;
};

template <typename T>
int build_hierarchy(Hierarchy<T>& H, int nx, int ny, double hx, double hy, int nouter,
                    const double* bx, const double* by) {
    if (nouter < 1 || nx < 2 || ny < 1) return 4;
    H.lv.clear();
    H.nouter = nouter;
    int cx = nx, cy = ny;
    double chx = hx, chy = hy;
    for (int l = 0; l < nouter; ++l) {
        if (l > 0) {
            if ((cx & 1) || (cy & 1) || cx < 4 || cy < 2) return 4;
            cx /= 2; cy /= 2; chx *= 2; chy *= 2;
        }
        H.lv.emplace_back();
        alloc_level(H.lv.back(), cx, cy, chx, chy);
    }
    while (!(cx & 1) && !(cy & 1) && cx / 2 >= 2 && cy / 2 >= 2) {
        cx /= 2; cy /= 2; chx *= 2; chy *= 2;
        H.lv.emplace_back();
        alloc_level(H.lv.back(), cx, cy, chx, chy);
    }
    if ((size_t)H.lv.back().nx * H.lv.back().ny > 1024) return 4;
    Level<T>& L0 = H.lv[0];
    for (size_t k = 0; k < L0.bx.size(); ++k) L0.bx[k] = T(bx[k]);
    for (size_t k = 0; k < L0.by.size(); ++k) L0.by[k] = T(by[k]);
    for (size_t l = 1; l < H.lv.size(); ++l) coarsen_beta(H.lv[l - 1], H.lv[l]);
    return 0;
}

// V-cycle on level l with whatever iterate lv[l].u holds (zero for a correction).
// Levels below the coarsest outer level form the inner hierarchy; the last level is
// solved densely.
template <typename T>
void vcycle_inner(Hierarchy<T>& H, size_t l, const Opts& o) {
    Level<T>& L = H.lv[l];
    if (l + 1 == H.lv.size()) { dense_solve(L); return; }
    smooth(L, o.nu1, false, o);
    residual(L);
    Level<T>& C = H.lv[l + 1];
    restrict_to(L, C, o.rt());
    std::fill(C.u.begin(), C.u.end(), T(0));
    vcycle_inner(H, l + 1, o);
    prolong_add(C, L, o.pconst());
    smooth(L, o.nu2, o.sym(), o);
}

// Coarsest outer level: ncoarse inner cycles from a zero iterate (a fixed linear,
// symmetric operator when o.sym), or a dense solve if it is the bottom level.
template <typename T>
void coarse_solve(Hierarchy<T>& H, const Opts& o) {
    const size_t lc = H.nouter - 1;
    Level<T>& L = H.lv[lc];
    std::fill(L.u.begin(), L.u.end(), T(0));
    if (lc + 1 == H.lv.size()) { dense_solve(L); return; }
    for (int c = 0; c < o.ncoarse; ++c) vcycle_inner(H, lc, o);
}

// Outer V-cycle from level l down, iterate in lv[l].u.  At the coarsest outer level
// the correction comes from coarse_solve in the hierarchy Hc (FP64 when T is float).
template <typename T, typename TC>
void vcycle_outer(Hierarchy<T>& H, Hierarchy<TC>& Hc, size_t l, const Opts& o) {
    const size_t lc = H.nouter - 1;
    Level<T>& L = H.lv[l];
    if (l == lc) {
        Level<TC>& D = Hc.lv[lc];
        for (size_t k = 0; k < D.f.size(); ++k) D.f[k] = TC(L.f[k]);
        coarse_solve(Hc, o);
        for (size_t k = 0; k < D.u.size(); ++k) L.u[k] = T(D.u[k]);
        return;
    }
    smooth(L, o.nu1, false, o);
    residual(L);
    Level<T>& C = H.lv[l + 1];
    restrict_to(L, C, o.rt());
    std::fill(C.u.begin(), C.u.end(), T(0));
    vcycle_outer(H, Hc, l + 1, o);
    prolong_add(C, L, o.pconst());
    smooth(L, o.nu2, o.sym(), o);
}

template <typename T>
double dot(const std::vector<T>& a, const std::vector<T>& b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static) if (a.size() > 65536)
    for (size_t k = 0; k < a.size(); ++k) s += double(a[k]) * double(b[k]);
    return s;
}

// FP64 residual r = f - A u of level L's operator.
void residual64(const Level<double>& L, const double* u, const double* f, double* r) {
#pragma omp parallel for schedule(static) if ((size_t)L.nx * L.ny > 65536)
    for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
            double sm, d;
            stencil_sums(L, u, i, j, sm, d);
            const size_t k = (size_t)j * L.nx + i;
            r[k] = f[k] - (sm - d * u[k]);
        }
}

void apply64(const Level<double>& L, const double* u, double* out) {
#pragma omp parallel for schedule(static) if ((size_t)L.nx * L.ny > 65536)
    for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
            double sm, d;
            stencil_sums(L, u, i, j, sm, d);
            const size_t k = (size_t)j * L.nx + i;
            out[k] = sm - d * u[k];
        }
}

struct Solver {
    Hierarchy<double> H;
    Hierarchy<float> S;
    bool mixed = false;
    Opts o{2, 2, 2, MG_SYM_SMOOTH | MG_RT};

    // z = M r: one V-cycle from a zero iterate (FP64), or one FP32 V-cycle with an
    // FP64 coarsest solve (mixed).  r and z are FP64 fine-level vectors.
    void precond(const std::vector<double>& r, std::vector<double>& z) {
        const size_t n = r.size();
        if (!mixed) {
            Level<double>& L0 = H.lv[0];
            std::memcpy(L0.f.data(), r.data(), n * sizeof(double));
            std::fill(L0.u.begin(), L0.u.end(), 0.0);
            vcycle_outer(H, H, 0, o);
            std::memcpy(z.data(), L0.u.data(), n * sizeof(double));
        } else {
            Level<float>& L0 = S.lv[0];
            for (size_t k = 0; k < n; ++k) { L0.f[k] = float(r[k]); L0.u[k] = 0.0f; }
            vcycle_outer(S, H, 0, o);
            for (size_t k = 0; k < n; ++k) z[k] = double(L0.u[k]);
        }
    }
};

}  // namespace

extern "C" {

// out = A u (FP64).
int orc_mg_apply(int nx, int ny, double hx, double hy, const double* bx, const double* by,
                 const double* u, double* out) {
    Level<double> L;
    alloc_level(L, nx, ny, hx, hy);
    std::memcpy(L.bx.data(), bx, sizeof(double) * L.bx.size());
    std::memcpy(L.by.data(), by, sizeof(double) * L.by.size());
    apply64(L, u, out);
    return 0;
}

// nsweeps red-black sweeps (reverse: black first) on one level, FP64, in place on u.
int orc_mg_smooth(int nx, int ny, double hx, double hy, const double* bx, const double* by,
                  const double* f, double* u, int nsweeps, int reverse) {
    Level<double> L;
    alloc_level(L, nx, ny, hx, hy);
    std::memcpy(L.bx.data(), bx, sizeof(double) * L.bx.size());
    std::memcpy(L.by.data(), by, sizeof(double) * L.by.size());
    std::memcpy(L.f.data(), f, sizeof(double) * L.f.size());
    std::memcpy(L.u.data(), u, sizeof(double) * L.u.size());
    rb_sweep(L, nsweeps, reverse != 0);
    std::memcpy(u, L.u.data(), sizeof(double) * L.u.size());
    return 0;
}

// Multigrid solve of A p = f (p holds the initial guess on entry).
//   method 0: stationary V-cycles on p (FP64 only: mixed must be 0).
//   method 1: defect correction p += M (f - A p), M one V-cycle (FP64 or mixed).
//   method 2: preconditioned CG with M as preconditioner (Fletcher-Reeves beta, true
//             residual recomputed every iteration), FP64 vectors; M is FP64 or mixed.
//             M must be symmetric: flags MG_SYM_SMOOTH|MG_PCONST (or |MG_RT).
//   mixed  : M runs its smoothing, restriction and prolongation in FP32 and its
//            coarsest-level solve in FP64.
// Convergence: ||f - A p||_2 / ||f||_2 <= rtol, with the true FP64 residual checked
// after every cycle.  res_hist (length max_cycles+1, may be null) receives the
// relative residual before the first cycle and after each cycle.
// PCG stops when FP64's attainable accuracy is reached: if the true residual rises at
// an iteration while the previous one is within 1000 rtol, the previous iterate is the
// result (the GPU solver's rule; past that point the recomputed residual is rounding
// noise, the directions lose conjugacy and the iteration diverges).
// Returns 0 converged, 1 not converged within max_cycles, 3 non-finite, 4 bad argument,
// 8 stalled at the attainable accuracy.
int orc_mg_solve(int nx, int ny, double hx, double hy, int nlevels, int nu1, int nu2, int ncoarse,
                 int sym, int method, int mixed, const double* f, const double* bx, const double* by,
                 double* p, double rtol, int max_cycles, int* cycles_out, double* rel_out,
                 double* res_hist) {
    Solver sv;
    sv.o = Opts{nu1, nu2, ncoarse, sym};
    sv.mixed = mixed != 0;
    if (method < 0 || method > 2 || (method == 0 && mixed)) return 4;
    int st = build_hierarchy(sv.H, nx, ny, hx, hy, nlevels, bx, by);
    if (st) return st;
    if (sv.mixed && (st = build_hierarchy(sv.S, nx, ny, hx, hy, nlevels, bx, by))) return st;
    Level<double>& L0 = sv.H.lv[0];
    const size_t n = (size_t)nx * ny;
    std::vector<double> fv(f, f + n), x(p, p + n), r(n), z(n), pd(n, 0.0), q(n);
    const double fn = std::sqrt(dot(fv, fv));
    const double fscale = (fn > 0.0) ? fn : 1.0;
    residual64(L0, x.data(), fv.data(), r.data());
    double rel = std::sqrt(dot(r, r)) / fscale;
    if (res_hist) res_hist[0] = rel;
    int c = 0, status = 1;
    double rz = 0.0, rel_prev = rel;
    std::vector<double> x_prev;
    while (true) {
        if (!std::isfinite(rel)) { status = 3; break; }
        if (rel <= rtol) { status = 0; break; }
        if (method == 2 && c > 0 && rel >= rel_prev && rel_prev <= 1e3 * rtol) {
            x = x_prev;
            rel = rel_prev;
            --c;
            status = 8;
            break;
        }
        if (c >= max_cycles) break;
        rel_prev = rel;
        if (method == 2) x_prev = x;
        if (method == 0) {
            std::memcpy(L0.f.data(), fv.data(), n * sizeof(double));
            std::memcpy(L0.u.data(), x.data(), n * sizeof(double));
            vcycle_outer(sv.H, sv.H, 0, sv.o);
            std::memcpy(x.data(), L0.u.data(), n * sizeof(double));
        } else if (method == 1) {
            sv.precond(r, z);
            for (size_t k = 0; k < n; ++k) x[k] += z[k];
        } else {
            // PCG: z = M r; rz = r.z; beta = rz / rz_prev (0 on the first iteration);
            // p = z + beta*p (p starts at 0); alpha = rz / (p.Ap); x += alpha*p;
            // then the true residual r = f - A x (below).
            sv.precond(r, z);
            // mixed: r.z takes the FP32 copy of r that the V-cycle consumed
            double rz_new = 0.0;
            if (sv.mixed) {
#pragma omp parallel for reduction(+ : rz_new) schedule(static) if (n > 65536)
                for (size_t k = 0; k < n; ++k) rz_new += double(float(r[k])) * z[k];
            } else {
                rz_new = dot(r, z);
            }
            const double beta = (c == 0) ? 0.0 : rz_new / rz;
            for (size_t k = 0; k < n; ++k) pd[k] = z[k] + beta * pd[k];
            rz = rz_new;
            apply64(L0, pd.data(), q.data());
            const double alpha = rz / dot(pd, q);
            for (size_t k = 0; k < n; ++k) x[k] += alpha * pd[k];
        }
        ++c;
        residual64(L0, x.data(), fv.data(), r.data());
        rel = std::sqrt(dot(r, r)) / fscale;
        if (res_hist) res_hist[c] = rel;
    }
    std::memcpy(p, x.data(), n * sizeof(double));
    if (cycles_out) *cycles_out = c;
    if (rel_out) *rel_out = rel;
    return status;
}

// z = M r: one application of the V-cycle preconditioner (tests compare the GPU's).
int orc_mg_precond(int nx, int ny, double hx, double hy, int nlevels, int nu1, int nu2, int ncoarse,
                   int sym, int mixed, const double* bx, const double* by, const double* r, double* z) {
    Solver sv;
    sv.o = Opts{nu1, nu2, ncoarse, sym};
    sv.mixed = mixed != 0;
    int st = build_hierarchy(sv.H, nx, ny, hx, hy, nlevels, bx, by);
    if (st) return st;
    if (sv.mixed && (st = build_hierarchy(sv.S, nx, ny, hx, hy, nlevels, bx, by))) return st;
    const size_t n = (size_t)nx * ny;
    std::vector<double> rv(r, r + n), zv(n);
    sv.precond(rv, zv);
    std::memcpy(z, zv.data(), n * sizeof(double));
    return 0;
}

}  // extern "C"
