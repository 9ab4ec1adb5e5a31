// ORACLE (test infrastructure only) -- CPU restatement of the reference's tridiagonal
// solvers and its 1-D pressure POISSON.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU legs load this code.
//
// Parity: the reference ships no tests or golden vectors and cannot be compiled here
// (no Fortran compiler); these routines follow the Fortran statement by statement
// and are pinned by known-answer tests (dense LU, manufactured solutions).
//
// Array conventions: every array is passed as the base address of the Fortran array,
// column-major, with the Fortran lower bound noted per argument.
#include <cstdint>
#include <cstdlib>
#include <vector>

extern "C" {

// TRDIAG3 (1d.f:3783-3811).  A,B,C,R,UU are Fortran (ld, *) arrays, 1-based in both
// indices: X(I,J) = x[(I-1) + (J-1)*ld].  Solves, for every line I in [ll1,ll2], the
// tridiagonal system along J in [l1,l2].  UU receives the solution; R(I,J) is
// overwritten with the solution for J in [l1,l2-1] (the reference's loop 30).  R and
// UU may alias (LHSW calls it with GK twice, 1d.f:1790).
int orc_trdiag3(const double* A, const double* B, const double* C, double* R, double* UU,
                int64_t l1, int64_t l2, int64_t ll1, int64_t ll2, int64_t ld) {
    if (l2 < l1 || ll2 < ll1 || ld < ll2) return 4;
    const int64_t nl = l2 - l1 + 1;
    std::vector<double> gam((size_t)nl + 1);
    auto at = [ld](int64_t i, int64_t j) { return (size_t)((i - 1) + (j - 1) * ld); };
    for (int64_t i = ll1; i <= ll2; ++i) {
        double bet = 1.0 / B[at(i, l1)];
        UU[at(i, l1)] = R[at(i, l1)] * bet;
        for (int64_t j = l1 + 1; j <= l2; ++j) {
            gam[j - l1] = C[at(i, j - 1)] * bet;
            bet = 1.0 / (B[at(i, j)] - A[at(i, j)] * gam[j - l1]);
            UU[at(i, j)] = (R[at(i, j)] - A[at(i, j)] * UU[at(i, j - 1)]) * bet;
        }
        for (int64_t j = l2 - 1; j >= l1; --j) {
            UU[at(i, j)] = UU[at(i, j)] - gam[j + 1 - l1] * UU[at(i, j + 1)];
            R[at(i, j)] = UU[at(i, j)];
        }
    }
    return 0;
}

// TRDIAG3P (1d.f:3929-3983): periodic (cyclic) tridiagonal systems.  A,B,C,F are
// Fortran (ld, *) arrays; lines K in [l1,l2] (first index), unknowns J in [j1,j2]
// (second index).  The solution overwrites F.
int orc_trdiag3p(const double* A, const double* B, const double* C, double* F,
                 int64_t j1, int64_t j2, int64_t l1, int64_t l2, int64_t ld) {
    if (j2 <= j1 || l2 < l1 || ld < l2) return 4;
    const int64_t nj = j2 - j1 + 1;
    auto at = [ld](int64_t k, int64_t j) { return (size_t)((k - 1) + (j - 1) * ld); };
    std::vector<double> Q((size_t)nj), S((size_t)nj), QE((size_t)nj);
    const int64_t ja = j1 + 1, jj = j1 + j2;
    for (int64_t k = l1; k <= l2; ++k) {
        auto q = [&](int64_t j) -> double& { return Q[(size_t)(j - j1)]; };
        auto s = [&](int64_t j) -> double& { return S[(size_t)(j - j1)]; };
        auto qe = [&](int64_t j) -> double& { return QE[(size_t)(j - j1)]; };
        const double binv = 1.0 / B[at(k, j1)];
        q(j1) = -C[at(k, j1)] * binv;
        s(j1) = -A[at(k, j1)] * binv;
        const double fn = F[at(k, j2)];
        F[at(k, j1)] = F[at(k, j1)] * binv;
        for (int64_t j = ja; j <= j2; ++j) {
            const double pn = 1.0 / (B[at(k, j)] + A[at(k, j)] * q(j - 1));
            q(j) = -C[at(k, j)] * pn;
            s(j) = -A[at(k, j)] * s(j - 1) * pn;
            F[at(k, j)] = (F[at(k, j)] - A[at(k, j)] * F[at(k, j - 1)]) * pn;
        }
        s(j2) = 1.0;
        qe(j2) = 0.0;
        for (int64_t i = ja; i <= j2; ++i) {
            const int64_t j = jj - i;
            s(j) = s(j) + q(j) * s(j + 1);
            qe(j) = F[at(k, j)] + q(j) * qe(j + 1);
        }
        F[at(k, j2)] = (fn - C[at(k, j2)] * qe(j1) - A[at(k, j2)] * qe(j2 - 1)) /
                       (C[at(k, j2)] * s(j1) + A[at(k, j2)] * s(j2 - 1) + B[at(k, j2)]);
        for (int64_t i = ja; i <= j2; ++i) {
            const int64_t j = jj - i;
            F[at(k, j)] = F[at(k, j2)] * s(j) + qe(j);
        }
    }
    return 0;
}

// POISSON (1d.f:3492-3578), the 1-D case the reference runs (I=J=1).
//   m1,m2,m3      : PARAM_VAR bounds; P and DENF_ZI are (0:m1,0:m2,0:m3)
//   n1m,n2m,n3m   : active cell counts
//   vvdz          : VVDZ(1:m3)      -> vvdz[k-1]
//   ssdz          : SSDZ(0:m3)      -> ssdz[k]
//   fixkl         : FIXKL(1:m3-1)   -> fixkl[k-1]
//   kpv           : KPV(0:m3+1)     -> kpv[k]
//   divgsum       : DIVGSUM(m1-1,m2-1,m3-1), 1-based
// Coefficients (1d.f:3535-3541): AK = VVDZ(K)*SSDZ(K)*DENF_ZI(1,1,K)*(1-FIXKL(K)),
// CK = VVDZ(KP1)*SSDZ(K)*DENF_ZI(1,1,KP1), BK = -(AK+CK); Thomas from kb=1
// (1d.f:3547-3564); P(1,1,K) = solution; ghosts P(I,J,0)=P(I,J,1), P(I,J,N3)=P(I,J,N3M)
// for I<=N1M, J<=N2M (1d.f:3570-3576).
int orc_poisson1d(int64_t m1, int64_t m2, int64_t m3, int64_t n1m, int64_t n2m, int64_t n3m,
                  const double* vvdz, const double* ssdz, const double* fixkl, const int64_t* kpv,
                  double* p, const double* divgsum, const double* denf_zi) {
    if (n3m < 1 || n3m > m3 - 1 || n1m < 1 || n1m > m1 - 1 || n2m < 1 || n2m > m2 - 1) return 4;
    const int64_t s1 = m1 + 1, s2 = (m1 + 1) * (m2 + 1);
    auto f3 = [&](int64_t i, int64_t j, int64_t k) { return (size_t)(i + s1 * j + s2 * k); };
    const int64_t d1 = m1 - 1, d2 = (m1 - 1) * (m2 - 1);
    auto dv = [&](int64_t i, int64_t j, int64_t k) { return (size_t)((i - 1) + d1 * (j - 1) + d2 * (k - 1)); };
    std::vector<double> ak((size_t)n3m + 2), bk((size_t)n3m + 2), ck((size_t)n3m + 2), gk((size_t)n3m + 2),
        uu((size_t)n3m + 2), gam((size_t)n3m + 2, 0.0);
    for (int64_t k = 1; k <= n3m; ++k) {
        const int64_t kp1 = kpv[k];
        ak[k] = vvdz[k - 1] * ssdz[k] * denf_zi[f3(1, 1, k)] * (1.0 - fixkl[k - 1]);
        ck[k] = vvdz[kp1 - 1] * ssdz[k] * denf_zi[f3(1, 1, kp1)];
        bk[k] = -(ak[k] + ck[k]);
        gk[k] = divgsum[dv(1, 1, k)];
    }
    double bet = 1.0 / bk[1];
    uu[1] = gk[1] * bet;
    for (int64_t k = 2; k <= n3m; ++k) {
        gam[k] = ck[k - 1] * bet;
        bet = 1.0 / (bk[k] - ak[k] * gam[k]);
        uu[k] = (gk[k] - ak[k] * uu[k - 1]) * bet;
    }
    for (int64_t k = n3m - 1; k >= 1; --k) uu[k] = uu[k] - gam[k + 1] * uu[k + 1];
    for (int64_t k = 1; k <= n3m; ++k) p[f3(1, 1, k)] = uu[k];
    for (int64_t j = 1; j <= n2m; ++j)
        for (int64_t i = 1; i <= n1m; ++i) {
            p[f3(i, j, 0)] = p[f3(i, j, 1)];
            p[f3(i, j, n3m + 1)] = p[f3(i, j, n3m)];
        }
    return 0;
}

}  // extern "C"
