"""Known-answer tests that pin the oracle's tridiagonal solvers and 1-D POISSON.

The reference ships no tests or golden vectors; these checks pin the CPU restatement
against mathematics (dense solves, a manufactured solution) and against the golden
fixture of the shipped column (tests/golden/poisson1d_ship.npz).
"""
import os

import numpy as np
import pytest

from oracle import oracle
from lica_boiling1d_b200.poisson import uniform_column_geometry

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _random_tridiag(ld, n, rng, dominant=True):
    A = rng.uniform(-1, 1, (ld, n))
    C = rng.uniform(-1, 1, (ld, n))
    B = rng.uniform(-1, 1, (ld, n)) + (np.sign(rng.uniform(-1, 1, (ld, n))) * 3.0 if dominant else 0.0)
    R = rng.standard_normal((ld, n))
    return [np.asfortranarray(x) for x in (A, B, C, R)]


def test_trdiag3_matches_dense_solve():
    rng = np.random.default_rng(1)
    ld, n = 7, 40
    A, B, C, R = _random_tridiag(ld, n, rng)
    l1, l2, ll1, ll2 = 3, 37, 2, 6
    Rout, UU = oracle.trdiag3(A, B, C, R, l1, l2, ll1, ll2)
    for i in range(ll1, ll2 + 1):
        m = l2 - l1 + 1
        M = np.zeros((m, m))
        for r in range(m):
            j = l1 + r
            M[r, r] = B[i - 1, j - 1]
            if r > 0:
                M[r, r - 1] = A[i - 1, j - 1]
            if r < m - 1:
                M[r, r + 1] = C[i - 1, j - 1]
        x = np.linalg.solve(M, R[i - 1, l1 - 1:l2])
        np.testing.assert_allclose(UU[i - 1, l1 - 1:l2], x, rtol=1e-12, atol=1e-13)
        # R holds the solution for J < L2 (loop 30 of 1d.f:3805-3809), R(I,L2) unchanged
        np.testing.assert_array_equal(Rout[i - 1, l1 - 1:l2 - 1], UU[i - 1, l1 - 1:l2 - 1])
        assert Rout[i - 1, l2 - 1] == R[i - 1, l2 - 1]
    # lines outside [ll1, ll2] untouched
    np.testing.assert_array_equal(Rout[0], R[0])


def test_trdiag3p_matches_dense_cyclic_solve():
    rng = np.random.default_rng(2)
    ld, n = 5, 33
    A, B, C, F = _random_tridiag(ld, n, rng)
    j1, j2, l1, l2 = 2, 31, 1, 4
    Fout = oracle.trdiag3p(A, B, C, F, j1, j2, l1, l2)
    for k in range(l1, l2 + 1):
        m = j2 - j1 + 1
        M = np.zeros((m, m))
        for r in range(m):
            j = j1 + r
            M[r, r] = B[k - 1, j - 1]
            M[r, (r - 1) % m] += A[k - 1, j - 1]
            M[r, (r + 1) % m] += C[k - 1, j - 1]
        x = np.linalg.solve(M, F[k - 1, j1 - 1:j2])
        np.testing.assert_allclose(Fout[k - 1, j1 - 1:j2], x, rtol=1e-11, atol=1e-12)


def _poisson_inputs(n3m, rng, rho_ratio=1000.0, z0=0.1):
    g = uniform_column_geometry(n3m)
    m1, m2, m3 = g["m1"], g["m2"], g["m3"]
    z = (np.arange(m3 + 1) - 0.5) / n3m           # cell centre of index k (k=1..n3m)
    rho = np.where(z < z0, 1.0, rho_ratio)          # vapour (rho=1) below z0
    denf_zi = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
    for k in range(1, n3m + 1):
        rf = rho[k] if k == 1 else 0.5 * (rho[k] + rho[k - 1])
        denf_zi[:, :, k] = 1.0 / rf
    denf_zi[:, :, n3m + 1] = denf_zi[:, :, n3m]     # 1d.f:2991-2992
    divg = np.asfortranarray(rng.standard_normal((m1 - 1, m2 - 1, m3 - 1)))
    p = np.asfortranarray(rng.standard_normal((m1 + 1, m2 + 1, m3 + 1)))
    return g, p, divg, denf_zi


def test_poisson1d_matches_dense_operator():
    rng = np.random.default_rng(3)
    n3m = 64
    g, p, divg, den = _poisson_inputs(n3m, rng)
    out = oracle.poisson1d(g, p, divg, den)
    # the tridiagonal operator of 1d.f:3535-3541
    h = 1.0 / n3m
    M = np.zeros((n3m, n3m))
    for k in range(1, n3m + 1):
        ak = (1.0 / h if k > 1 else 2.0 / h) * (1.0 / h) * den[1, 1, k] * (1.0 - g["fixkl"][k - 1])
        vv_kp1 = 2.0 / h if k == n3m else 1.0 / h
        ck = vv_kp1 * (1.0 / h) * den[1, 1, k + 1]
        M[k - 1, k - 1] = -(ak + ck)
        if k > 1:
            M[k - 1, k - 2] = ak
        if k < n3m:
            M[k - 1, k] = ck
    x = np.linalg.solve(M, divg[0, 0, :n3m])
    np.testing.assert_allclose(out[1, 1, 1:n3m + 1], x, rtol=1e-9, atol=1e-12 * np.abs(x).max())
    np.testing.assert_array_equal(out[1, 1, 0], out[1, 1, 1])
    np.testing.assert_array_equal(out[1, 1, n3m + 1], out[1, 1, n3m])
    # entries the reference does not write keep their values
    np.testing.assert_array_equal(out[0], p[0])
    np.testing.assert_array_equal(out[2], p[2])


def test_poisson1d_manufactured_solution():
    # constant beta, p = cos(pi z / 2): p'(0) = 0 (Neumann wall), p(1) = 0 on the top
    # face; the discrete solve converges to p at second order.
    errs = []
    for n3m in (64, 128, 256):
        g = uniform_column_geometry(n3m)
        m1, m2, m3 = g["m1"], g["m2"], g["m3"]
        h = 1.0 / n3m
        zc = (np.arange(1, n3m + 1) - 0.5) * h
        exact = np.cos(0.5 * np.pi * zc)
        f = -(0.5 * np.pi) ** 2 * exact
        den = np.ones((m1 + 1, m2 + 1, m3 + 1), order="F")
        divg = np.zeros((m1 - 1, m2 - 1, m3 - 1), order="F")
        divg[0, 0, :] = f
        p = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
        out = oracle.poisson1d(g, p, divg, den)
        errs.append(np.abs(out[1, 1, 1:n3m + 1] - exact).max())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert errs[-1] < 1e-4
    assert np.all(rates > 1.8), (errs, rates)


def test_poisson1d_golden_fixture():
    # golden: the shipped column (256 cells, DENR=1605.36, interface at z=0.0607) solved
    # by a dense LAPACK solve in tests/golden/make_golden.py
    d = np.load(os.path.join(GOLDEN, "poisson1d_ship.npz"))
    n3m = int(d["n3m"])
    g = uniform_column_geometry(n3m)
    out = oracle.poisson1d(g, d["p_in"], d["divgsum"], d["denf_zi"])
    ref = d["p_out"]
    scale = np.abs(ref).max()
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-10 * scale)
