"""Generates the golden fixtures in this folder (committed; rerun only to refresh).

The reference ships no test vectors and cannot be compiled here, so each fixture is
a known answer computed independently of both the oracle and the CUDA path:

* poisson1d_ship.npz -- the reference's shipped 1-D column (grid.in: 256 cells on
  [0,1]; lica.in: DENR = 1605.36; LVSINIT: interface at z = 0.0607, two_phase.f:109)
  with a seeded random DIVGSUM; P solved by a dense LAPACK solve of the tridiagonal
  operator of POISSON (1d.f:3535-3541) with its ghost copies (1d.f:3570-3576).
* mg_bubbles64.npz -- a 64x64 2-D pressure Poisson with 8 seeded bubbles of density
  1000 and a Gaussian right-hand side, solved by scipy's sparse direct solver.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lica_boiling1d_b200.inputs import bubble_density, face_beta, gaussian_rhs  # noqa: E402


def poisson1d_ship():
    n3m, m1, m2 = 256, 2, 2
    m3 = n3m + 1
    h = 1.0 / n3m
    denr, z0 = 1605.36, 0.0607
    # face density by the volume fraction of vapour (rho=1, below z0) over the face's
    # control volume [z_face - h/2, z_face + h/2]
    den = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
    for k in range(1, n3m + 1):
        zf = (k - 1) * h
        lo, hi = max(zf - 0.5 * h, 0.0), zf + 0.5 * h
        liq = np.clip((hi - max(lo, z0)) / (hi - lo), 0.0, 1.0)
        rho = 1.0 + (denr - 1.0) * liq
        den[:, :, k] = 1.0 / rho
    den[:, :, n3m + 1] = den[:, :, n3m]
    rng = np.random.default_rng(20240607)
    divg = np.asfortranarray(rng.standard_normal((m1 - 1, m2 - 1, m3 - 1)))
    p_in = np.asfortranarray(rng.standard_normal((m1 + 1, m2 + 1, m3 + 1)))
    M = np.zeros((n3m, n3m))
    for k in range(1, n3m + 1):
        vv_k = 2.0 / h if k == 1 else 1.0 / h
        vv_kp1 = 2.0 / h if k == n3m else 1.0 / h
        ak = vv_k / h * den[1, 1, k] * (0.0 if k == 1 else 1.0)
        ck = vv_kp1 / h * den[1, 1, k + 1]
        M[k - 1, k - 1] = -(ak + ck)
        if k > 1:
            M[k - 1, k - 2] = ak
        if k < n3m:
            M[k - 1, k] = ck
    x = np.linalg.solve(M, divg[0, 0, :n3m])
    p_out = p_in.copy(order="F")
    p_out[1, 1, 1:n3m + 1] = x
    p_out[1, 1, 0] = x[0]
    p_out[1, 1, n3m + 1] = x[-1]
    np.savez_compressed(os.path.join(HERE, "poisson1d_ship.npz"), n3m=n3m, p_in=p_in, divgsum=divg, denf_zi=den,
                        p_out=p_out)


def mg_bubbles64():
    n = 64
    h = 1.0 / n
    rho = bubble_density(n, n, nbubbles=8, rmin=2.0, rmax=8.0, seed=11)
    bx, by = face_beta(rho)
    f = gaussian_rhs(n, n, seed=12)
    N = n * n
    rows, cols, vals = [], [], []
    c = 1.0 / (h * h)
    for j in range(n):
        for i in range(n):
            r = j * n + i
            aw, ae = c * bx[j, i], c * bx[j, (i + 1) % n]
            as_ = c * by[j, i] if j > 0 else 0.0
            an = c * by[j + 1, i] if j < n - 1 else 2.0 * c * by[n, i]
            rows += [r, r, r]
            cols += [r, j * n + (i - 1) % n, j * n + (i + 1) % n]
            vals += [-(aw + ae + as_ + an), aw, ae]
            if j > 0:
                rows.append(r); cols.append((j - 1) * n + i); vals.append(as_)
            if j < n - 1:
                rows.append(r); cols.append((j + 1) * n + i); vals.append(an)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(N, N))
    p = spl.spsolve(A.tocsc(), f.ravel()).reshape(n, n)
    np.savez_compressed(os.path.join(HERE, "mg_bubbles64.npz"), f=f, bx=bx, by=by, rho=rho, p=p, h=h)


if __name__ == "__main__":
    poisson1d_ship()
    mg_bubbles64()
    print("written:", sorted(x for x in os.listdir(HERE) if x.endswith(".npz")))
