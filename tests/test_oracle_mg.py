"""Known-answer tests that pin the oracle's 2-D multigrid (new build; the reference's
POISSON is 1-D).  The operator is checked for symmetry and definiteness, the solver
against scipy's sparse direct solve (golden fixture) and the exact 1-D solution."""
import os

import numpy as np
import pytest

from oracle import oracle
from lica_boiling1d_b200.inputs import bubble_poisson_case, face_beta, gaussian_rhs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PCG = dict(sym=5, method="pcg")   # symmetric smoothing + piecewise-constant prolongation


def _matrix(nx, ny, h, bx, by):
    n = nx * ny
    A = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        A[:, k] = oracle.mg_apply(e.reshape(ny, nx), bx, by, h, h).ravel()
    return A


def test_operator_symmetric_negative_definite():
    nx, ny = 8, 6
    rho = np.ones((ny, nx))
    rho[2:4, 3:6] = 1000.0
    bx, by = face_beta(rho)
    A = _matrix(nx, ny, 1.0 / nx, bx, by)
    np.testing.assert_allclose(A, A.T, rtol=0, atol=1e-9 * np.abs(A).max())
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).max() < 0


def test_operator_reduces_to_reference_1d_column():
    # with beta constant along x, a field constant in x sees the 1-D operator of
    # POISSON (1d.f:3535-3541): AK = beta_k/h^2 (0 at k=1), CK = beta_{k+1}/h^2 (2x at top)
    nx, ny = 4, 16
    h = 1.0 / ny
    rng = np.random.default_rng(0)
    bcol = rng.uniform(0.001, 1.0, ny + 1)
    bx = np.ones((ny, nx))
    by = np.repeat(bcol[:, None], nx, axis=1)
    u = np.repeat(rng.standard_normal(ny)[:, None], nx, axis=1)
    Au = oracle.mg_apply(u, bx, by, h, h)
    col = u[:, 0]
    ref = np.zeros(ny)
    for k in range(ny):
        ak = bcol[k] / h**2 if k > 0 else 0.0
        ck = bcol[k + 1] / h**2 * (2.0 if k == ny - 1 else 1.0)
        ref[k] = -(ak + ck) * col[k] + (ak * col[k - 1] if k > 0 else 0.0) + (ck * col[k + 1] if k < ny - 1 else 0.0)
    np.testing.assert_allclose(Au[:, 0], ref, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("mixed", [False, True])
def test_pcg_matches_sparse_direct_solve(mixed):
    d = np.load(os.path.join(GOLDEN, "mg_bubbles64.npz"))
    h = float(d["h"])
    p, cyc, rel, hist, st = oracle.mg_solve(d["f"], d["bx"], d["by"], h, h, nlevels=2, ncoarse=2, rtol=1e-12,
                                           max_cycles=60, mixed=mixed, **PCG)
    assert st == 0 and rel <= 1e-12
    err = np.linalg.norm(p - d["p"]) / np.linalg.norm(d["p"])
    assert err < 1e-9, err


def test_pcg_bubbles_1024_converges_in_few_iterations():
    c = bubble_poisson_case(256)
    p, cyc, rel, hist, st = oracle.mg_solve(c.f, c.bx, c.by, c.hx, c.hy, nlevels=4, ncoarse=2, rtol=1e-10,
                                           max_cycles=60, **PCG)
    assert st == 0 and rel <= 1e-10 and cyc <= 30, (cyc, rel)
    r = c.f - oracle.mg_apply(p, c.bx, c.by, c.hx, c.hy)
    assert np.linalg.norm(r) / np.linalg.norm(c.f) <= 1e-10


def test_vcycle_constant_coefficient_rate():
    n = 64
    rho = np.ones((n, n))
    bx, by = face_beta(rho)
    f = gaussian_rhs(n, n)
    p, cyc, rel, hist, st = oracle.mg_solve(f, bx, by, 1 / n, 1 / n, nlevels=3, sym=0, method="vcycle",
                                           max_cycles=30)
    assert st == 0 and cyc <= 12
    assert np.max(hist[2:] / hist[1:-1]) < 0.2


def test_mixed_precond_close_to_fp64():
    c = bubble_poisson_case(128)
    z64 = oracle.mg_precond(c.f, c.bx, c.by, c.hx, c.hy, nlevels=3, sym=5, mixed=False)
    z32 = oracle.mg_precond(c.f, c.bx, c.by, c.hx, c.hy, nlevels=3, sym=5, mixed=True)
    err = np.linalg.norm(z64 - z32) / np.linalg.norm(z64)
    assert 0 < err < 1e-5, err


def test_status_codes():
    c = bubble_poisson_case(64)
    _, cyc, rel, _, st = oracle.mg_solve(c.f, c.bx, c.by, c.hx, c.hy, nlevels=2, max_cycles=0, **PCG)
    assert st == 1 and cyc == 0 and rel == pytest.approx(1.0)
    f = c.f.copy()
    f[3, 3] = np.nan
    _, _, _, _, st = oracle.mg_solve(f, c.bx, c.by, c.hx, c.hy, nlevels=2, max_cycles=5, **PCG)
    assert st == 3
    _, cyc, rel, _, st = oracle.mg_solve(np.zeros_like(c.f), c.bx, c.by, c.hx, c.hy, nlevels=2, **PCG)
    assert st == 0 and cyc == 0 and rel == 0.0
