"""Non-uniform grids on the GPU: the POISSON drop-in on a stretched column against the
oracle bit for bit, and the multigrid on a stretched 2-D pressure system against a direct
sparse solve of the stretched operator."""
import numpy as np
import pytest

from oracle import grid as OG
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_poisson_drop_in_on_a_stretched_column():
    from lica_boiling1d_b200 import poisson as PP
    ny = 256
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, 2.0, 1.0, np.zeros(ny + 1))
    zc = 0.5 * (y[1:] + y[:-1])
    rho = np.where(zc < 0.0607, 1.0, 1605.36)
    g = PP.column_geometry(y)
    m1, m2, m3 = g["m1"], g["m2"], g["m3"]
    den = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
    for k in range(1, ny + 1):
        den[:, :, k] = 1.0 / (rho[0] if k == 1 else 0.5 * (rho[k - 1] + rho[k - 2]))
    den[:, :, ny + 1] = den[:, :, ny]
    rng = np.random.default_rng(9)
    divg = np.asfortranarray(rng.standard_normal((m1 - 1, m2 - 1, m3 - 1)))
    p0 = np.asfortranarray(rng.standard_normal((m1 + 1, m2 + 1, m3 + 1)))
    ref = O.poisson1d(g, p0, divg, den)
    P = p0.copy(order="F")
    PP.poisson(g, P, divg, den)
    np.testing.assert_array_equal(P, ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multigrid_on_a_stretched_system(precision):
    import scipy.sparse.linalg as spla
    from lica_boiling1d_b200 import poisson as PP
    nx = ny = 128
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, 1.5, 1.0, np.zeros(ny + 1))
    rng = np.random.default_rng(0)
    rho = np.where(rng.random((ny, nx)) < 0.2, 1.0, 40.0)
    bx = 1.0 / (0.5 * (rho + np.roll(rho, 1, axis=1)))
    by = np.ones((ny + 1, nx))
    by[1:ny] = 1.0 / (0.5 * (rho[1:] + rho[:-1]))
    by[0] = 1.0 / rho[0]
    by[ny] = 1.0 / rho[ny - 1]
    f = rng.standard_normal((ny, nx))
    bxs, bys, fs = PP.stretched_system(y, bx, by, f)
    x = spla.spsolve(OG.stretched_operator(y, bx, by, 1.0 / nx).tocsc(), f.ravel()).reshape(ny, nx)
    mg = PP.MultigridPoisson(nx, ny, 1.0 / nx, 1.0, nlevels=5, precision=precision)
    p = np.zeros((ny, nx))
    it, rel, st = mg.solve(p, fs, bxs, bys, rtol=1e-10, max_iters=200)
    mg.close()
    assert st == 0 and it < 50
    assert np.abs(p - x).max() <= 1e-9 * np.abs(x).max()


def _strong_stretch_system(nx, ny, gam, seed=0):
    from lica_boiling1d_b200 import poisson as PP
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, gam, 1.0, np.zeros(ny + 1))
    rng = np.random.default_rng(seed)
    rho = np.where(rng.random((ny, nx)) < 0.2, 1.0, 40.0)
    bx = 1.0 / (0.5 * (rho + np.roll(rho, 1, axis=1)))
    by = np.ones((ny + 1, nx))
    by[1:ny] = 1.0 / (0.5 * (rho[1:] + rho[:-1]))
    by[0] = 1.0 / rho[0]
    by[ny] = 1.0 / rho[ny - 1]
    f = rng.standard_normal((ny, nx))
    bxs, bys, fs = PP.stretched_system(y, bx, by, f)
    return y, bx, by, f, bxs, bys, fs


@pytest.mark.parametrize("n,nlevels,gam", [(128, 5, 3.0), (256, 6, 4.0), (64, 3, 1.5)])
def test_yline_preconditioner_bitwise(n, nlevels, gam):
    """smoother = 1 (y-line zebra relaxation): one V-cycle on a strongly stretched system
    is bit-identical to the oracle's cycle with flag MG_YLINE (sym = 13)."""
    import torch
    from lica_boiling1d_b200 import poisson as PP
    _, _, _, _, bxs, bys, fs = _strong_stretch_system(n, n, gam)
    ref = O.mg_precond(fs, bxs, bys, 1.0 / n, 1.0, nlevels=nlevels, ncoarse=2, sym=13)
    mg = PP.MultigridPoisson(n, n, 1.0 / n, 1.0, nlevels=nlevels, ncoarse=2, smoother="yline")
    z = torch.empty((n, n), dtype=torch.float64, device="cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    mg.precond(z, t(fs), t(bxs), t(bys))
    mg.close()
    np.testing.assert_array_equal(z.cpu().numpy(), ref)


@pytest.mark.parametrize("use_graph", [True, False])
def test_yline_solve_on_anisotropic_cells(use_graph):
    """Cells up to 33x finer in y than in x: the y-line cycle reaches 1e-10 in about 31
    iterations where red-black point smoothing needs about 139 (the oracle's counts), and
    both match a direct sparse solve of the stretched operator."""
    import scipy.sparse.linalg as spla
    from lica_boiling1d_b200 import poisson as PP
    n = 128
    y, bx, by, f, bxs, bys, fs = _strong_stretch_system(n, n, 3.0)
    dy = np.diff(y)
    assert (1.0 / n) / dy.min() > 30
    x = spla.spsolve(OG.stretched_operator(y, bx, by, 1.0 / n).tocsc(), f.ravel()).reshape(n, n)
    its = {}
    for sm in ("yline", "rb"):
        mg = PP.MultigridPoisson(n, n, 1.0 / n, 1.0, nlevels=5, ncoarse=2, smoother=sm, use_graph=use_graph)
        p = np.zeros((n, n))
        it, rel, st = mg.solve(p, fs, bxs, bys, rtol=1e-10, max_iters=400)
        mg.close()
        assert st == 0 and rel <= 1e-10, (sm, it, rel, st)
        assert np.abs(p - x).max() <= 1e-8 * np.abs(x).max(), sm
        its[sm] = it
    p_ref, it_ref, _, _, st_ref = O.mg_solve(fs, bxs, bys, 1.0 / n, 1.0, nlevels=5, ncoarse=2, sym=13, rtol=1e-10,
                                             max_cycles=400)
    assert st_ref == 0 and abs(its["yline"] - it_ref) <= 1
    assert its["yline"] * 2 <= its["rb"], its
