"""Non-uniform grids (lica_grid_*, lica_mg_stretched_system; host code): the generator's
sections and GEOMETRIC's metrics against the oracle bit for bit and against their known
answers, grid.in / grid.dat handling, POISSON on a stretched column against its dense
operator, and the stretched 2-D pressure system solved by the multigrid against a direct
sparse solve and against the reference's 1-D POISSON."""
import numpy as np
import pytest

from oracle import grid as OG
from oracle import oracle as O

SHIPPED_GRID_IN = """ISPARE_NSE_X    ISPARE_NSE_Y    ISPARE_LVS_X   ISPARE_LVS_Y
0               0               0              0
##NAVIER-STOKES GRID##
NSECT   N1      N2    N3      XL      YL      ZL
3       2       2     257      1.      1.      1.
IDIR    XYZI    XYZF    NGI     NGF     IOPT    ER(GAM) YESEXP(XSI)
1       0.      1.      1       2       1       1.      1.
2       0.      1.      1       2       1       1.      1.
3       0.      1.      1       257     1       1.      1.
##LEVEL-SET G_GRID##
NSECT   N1F     N2F     N3F     XL      YL      ZL
3       3       3       513     1.      1.      1.
IDIR    XYZI    XYZF    NGI     NGF     IOPT    ER(GAM) YESEXP(XSI)
4       0.      1.      1       3       1       1.      1.
5       0.      1.      1       3       1       1.      1.
6       0.      1.      1       513     1       1.      1.
"""

SECTIONS = [(1, 0.0, 1.0, 1, 257, 1.0, 1.0), (1, -0.5, 2.0, 3, 40, 1.0, 1.0), (2, 0.0, 1.0, 1, 129, 1.03, 1.0),
            (2, 0.0, 2.0, 1, 65, 1.05, 0.0), (3, 0.0, 1.0, 1, 257, 2.5, 1.0), (3, 0.0, 1.0, 1, 129, 3.0, 0.5),
            (3, 0.0, 1.0, 1, 129, 2.0, 0.0), (7, 1.0, 3.0, 5, 70, 1.7, 1.0)]


@pytest.mark.parametrize("args", SECTIONS)
def test_sections_match_the_oracle(args):
    from lica_boiling1d_b200 import grid as G
    iopt, xi, xf, ngi, ngf, f1, f2 = args
    a = np.full(ngf, -7.0)
    G.section(G.Section(3, xi, xf, ngi, ngf, iopt, f1, f2), a)
    b = OG.section(*args, np.full(ngf, -7.0))
    assert np.array_equal(a, b)
    assert np.all(a[:ngi - 1] == -7.0)                # points before the section untouched
    assert abs(a[ngi - 1] - xi) <= 1e-15 and abs(a[ngf - 1] - xf) <= 1e-14
    assert np.all(np.diff(a[ngi - 1:]) > 0)


def test_section_known_answers():
    from lica_boiling1d_b200 import grid as G
    x = np.zeros(129)
    G.section(G.Section(3, 0.0, 1.0, 1, 129, 2, 1.03, 1.0), x)         # expansion 1.03
    d = np.diff(x)
    np.testing.assert_allclose(d[1:] / d[:-1], 1.03, rtol=1e-9)
    np.testing.assert_allclose(d[0], 0.03 / (1.03 ** 128 - 1.0), rtol=1e-12)
    G.section(G.Section(3, 0.0, 1.0, 1, 129, 2, 1.03, 0.0), x)         # compression
    d = np.diff(x)
    np.testing.assert_allclose(d[1:] / d[:-1], 1 / 1.03, rtol=1e-9)
    G.section(G.Section(3, 0.0, 1.0, 1, 129, 3, 3.0, 0.5), x)          # channel: symmetric
    np.testing.assert_allclose(x + x[::-1], 1.0, atol=1e-15)
    G.section(G.Section(3, 0.0, 1.0, 1, 129, 3, 2.0, 1.0), x)          # flat plate: fine at the wall
    d = np.diff(x)
    assert np.all(np.diff(d) > 0) and d[-1] / d[0] > 3.0
    G.section(G.Section(3, 0.0, 1.0, 1, 129, 3, 2.0, 0.0), x)          # XSI = 0: fine at the far end
    np.testing.assert_allclose(x, np.tanh(2.0 * np.arange(129) / 128) / np.tanh(2.0), rtol=0, atol=1e-15)
    with pytest.raises(Exception):
        G.section(G.Section(3, 0.0, 1.0, 1, 129, 2, 1.0, 1.0), x)      # ER = 1 stops the generator


def test_shipped_grid_in_is_the_uniform_column(tmp_path):
    from lica_boiling1d_b200 import grid as G
    from lica_boiling1d_b200 import poisson as PP
    p = tmp_path / "grid.in"
    p.write_text(SHIPPED_GRID_IN)
    spec = G.read_grid_in(str(p))
    assert spec["flow"]["n"] == (2, 2, 257) and spec["levelset"]["n"] == (3, 3, 513)
    xyz = G.generate(spec)
    assert np.array_equal(xyz[3], np.arange(257) / 256.0)
    assert np.array_equal(xyz[6], np.arange(513) / 512.0)
    g = PP.column_geometry(xyz[3])
    u = PP.uniform_column_geometry(256)
    for k, v in u.items():
        assert np.array_equal(np.asarray(g[k]), np.asarray(v)), k
    out = tmp_path / "grid.dat"
    G.write_grid_dat(str(out), spec, xyz)
    lines = out.read_text().splitlines()
    assert lines[0] == "%23d%23d%23d" % (2, 2, 257)
    assert lines[1] == "1.000000000000000".rjust(23) * 3
    assert lines[2] == "  0.000000000000000E+00  1.000000000000000E+00"
    vals = [float(t) for ln in lines for t in ln.split()]
    assert len(vals) == 3 + 3 + 2 + 2 + 257 + 3 + 3 + 3 + 3 + 513
    np.testing.assert_array_equal(vals[10:267], xyz[3])


def test_metrics_match_the_oracle():
    from lica_boiling1d_b200 import grid as G
    for args in SECTIONS[:7]:
        z = OG.section(*args, np.zeros(args[4]))[args[3] - 1:]
        a, b = G.metrics(z), OG.metrics(z)
        for k in a:
            assert np.array_equal(a[k], b[k]), (args, k)
        n = len(z)
        assert a["vdz"][1] == 0.5 * a["sdz"][1] and a["vdz"][n] == 0.5 * a["sdz"][n - 1]
        assert a["zp"][0] == z[0] and a["zp"][n] == z[-1]


def _stretched_column(ny, gam, ratio=40.0, z0=0.1, zl=1.0):
    y = OG.section(3, 0.0, zl, 1, ny + 1, gam, 1.0, np.zeros(ny + 1))
    zc = 0.5 * (y[1:] + y[:-1])
    rho = np.where(zc < z0, 1.0, ratio)
    byc = np.empty(ny + 1)
    byc[1:ny] = 1.0 / (0.5 * (rho[1:] + rho[:-1]))
    byc[0] = 1.0 / rho[0]
    byc[ny] = 1.0 / rho[ny - 1]
    return y, zc, rho, byc


def test_poisson_on_a_stretched_column():
    """POISSON (1d.f:3492-3578) with GEOMETRIC's metrics of a tanh grid: the solution of
    the tridiagonal operator AK / CK = VVDZ SSDZ DENF_ZI (1d.f:3535-3541)."""
    from lica_boiling1d_b200 import poisson as PP
    ny = 96
    y, zc, rho, byc = _stretched_column(ny, 2.0)
    g = PP.column_geometry(y)
    m1, m2, m3 = g["m1"], g["m2"], g["m3"]
    den = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
    for k in range(1, ny + 1):
        den[:, :, k] = byc[k - 1]
    den[:, :, ny + 1] = byc[ny]
    divg = np.zeros((m1 - 1, m2 - 1, m3 - 1), order="F")
    divg[0, 0, :] = np.cos(3.0 * zc) - 0.3
    P = O.poisson1d(g, np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F"), divg, den)
    vv, ss = g["vvdz"], g["ssdz"]
    M = np.zeros((ny, ny))
    for k in range(1, ny + 1):
        ak = vv[k - 1] * ss[k] * den[1, 1, k] * (0.0 if k == 1 else 1.0)
        ck = vv[k] * ss[k] * den[1, 1, k + 1]
        M[k - 1, k - 1] = -(ak + ck)
        if k > 1:
            M[k - 1, k - 2] = ak
        if k < ny:
            M[k - 1, k] = ck
    x = np.linalg.solve(M, divg[0, 0, :ny])
    np.testing.assert_allclose(P[1, 1, 1:ny + 1], x, rtol=0, atol=1e-10 * np.abs(x).max())


def _bubbly(nx, ny, seed=0, ratio=40.0):
    rng = np.random.default_rng(seed)
    rho = np.where(rng.random((ny, nx)) < 0.2, 1.0, ratio)
    bx = 1.0 / (0.5 * (rho + np.roll(rho, 1, axis=1)))
    by = np.ones((ny + 1, nx))
    by[1:ny] = 1.0 / (0.5 * (rho[1:] + rho[:-1]))
    by[0] = 1.0 / rho[0]
    by[ny] = 1.0 / rho[ny - 1]
    return bx, by, rng.standard_normal((ny, nx))


def test_stretched_system_matches_the_oracle_and_a_direct_solve():
    """The library's rescaling equals the oracle's bit for bit, and the multigrid's solution
    of it is the solution of the stretched operator assembled directly (cells of aspect
    ratio up to 3.3, density ratio 40; the product's cycle: symmetric smoothing and
    piecewise-constant prolongation)."""
    import scipy.sparse.linalg as spla
    from lica_boiling1d_b200 import poisson as PP
    nx = ny = 128
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, 1.5, 1.0, np.zeros(ny + 1))
    bx, by, f = _bubbly(nx, ny)
    a = PP.stretched_system(y, bx, by, f)
    b = OG.stretched_system(y, bx, by, f)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    x = spla.spsolve(OG.stretched_operator(y, bx, by, 1.0 / nx).tocsc(), f.ravel()).reshape(ny, nx)
    p, cyc, rel, _, st = O.mg_solve(b[2], b[0], b[1], 1.0 / nx, 1.0, nlevels=5, ncoarse=2, sym=5, rtol=1e-10,
                                    max_cycles=200)
    assert st == 0 and cyc < 50
    assert np.abs(p - x).max() <= 1e-9 * np.abs(x).max()


def test_stretched_multigrid_reduces_to_poisson():
    """x-independent data: every column of the 2-D stretched solution is the reference's
    1-D POISSON solution on the same faces."""
    from lica_boiling1d_b200 import poisson as PP
    nx = ny = 64
    y = OG.section(2, 0.0, 1.0, 1, ny + 1, 1.01, 1.0, np.zeros(ny + 1))
    zc = 0.5 * (y[1:] + y[:-1])
    rho = np.where(zc < 0.1, 1.0, 40.0)
    byc = np.empty(ny + 1)
    byc[1:ny] = 1.0 / (0.5 * (rho[1:] + rho[:-1]))
    byc[0] = 1.0 / rho[0]
    byc[ny] = 1.0 / rho[ny - 1]
    fc = np.cos(3.0 * zc) - 0.3
    bx = np.tile((1.0 / rho)[:, None], (1, nx))
    by = np.tile(byc[:, None], (1, nx))
    f = np.tile(fc[:, None], (1, nx))
    s = PP.stretched_system(y, bx, by, f)
    p, cyc, rel, _, st = O.mg_solve(s[2], s[0], s[1], 1.0 / nx, 1.0, nlevels=5, ncoarse=2, sym=5, rtol=1e-11,
                                    max_cycles=200)
    assert st == 0 and cyc < 50
    g = PP.column_geometry(y)
    m1, m2, m3 = g["m1"], g["m2"], g["m3"]
    den = np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F")
    for k in range(1, ny + 1):
        den[:, :, k] = byc[k - 1]
    den[:, :, ny + 1] = byc[ny]
    divg = np.zeros((m1 - 1, m2 - 1, m3 - 1), order="F")
    divg[0, 0, :] = fc
    P = O.poisson1d(g, np.zeros((m1 + 1, m2 + 1, m3 + 1), order="F"), divg, den)
    assert np.abs(p - P[1, 1, 1:ny + 1][:, None]).max() <= 1e-9 * np.abs(P).max()


def test_bad_grids_rejected():
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200 import grid as G
    from lica_boiling1d_b200 import poisson as PP
    with pytest.raises(native.LicaError):
        G.metrics(np.array([0.0, 0.5, 0.5, 1.0]))
    y = np.array([0.0, 0.2, 0.1, 1.0])
    with pytest.raises(native.LicaError):
        PP.stretched_system(y, np.ones((3, 4)), np.ones((4, 4)), np.ones((3, 4)))


YLINE = 13   # symmetric smoothing + piecewise-constant prolongation + y-line relaxation


def test_yline_relaxation_solves_decoupled_columns_in_one_cycle():
    """With no x coupling every column is one tridiagonal system: one V-cycle whose
    smoother solves y-lines exactly leaves only rounding (the point smoother leaves 40%)."""
    ny, nx = 64, 32
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, 3.0, 1.0, np.zeros(ny + 1))
    bx, by, f = _bubbly(nx, ny, seed=4)
    s = OG.stretched_system(y, 0.0 * bx, by, f)
    rels = {}
    for flags in (5, YLINE):
        _, cyc, rels[flags], _, st = O.mg_solve(s[2], s[0], s[1], 1.0 / nx, 1.0, nlevels=3, ncoarse=2, sym=flags,
                                                method="vcycle", rtol=1e-16, max_cycles=1)
        assert cyc == 1
    assert rels[YLINE] < 1e-11 and rels[5] > 0.1


def test_yline_preconditioner_is_symmetric():
    """PCG needs a symmetric preconditioner: <M r1, r2> = <r1, M r2>."""
    nx, ny = 64, 64
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, 3.0, 1.0, np.zeros(ny + 1))
    bx, by, f = _bubbly(nx, ny, seed=5)
    s = OG.stretched_system(y, bx, by, f)
    rng = np.random.default_rng(6)
    r1, r2 = rng.standard_normal((2, ny, nx))
    z1 = O.mg_precond(r1, s[0], s[1], 1.0 / nx, 1.0, nlevels=4, ncoarse=2, sym=YLINE)
    z2 = O.mg_precond(r2, s[0], s[1], 1.0 / nx, 1.0, nlevels=4, ncoarse=2, sym=YLINE)
    a, b = np.vdot(z1, r2), np.vdot(r1, z2)
    assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))


@pytest.mark.parametrize("gam", [2.5, 4.0, 5.0])
def test_yline_relaxation_keeps_the_rate_on_anisotropic_cells(gam):
    """Wall cells 15 to 1000 times finer in y than in x: point relaxation needs 85 to more
    than 300 PCG iterations; y-line relaxation converges in under 50, to the direct solve."""
    import scipy.sparse.linalg as spla
    nx = ny = 128
    y = OG.section(3, 0.0, 1.0, 1, ny + 1, gam, 1.0, np.zeros(ny + 1))
    assert (1.0 / nx) / np.diff(y).min() > 14
    bx, by, f = _bubbly(nx, ny)
    s = OG.stretched_system(y, bx, by, f)
    x = spla.spsolve(OG.stretched_operator(y, bx, by, 1.0 / nx).tocsc(), f.ravel()).reshape(ny, nx)
    p, cyc, rel, _, st = O.mg_solve(s[2], s[0], s[1], 1.0 / nx, 1.0, nlevels=5, ncoarse=2, sym=YLINE, rtol=1e-10,
                                    max_cycles=200)
    assert st == 0 and cyc < 50
    assert np.abs(p - x).max() <= 1e-9 * np.abs(x).max()


def _coupling_grids(n=48):
    zf = np.arange(2 * n + 1) / (2.0 * n)
    return zf, {
        "uniform": np.arange(n + 1) / float(n),
        "tanh": OG.section(3, 0.0, 1.0, 1, n + 1, 2.0, 1.0, np.zeros(n + 1)),
        "geometric": OG.section(2, 0.0, 1.0, 1, n + 1, 1.03, 1.0, np.zeros(n + 1)),
        # faces on refined faces, 1 to 3 refined cells per flow cell
        "snapped": np.concatenate([[0.0], np.cumsum(np.resize([1, 2, 3], n))]) / np.cumsum(np.resize([1, 2, 3], n))[-1],
    }


def test_coupling_tables_match_the_oracle():
    from lica_boiling1d_b200 import grid as G
    zf, grids = _coupling_grids()
    for name, z in grids.items():
        zz = z if name != "snapped" else np.round(z * 96) / 96
        a, b = G.coupling_z(zz, zf), OG.coupling_z(zz, zf)
        for k in a:
            assert np.array_equal(a[k], b[k]), (name, k)


def test_coupling_tables_of_the_uniform_column():
    """The uniform column's closed forms: flow cell K covers refined cells 2K-1..2K, face K's
    box 2K-2..2K-1, and KCOUMP_VEL(k) is the flow centre at or below the refined centre."""
    from lica_boiling1d_b200 import grid as G
    n = 64
    t = G.coupling_z(np.arange(n + 1) / n, np.arange(2 * n + 1) / (2.0 * n))
    K = np.arange(1, n + 1)
    assert np.array_equal(t["kcou2"][K + 1], 2 * K - 1) and np.array_equal(t["kcou1"][K + 2], 2 * K)
    K = np.arange(2, n + 1)
    assert np.array_equal(t["kcoump2"][K], 2 * K - 2) and np.array_equal(t["kcoump1"][K + 1], 2 * K - 1)
    k = np.arange(1, 2 * n + 1)
    zpf = (k - 0.5) / (2.0 * n)
    assert np.array_equal(t["kcoump_vel"][1:2 * n + 1], np.clip(np.floor(zpf * n + 0.5), 1, n).astype(np.int32))


def test_box_means_over_stretched_flow_cells():
    """INTER_PSI's box over flow cell K (refined cells KCOU2(K)..KCOU1(K+1)) is the
    overlap-weighted mean of the refined values, for faces on and off the refined faces,
    and the flow-cell means conserve the refined field's integral."""
    from lica_boiling1d_b200 import grid as G
    zf, grids = _coupling_grids()
    rng = np.random.default_rng(3)
    nf = len(zf) - 1
    f = np.concatenate([[0.0], rng.random(nf)])
    for name, z in grids.items():
        if name == "snapped":
            z = np.round(z * 96) / 96
        t = G.coupling_z(z, zf)
        total = 0.0
        for K in range(1, len(z)):
            z1, z2 = z[K - 1], z[K]
            m = OG.box_mean(f, zf, int(t["kcou2"][K + 1]), int(t["kcou1"][K + 2]), z1, z2)
            ov = np.clip(np.minimum(zf[1:], z2) - np.maximum(zf[:-1], z1), 0.0, None)
            assert abs(m - (ov * f[1:]).sum() / ov.sum()) <= 1e-13, (name, K)
            total += m * (z2 - z1)
        assert abs(total - f[1:].sum() / nf) <= 1e-13, name


def test_coupling_rejects_a_flow_grid_beyond_the_level_set():
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200 import grid as G
    with pytest.raises(native.LicaError):
        G.coupling_z(np.linspace(0.0, 1.2, 33), np.linspace(0.0, 1.0, 65))
