"""GPU parity: the CUDA path, called through the C ABI, against the oracle.

Tolerances: the kernels follow the oracle's operation order without FMA contraction,
so single applications (operator, preconditioner, tridiagonal solves, POISSON) must
be bit-identical; solves differ only through the summation order of the CG dot
products and must agree to 1e-10 relative L2 (the pressure fields' tolerance), with the
true residual at or below the requested tolerance.
"""
import os

import numpy as np
import pytest

from oracle import oracle
from lica_boiling1d_b200 import native, poisson
from lica_boiling1d_b200.inputs import bubble_poisson_case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# ---------------------------------------------------------------- tridiagonal / POISSON
def _random_tridiag(ld, n, rng):
    A = rng.uniform(-1, 1, (ld, n))
    C = rng.uniform(-1, 1, (ld, n))
    B = rng.uniform(-1, 1, (ld, n)) + np.sign(rng.uniform(-1, 1, (ld, n))) * 3.0
    R = rng.standard_normal((ld, n))
    return [np.asfortranarray(x) for x in (A, B, C, R)]


@pytest.mark.parametrize("alias", [False, True])
def test_trdiag3_bitwise(alias):
    rng = np.random.default_rng(5)
    ld, n = 300, 129
    A, B, C, R = _random_tridiag(ld, n, rng)
    l1, l2, ll1, ll2 = 2, 128, 1, 297
    R_ref, UU_ref = oracle.trdiag3(A, B, C, R, l1, l2, ll1, ll2)
    Rg = R.copy(order="F")
    if alias:
        poisson.trdiag3(A, B, C, Rg, Rg, l1, l2, ll1, ll2)
        np.testing.assert_array_equal(Rg[ll1 - 1:ll2, l1 - 1:l2], UU_ref[ll1 - 1:ll2, l1 - 1:l2])
        np.testing.assert_array_equal(Rg[ll2:], R[ll2:])  # lines outside [ll1, ll2] untouched
    else:
        UUg = np.zeros_like(R, order="F")
        poisson.trdiag3(A, B, C, Rg, UUg, l1, l2, ll1, ll2)
        np.testing.assert_array_equal(UUg, UU_ref)
        np.testing.assert_array_equal(Rg, R_ref)


def test_trdiag3p_bitwise():
    rng = np.random.default_rng(6)
    ld, n = 200, 65
    A, B, C, F = _random_tridiag(ld, n, rng)
    ref = oracle.trdiag3p(A, B, C, F, 1, 64, 3, 190)
    Fg = F.copy(order="F")
    poisson.trdiag3p(A, B, C, Fg, 1, 64, 3, 190)
    np.testing.assert_array_equal(Fg, ref)


def test_poisson1d_shipped_column_bitwise_and_golden():
    d = np.load(os.path.join(GOLDEN, "poisson1d_ship.npz"))
    g = poisson.uniform_column_geometry(int(d["n3m"]))
    ref = oracle.poisson1d(g, d["p_in"], d["divgsum"], d["denf_zi"])
    P = d["p_in"].copy(order="F")
    poisson.poisson(g, P, d["divgsum"], d["denf_zi"])
    np.testing.assert_array_equal(P, ref)
    gold = d["p_out"]
    assert np.abs(P - gold).max() <= 1e-10 * np.abs(gold).max()


def test_poisson1d_rejects_3d_fields():
    g = poisson.uniform_column_geometry(32, m1=4, m2=2)
    P = np.zeros((5, 3, 34), order="F")
    with pytest.raises(native.LicaError):
        poisson.poisson(g, P, np.zeros((3, 1, 32), order="F"), np.ones((5, 3, 34), order="F"))


# ---------------------------------------------------------------- multigrid
def _solver(n, nlevels, precision="fp64", use_graph=True, ncoarse=2, ny=None):
    ny = n if ny is None else ny
    return poisson.MultigridPoisson(n, ny, 1.0 / n, 1.0 / n, nlevels=nlevels, ncoarse=ncoarse, precision=precision,
                                    use_graph=use_graph)


def test_operator_bitwise():
    import torch
    c = bubble_poisson_case(128)
    rng = np.random.default_rng(1)
    u = rng.standard_normal((128, 128))
    ref = oracle.mg_apply(u, c.bx, c.by, c.hx, c.hy)
    s = _solver(128, 3)
    out = torch.empty((128, 128), dtype=torch.float64, device="cuda")
    s.apply(out, _t(u), _t(c.bx), _t(c.by))
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("n,nlevels", [(128, 3), (256, 4), (1024, 6), (2048, 7)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_preconditioner_bitwise(n, nlevels, precision):
    """One V-cycle, bit-identical to the oracle's, from 128^2 (3 levels) to 2048^2 (7)."""
    import torch
    c = bubble_poisson_case(n)
    ref = oracle.mg_precond(c.f, c.bx, c.by, c.hx, c.hy, nlevels=nlevels, ncoarse=2, sym=5,
                            mixed=(precision == "mixed"))
    s = _solver(n, nlevels, precision)
    z = torch.empty((n, n), dtype=torch.float64, device="cuda")
    s.precond(z, _t(c.f), _t(c.bx), _t(c.by))
    np.testing.assert_array_equal(z.cpu().numpy(), ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cross_level_kernels_bitwise(monkeypatch, precision):
    """LICA_MG_CROSS_LEVEL=1: levels 1 .. 4 of each V-cycle leg in one cooperative launch with
    grid barriers (k_down_mid, k_up_mid); the preconditioner stays bit-identical to the
    oracle, and a graph-captured solve equals the per-level kernels' solve bit for bit."""
    import torch
    c = bubble_poisson_case(1024)
    ref = oracle.mg_precond(c.f, c.bx, c.by, c.hx, c.hy, nlevels=6, ncoarse=2, sym=5, mixed=(precision == "mixed"))
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("LICA_MG_CROSS_LEVEL", flag)
        s = _solver(1024, 6, precision)
        z = torch.empty((1024, 1024), dtype=torch.float64, device="cuda")
        s.precond(z, _t(c.f), _t(c.bx), _t(c.by))
        np.testing.assert_array_equal(z.cpu().numpy(), ref)
        p = torch.zeros((1024, 1024), dtype=torch.float64, device="cuda")
        it, rel, st = s.solve(p, _t(c.f), _t(c.bx), _t(c.by), rtol=TOL, max_iters=100)
        assert st == 0
        out[flag] = (it, rel, p.cpu().numpy())
        s.close()
    assert out["0"][0] == out["1"][0] and out["0"][1] == out["1"][1]
    np.testing.assert_array_equal(out["0"][2], out["1"][2])


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_matches_oracle_1024(use_graph, precision):
    import torch
    c = bubble_poisson_case(1024)
    mixed = precision == "mixed"
    p_ref, it_ref, rel_ref, _, st_ref = oracle.mg_solve(c.f, c.bx, c.by, c.hx, c.hy, nlevels=6, ncoarse=2, sym=5,
                                                       method="pcg", mixed=mixed, rtol=TOL, max_cycles=100)
    s = _solver(1024, 6, precision, use_graph)
    p = torch.zeros((1024, 1024), dtype=torch.float64, device="cuda")
    it, rel, st = s.solve(p, _t(c.f), _t(c.bx), _t(c.by), rtol=TOL, max_iters=100)
    assert st == 0 and st_ref == 0
    assert rel <= TOL
    assert abs(it - it_ref) <= 1, (it, it_ref)
    pg = p.cpu().numpy()
    assert np.linalg.norm(pg - p_ref) / np.linalg.norm(p_ref) <= TOL
    # the reported residual is the true FP64 residual
    r = c.f - oracle.mg_apply(pg, c.bx, c.by, c.hx, c.hy)
    assert np.linalg.norm(r) / np.linalg.norm(c.f) == pytest.approx(rel, rel=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_matches_oracle_2048(precision):
    """The 2048^2 solve of the mixed-precision config: same 64 bubbles (radii 16-96 cells),
    7 levels, 1e-10; the GPU solution within 1e-10 relative L2 of the oracle's."""
    import torch
    c = bubble_poisson_case(2048)
    mixed = precision == "mixed"
    p_ref, it_ref, rel_ref, _, st_ref = oracle.mg_solve(c.f, c.bx, c.by, c.hx, c.hy, nlevels=7, ncoarse=1, sym=5,
                                                       method="pcg", mixed=mixed, rtol=TOL, max_cycles=100)
    s = _solver(2048, 7, precision, ncoarse=1)
    p = torch.zeros((2048, 2048), dtype=torch.float64, device="cuda")
    it, rel, st = s.solve(p, _t(c.f), _t(c.bx), _t(c.by), rtol=TOL, max_iters=100)
    assert st == 0 and st_ref == 0
    assert rel <= TOL
    assert abs(it - it_ref) <= 1, (it, it_ref)
    pg = p.cpu().numpy()
    assert np.linalg.norm(pg - p_ref) / np.linalg.norm(p_ref) <= TOL


def test_solve_golden_sparse_direct():
    d = np.load(os.path.join(GOLDEN, "mg_bubbles64.npz"))
    s = _solver(64, 2)
    p = np.zeros((64, 64))
    it, rel, st = s.solve(p, d["f"], d["bx"], d["by"], rtol=1e-12, max_iters=100)
    assert st == 0
    assert np.linalg.norm(p - d["p"]) / np.linalg.norm(d["p"]) < 1e-9


def test_host_entry_matches_device_entry():
    import torch
    c = bubble_poisson_case(256)
    s = _solver(256, 4)
    ph = np.zeros((256, 256))
    it_h, rel_h, _ = s.solve(ph, c.f, c.bx, c.by, rtol=TOL)
    pd = torch.zeros((256, 256), dtype=torch.float64, device="cuda")
    it_d, rel_d, _ = s.solve(pd, _t(c.f), _t(c.bx), _t(c.by), rtol=TOL)
    assert it_h == it_d
    np.testing.assert_array_equal(ph, pd.cpu().numpy())


def test_repeat_solves_deterministic_and_warm_start():
    import torch
    c = bubble_poisson_case(512)
    s = _solver(512, 5)
    f, bx, by = _t(c.f), _t(c.bx), _t(c.by)
    p1 = torch.zeros((512, 512), dtype=torch.float64, device="cuda")
    p2 = torch.zeros_like(p1)
    r1 = s.solve(p1, f, bx, by)
    r2 = s.solve(p2, f, bx, by)
    assert r1 == r2 and torch.equal(p1, p2)
    # a converged solution as the initial guess needs no iteration
    it, rel, st = s.solve(p1, f, bx, by)
    assert st == 0 and it == 0 and rel <= TOL


def test_non_square_film_grid():
    c = bubble_poisson_case(512, ny=1536)
    p_ref, it_ref, _, _, _ = oracle.mg_solve(c.f, c.bx, c.by, c.hx, c.hy, nlevels=5, ncoarse=2, sym=5, method="pcg",
                                           rtol=TOL, max_cycles=100)
    s = poisson.MultigridPoisson(512, 1536, c.hx, c.hy, nlevels=5)
    p = np.zeros((1536, 512))
    it, rel, st = s.solve(p, c.f, c.bx, c.by, rtol=TOL)
    assert st == 0 and abs(it - it_ref) <= 1
    assert np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref) <= TOL


def test_status_not_converged_and_nan():
    c = bubble_poisson_case(128)
    s = _solver(128, 3)
    p = np.zeros((128, 128))
    it, rel, st = s.solve(p, c.f, c.bx, c.by, rtol=TOL, max_iters=2)
    assert st == 1 and it == 2
    f = c.f.copy()
    f[5, 7] = np.nan
    p = np.zeros((128, 128))
    with pytest.raises(native.LicaError) as e:
        s.solve(p, f, c.bx, c.by)
    assert e.value.code == 3


def test_bad_sizes_rejected():
    with pytest.raises(native.LicaError):
        poisson.MultigridPoisson(100, 64, 0.01, 0.01, nlevels=3)


def test_misaligned_device_arrays_rejected():
    import torch
    c = bubble_poisson_case(64)
    s = _solver(64, 2)
    buf = torch.zeros(64 * 64 + 1, dtype=torch.float64, device="cuda")
    p = buf[1:].view(64, 64)   # 8-byte offset: not 16-byte aligned
    with pytest.raises(native.LicaError) as e:
        s.solve(p, _t(c.f), _t(c.bx), _t(c.by))
    assert e.value.code == 4


def test_host_batch_matches_single_solves():
    """lica_mg_solve_host_batch (uploads and downloads overlapping the solves) gives each
    system exactly the single host-entry solution."""
    import torch
    from lica_boiling1d_b200 import poisson
    from lica_boiling1d_b200.inputs import bubble_poisson_case
    c = bubble_poisson_case(128, nbubbles=6, seed=3)
    s = poisson.MultigridPoisson(128, 128, c.hx, c.hy, nlevels=3)
    rng = np.random.default_rng(1)
    fs = [np.ascontiguousarray(c.f * (1.0 + 0.5 * k) + 0.01 * rng.standard_normal(c.f.shape)) for k in range(5)]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    ps = [pin(np.zeros_like(c.f)) for _ in fs]
    res = s.solve_batch(ps, [pin(f) for f in fs], [pin(c.bx)] * 5, [pin(c.by)] * 5, rtol=TOL)
    for k, f in enumerate(fs):
        q = np.zeros_like(c.f)
        it, rel, st = s.solve(q, f, c.bx, c.by, rtol=TOL)
        assert res[k][2] == 0 and res[k][0] == it
        np.testing.assert_array_equal(ps[k], q)
    s.close()


def test_solvers_of_different_sizes_coexist():
    """A solver keeps working after another, with smaller coarse levels, is created and
    destroyed (the coarse kernel's shared-memory cap is per function, not per solver)."""
    from lica_boiling1d_b200 import poisson
    from lica_boiling1d_b200.inputs import bubble_poisson_case
    big = bubble_poisson_case(256, nbubbles=8, seed=4)
    a = poisson.MultigridPoisson(256, 256, big.hx, big.hy, nlevels=4)
    p1 = np.zeros_like(big.f)
    it1, rel1, st1 = a.solve(p1, big.f, big.bx, big.by, rtol=TOL)
    small = bubble_poisson_case(64, ny=192, nbubbles=2, seed=5)
    b = poisson.MultigridPoisson(64, 192, small.hx, small.hy, nlevels=3)
    q = np.zeros_like(small.f)
    assert b.solve(q, small.f, small.bx, small.by, rtol=TOL)[2] == 0
    b.close()
    p2 = np.zeros_like(big.f)
    it2, rel2, st2 = a.solve(p2, big.f, big.bx, big.by, rtol=TOL)
    assert st1 == st2 == 0 and it1 == it2
    np.testing.assert_array_equal(p1, p2)
    a.close()
