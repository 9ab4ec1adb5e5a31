"""The 2-D film-boiling restatement (oracle/film2d.py) on the CPU: the projection, the level-set
operators and the inputs the GPU step shares with it."""
import numpy as np
import pytest

from oracle import film2d as F

NX, NY = 64, 192


@pytest.fixture(scope="module")
def one_step():
    P = F.default_props()
    st = F.initial_state(NX, NY, y0_cells=8, amp_cells=2)
    dt = F.stable_dt(NX, P)
    s1, info = F.step(st, dt, P, F.oracle_mg(3, P["rtol"]))
    return P, st, dt, s1, info


def test_step_converges_and_stays_finite(one_step):
    P, st, dt, s1, info = one_step
    assert info["status"] == [0, 0, 0] and all(r <= P["rtol"] for r in info["rel"])
    for k, a in s1.items():
        assert np.isfinite(a).all(), k
    # a film from rest: velocities small, theta within [0, 1]
    assert np.abs(s1["u"]).max() < 0.1 and np.abs(s1["v"]).max() < 0.1
    assert s1["th"].min() >= 0.0 and s1["th"].max() <= 1.0


def test_projection_meets_the_volume_source(one_step):
    """After the correction div u = S of the last substep up to the solve's residual."""
    P, st, dt, s1, info = one_step
    D = F.Derived(NX, NY, P)
    div = F.divergence(s1["u"], s1["v"], D.h)
    S = info["S"]
    assert np.abs(S).max() > 0
    assert np.abs(div - S).max() <= 1e-6 * np.abs(S).max()


def test_mass_flux_only_at_the_interface(one_step):
    P, st, dt, s1, info = one_step
    md = info["mdot"]
    D = F.Derived(NX, NY, P)
    psi = F.properties(s1["phi"], D)[0]
    assert (md >= 0).all()
    # no flux in the pure liquid (theta = 0, grad theta = 0) or deep in the vapour (grad psi = 0)
    assert np.abs(md[psi == 1.0]).max() == 0.0
    assert np.abs(md[:2]).max() == 0.0


def test_transport_without_velocity_is_identity():
    D = F.Derived(NX, NY, F.default_props())
    phi = F.initial_state(NX, NY, y0_cells=8, amp_cells=2)["phi"]
    u = np.zeros((NY, NX))
    v = np.zeros((NY + 1, NX))
    uf, vf = F.refined_velocity(u, v)
    L = F.ls_rhs(phi, uf, vf, D)
    assert np.abs(L).max() == 0.0


def test_refined_velocity_is_exact_for_linear_fields():
    """Bilinear interpolation reproduces a field linear in x and y away from the walls."""
    h = 1.0 / NX
    y_u = (np.arange(NY) + 0.5) * h
    u = np.tile(0.3 + 2.0 * y_u[:, None], (1, NX))       # linear in y on the u rows
    y_v = np.arange(NY + 1) * h
    v = np.tile(-0.1 + 1.5 * y_v[:, None], (1, NX))      # linear in y on the v rows
    uf, vf = F.refined_velocity(u, v)
    yf = (np.arange(2 * NY) + 0.5) * 0.5 * h
    assert np.allclose(uf[2:-2], (0.3 + 2.0 * yf[2:-2])[:, None], rtol=0, atol=1e-13)
    assert np.allclose(vf, (-0.1 + 1.5 * yf)[:, None], rtol=0, atol=1e-13)


def test_weno_derivatives_are_fifth_order_on_a_smooth_field():
    D = F.Derived(NX, NY, F.default_props())
    xf = (np.arange(2 * NX) + 0.5) * D.hf
    phi = np.tile(np.sin(2 * np.pi * xf), (8, 1))
    dmx, dplx, *_ = F.weno_xy(phi, D)
    exact = 2 * np.pi * np.cos(2 * np.pi * xf)
    assert np.abs(dmx[3] - exact).max() < 1e-6 and np.abs(dplx[3] - exact).max() < 1e-6


def test_reinitialisation_keeps_a_signed_distance():
    D = F.Derived(NX, NY, dict(F.default_props(), nreinit=3))
    hf = D.hf
    yf = (np.arange(2 * NY) + 0.5) * hf
    phi = np.tile((yf - 0.3)[:, None], (1, 2 * NX))
    out = F.reinitialize(phi, D)
    assert np.abs(out - phi).max() < 1e-12


def test_reinitialisation_restores_unit_gradient():
    D = F.Derived(NX, NY, dict(F.default_props(), nreinit=8))
    yf = (np.arange(2 * NY) + 0.5) * D.hf
    phi = np.tile((2.0 * (yf - 0.3))[:, None], (1, 2 * NX))  # |grad phi| = 2, zero level y = 0.3
    out = F.reinitialize(phi, D)
    # the correction travels one pseudo-time unit per iteration (dtau = hf / 2): check the
    # cells within two refined cells of the interface
    band = np.abs(yf - 0.3) < 2 * D.hf
    g = np.gradient(out[:, 5], D.hf)
    assert np.abs(g[band] - 1.0).max() < 0.1
    # the zero level does not move
    assert np.abs(out[band, 5]).min() < D.hf


def test_product_inputs_match_the_restatement():
    from lica_boiling1d_b200 import film2d as G
    a = F.initial_state(NX, NY, y0_cells=8, amp_cells=2)
    b = G.initial_state(NX, NY, y0_cells=8, amp_cells=2)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert F.default_props() == G.default_props()


def test_curvature_of_a_circle():
    """CAL_CUR in 2-D on phi = r - R (vapour inside): CURF_TMP = -div(grad phi / |grad phi|) =
    -1/r on the band and 0 beyond it; CURF at the interface foot is -1/R within 2%;
    the face curvatures are -1/R on every face where psi jumps and 0 elsewhere."""
    nx, ny = 64, 64
    D = F.Derived(nx, ny, F.default_props())
    hf = D.hf
    xf = (np.arange(2 * nx) + 0.5) * hf
    yf = (np.arange(2 * ny) + 0.5) * hf
    R = 0.25
    r = np.sqrt((xf[None, :] - 0.5) ** 2 + (yf[:, None] - 0.5) ** 2)
    phi = r - R
    kt = F.curvature_refined(phi, D)
    band = np.abs(phi) < 5 * hf
    assert np.abs(kt[band] * r[band] + 1.0).max() < 1e-3
    assert np.all(kt[~band] == 0.0)
    cf = F.curvature_interface(phi, kt, D)
    near = np.abs(phi) < 4 * hf
    assert np.abs(cf[near] * R + 1.0).max() < 0.02
    assert np.all(cf[~near] == 0.0)
    psi = F.properties(phi, D)[0]
    cx, cy = F.curvature(phi, psi, D)
    jx = (psi - np.roll(psi, 1, axis=1)) != 0.0
    jy = np.zeros_like(jx)
    jy[1:] = (psi[1:] - psi[:-1]) != 0.0
    assert jx.sum() > 50 and jy.sum() > 50
    assert np.abs(cx[jx] * R + 1.0).max() < 0.005 and np.abs(cy[jy] * R + 1.0).max() < 0.005
    assert np.all(cx[~jx] == 0.0) and np.all(cy[~jy] == 0.0)


def test_cpp_restatement_is_bit_identical_to_numpy():
    """oracle/film2d.cpp (C++/OpenMP, the fast CPU baseline) reproduces the numpy restatement bit
    for bit over two steps (at this size the multigrid's reductions run serially)."""
    P = F.default_props()
    st = F.initial_state(NX, NY, y0_cells=8, amp_cells=2, props=P)
    dt = F.stable_dt(NX, P)
    a, b = st, st
    for _ in range(2):
        a, ia = F.step(a, dt, P, F.oracle_mg(3, P["rtol"]))
        b, ib = F.step_native(b, dt, P, 3)
        assert ia["iterations"] == ib["iterations"] and ib["status"] == [0, 0, 0]
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(ia["mdot"], ib["mdot"])


class _FirstSystem(Exception):
    pass


def test_pressure_solve_stops_at_fp64_floor_at_config_size():
    """At the config's 512 x 1536 the first substep's pressure increment is so large against
    its right-hand side (||A|| ||dp|| / ||f|| ~ 1e7) that FP64 cannot hold a solution with a
    1e-10 relative residual: rounding the converged increment by random half-ulps alone gives
    a residual above 1e-10.  The PCG then stops at that floor (LICA_STALLED, status 8) with
    the iterate before the residual rose, instead of diverging as an unguarded PCG does."""
    from oracle import oracle as orc
    nx, ny = 512, 1536
    P = F.default_props()
    st = F.initial_state(nx, ny, y0_cells=64, amp_cells=4)
    dt = F.stable_dt(nx, P)
    got = {}

    def capture(f, bx, by, h, p0):
        got.update(f=f, bx=bx, by=by, h=h)
        raise _FirstSystem

    with pytest.raises(_FirstSystem):
        F.step(st, dt, P, capture)
    f, bx, by, h = got["f"], got["bx"], got["by"], got["h"]
    p, it, rel, hist, status = orc.mg_solve(f, bx, by, h, h, nlevels=6, ncoarse=2, rtol=1e-10, max_cycles=60)
    assert status == 8 and 1e-10 < rel < 1e-9 and it <= 16, (status, rel, it)
    assert rel == hist[-1] == hist.min()
    rng = np.random.default_rng(0)
    delta = rng.uniform(-0.5, 0.5, p.shape) * np.spacing(np.abs(p))
    floor = np.linalg.norm(orc.mg_apply(delta, bx, by, h, h)) / np.linalg.norm(f)
    assert floor > 1e-10, floor
