"""The oracle's BUBBLE_TRACKING / BUBBLE_EIGENV / Jacobi_bub (oracle/bubble3d.cpp) against
known answers: numpy's symmetric eigensolver, an independent numpy restatement of the sums,
the moments of a sampled ellipsoid, the periodic z shift, the cylindrical record and an
empty level set."""
import numpy as np
import pytest

from lica_boiling1d_b200.bubbles import BubbleGrid, append_records, contact_times, format_records
from oracle import oracle
from tests import bubble_cases as bc


def _orc(grid, psi, u, v, w, **kw):
    return oracle.bubble_tracking(grid.as_dict(), psi, u, v, w, **kw)


@pytest.mark.parametrize("seed", range(6))
def test_jacobi_matches_eigh(seed):
    rng = np.random.default_rng(seed)
    q = np.linalg.qr(rng.standard_normal((3, 3)))[0]
    lam = np.sort(rng.uniform(0.1, 3.0, 3))
    a = q @ np.diag(lam) @ q.T
    d, x = oracle.jacobi3(a)
    ev = np.diag(d)
    assert np.allclose(np.sort(ev), lam, rtol=1e-10, atol=0)
    # the reference's stopping rule: squared off-diagonal sum <= 1e-12
    assert (d - np.diag(ev))[~np.eye(3, dtype=bool)].__pow__(2).sum() <= 1e-12
    assert np.abs(x.T @ x - np.eye(3)).max() < 1e-14
    assert np.abs(a @ x - x * ev).max() < 1e-5


def test_jacobi_diagonal_input_returns_at_once():
    d, x = oracle.jacobi3(np.diag([3.0, 1.0, 2.0]))
    assert np.array_equal(d, np.diag([3.0, 1.0, 2.0])) and np.array_equal(x, np.eye(3))


def test_sums_match_numpy_restatement():
    grid, psi, (u, v, w) = bc.three_bubbles()
    rec = _orc(grid, psi, u, v, w, time=0.25, llvs0=4)
    assert list(rec["llvs"]) == [4, 5, 6] and np.all(rec["time"] == 0.25)
    for q in range(3):
        ref = bc.numpy_tracking(grid, psi[q], u, v, w)
        r = rec[q]
        assert r["vol"] == pytest.approx(ref["vol"], rel=1e-13)
        assert np.allclose(r["col"][:3], ref["cen"], rtol=1e-13, atol=0)
        assert np.allclose(r["col"][3:6], ref["vel"], rtol=1e-11, atol=1e-15)
        assert np.allclose(np.sort(r["ami"]), np.linalg.eigvalsh(ref["ami"]), rtol=1e-9, atol=0)
        assert np.array_equal(r["vel"], r["col"][3:6])


def test_ellipsoid_moments():
    """A sampled ellipsoid: volume 4/3 pi abc, centroid at its centre, second moments a^2/5,
    b^2/5, c^2/5 along its axes; the aspect ratio a/c and the angles of the c axis."""
    grid = BubbleGrid.uniform(96, 96, 96, 1.0, 1.0, 1.0)
    axes = (0.30, 0.20, 0.12)
    rot = bc.rotation(0.0, np.deg2rad(30.0), 0.0)  # c axis tilted 30 degrees from z towards x
    psi = bc.ellipsoid_psi(grid, (0.5, 0.5, 0.5), axes, rot)[None]
    z = np.zeros(grid.field_shape)
    r = _orc(grid, psi, z, z, z)[0]
    assert r["vol"] == pytest.approx(4.0 / 3.0 * np.pi * np.prod(axes), rel=5e-3)
    assert np.allclose(r["col"][:3], 0.5, atol=1e-6)
    assert np.allclose(np.sort(r["ami"])[::-1], np.array(axes) ** 2 / 5.0, rtol=2e-2)
    assert r["col"][6] == pytest.approx(axes[0] / axes[2], rel=1e-2)
    # the c axis (smallest moment) is (sin 30, 0, cos 30): 60 degrees from x, 30 from z
    assert r["col"][7] == pytest.approx(60.0, abs=0.5)
    assert r["col"][8] == pytest.approx(30.0, abs=0.5)
    assert r["iz_periodic"] == 0


def test_periodic_z_shift():
    """A bubble across the z = 0 / ZL seam with IPZ = 1 has its centroid above ZL; the same
    bubble moved to mid-height has it at the moved centre, and the moments agree."""
    kw = dict(ipx=1, ipy=1, ipz=1)
    grid = BubbleGrid.uniform(32, 32, 64, 1.0, 1.0, 2.0, **kw)
    axes, rot = (0.2, 0.15, 0.3), bc.rotation(0.2, 0.3, 0.0)
    seam = bc.ellipsoid_psi(grid, (0.5, 0.5, 0.1), axes, rot, zshift=(0.0, 2.0, -2.0))[None]
    mid = bc.ellipsoid_psi(grid, (0.5, 0.5, 1.1), axes, rot)[None]
    z = np.zeros(grid.field_shape)
    a, b = _orc(grid, seam, z, z, z)[0], _orc(grid, mid, z, z, z)[0]
    assert a["iz_periodic"] == 1 and b["iz_periodic"] == 0
    assert a["vol"] == pytest.approx(b["vol"], rel=1e-12)
    assert a["col"][2] == pytest.approx(b["col"][2] + 1.0, abs=1e-9)
    assert np.allclose(a["ami"], b["ami"], rtol=1e-9)
    # without IPZ the seam bubble is two halves: centroid near mid-height, not above ZL
    grid0 = BubbleGrid.uniform(32, 32, 64, 1.0, 1.0, 2.0, ipz=0)
    c = _orc(grid0, seam, z, z, z)[0]
    assert 0.5 < c["col"][2] < 1.5


def test_cylindrical_record():
    grid, psi, (u, v, w) = bc.three_bubbles(seed=3)
    grid.xp = grid.xp - 0.6  # centre the box on the axis so the bubbles sit in several quadrants
    grid.yp = grid.yp - 0.5
    c1 = _orc(grid, psi, u, v, w, icacy=1)
    c2 = _orc(grid, psi, u, v, w, icacy=2)
    for r1, r2 in zip(c1, c2):
        x, y = r1["col"][0], r1["col"][1]
        assert r2["col"][0] == pytest.approx(np.hypot(x, y), rel=1e-14)
        assert r2["col"][1] == pytest.approx(np.arctan2(y, x) % (2 * np.pi), rel=1e-13)
        t = r2["col"][1]
        assert r2["col"][3] == pytest.approx(r1["col"][3] * np.cos(t) + r1["col"][4] * np.sin(t), rel=1e-12)
        assert r2["col"][4] == pytest.approx(-r1["col"][3] * np.sin(t) + r1["col"][4] * np.cos(t), rel=1e-12)
        assert np.allclose(r2["col"][5:], r1["col"][5:], rtol=1e-9)
        assert np.array_equal(r2["vel"], r1["vel"])


def test_uniform_velocity_and_empty_level_set():
    grid = BubbleGrid.uniform(24, 20, 16, 1.0, 1.0, 1.0)
    psi = np.stack([bc.ellipsoid_psi(grid, (0.5, 0.5, 0.5), (0.3, 0.2, 0.1)), np.ones(grid.field_shape)])
    one = np.ones(grid.field_shape)
    r = _orc(grid, psi, one, 2 * one, 3 * one)
    assert np.allclose(r[0]["col"][3:6], [1.0, 2.0, 3.0], rtol=1e-14)
    e = r[1]
    assert e["vol"] == 0.0 and np.all(e["col"][:6] == 0.0) and np.all(e["ami"] == 0.0)
    assert np.isnan(e["col"][6])  # sqrt(0/0), as the reference's formulas give
    assert e["col"][7] == pytest.approx(90.0, abs=1e-12) and e["col"][8] == 0.0


def test_column_grid():
    """N1M = N2M = 1, the reference's own 1-D column: the gas volume is the vapour length."""
    n = 64
    grid = BubbleGrid.uniform(1, 1, n, 1.0, 1.0, 1.0, ipx=1, ipy=1)
    psi = np.ones((1,) + grid.field_shape)
    psi[0, 1:21, 1, 1] = 0.0
    psi[0, 21, 1, 1] = 0.25
    z = np.zeros(grid.field_shape)
    r = _orc(grid, psi, z, z, z)[0]
    assert r["vol"] == pytest.approx((20 + 0.75) / n, rel=1e-14)
    assert r["col"][0] == pytest.approx(0.5, rel=1e-14)


def test_format_records():
    rec = np.zeros(1, dtype=oracle.BUB_RECORD)
    rec["time"], rec["llvs"], rec["col"] = 1.5, 3, np.arange(9) * 0.5
    line = format_records(rec)[0]
    assert len(line) == 15 + 5 + 9 * 15
    assert line.startswith("  1.5000000E+00    3  0.0000000E+00  5.0000000E-01")


def test_append_records(tmp_path):
    """Two calls append two lines each, in the reference's record format."""
    grid, psi, (u, v, w) = bc.three_bubbles()
    rec = _orc(grid, psi[:2], u, v, w, time=0.5, llvs0=1)
    path = tmp_path / "0bub_tracking.dat"
    append_records(path, rec)
    append_records(path, rec)
    lines = path.read_text().splitlines()
    assert lines == format_records(rec) * 2
    assert [int(x[15:20]) for x in lines] == [1, 2, 1, 2]
    assert float(lines[0][20:35]) == pytest.approx(rec[0]["col"][0], rel=1e-7)


def test_contact_times():
    """CAL_TCON on three bubbles: symmetric, the smaller original volume sets the length, and a
    known case: relative speed 5 (a velocity difference of (0, 3, -4)), volume pi/6 * 8 (a
    sphere of diameter 2), SURF_J 0.5 -> 0.5 * 25 * 0.5 (8 pi / 3.14159)^(1/3)."""
    rec = np.zeros(3, dtype=oracle.BUB_RECORD)
    rec["vel"][0] = [1.0, 2.0, 0.0]
    rec["vel"][1] = [1.0, -1.0, 4.0]
    rec["vel"][2] = [1.0, 2.0, 0.0]
    vol = np.array([np.pi / 6 * 8, np.pi / 6 * 27, 1.0])
    t = contact_times(rec, vol, 0.5)
    assert np.array_equal(t, t.T) and np.all(np.diag(t) == 0.0)
    assert t[0, 1] == pytest.approx(0.5 * 25.0 * 0.5 * (8 * np.pi / 3.14159) ** (1 / 3), rel=1e-14)
    assert t[0, 2] == 0.0  # same velocity
    assert t[1, 2] == pytest.approx(0.5 * 25.0 * 0.5 * (6 / 3.14159) ** (1 / 3), rel=1e-14)


def test_host_api_rejects_bad_shapes():
    """The bubble API checks shapes before it reaches the GPU."""
    from lica_boiling1d_b200 import bubbles
    grid = BubbleGrid.uniform(8, 6, 4, 1.0, 1.0, 1.0)
    fs = grid.field_shape
    good = np.ones(fs)
    with pytest.raises(ValueError):
        bubbles.track(grid, np.ones((2,) + fs[:-1] + (fs[-1] + 1,)), good, good, good)
    with pytest.raises(ValueError):
        bubbles.track(grid, np.ones((1,) + fs), good, good, np.ones(fs[::-1]))
    with pytest.raises(ValueError):
        bubbles.track(grid, np.ones(fs), good, good, good)  # no level-set axis
    bad = BubbleGrid.uniform(8, 6, 4, 1.0, 1.0, 1.0)
    bad.sdy = np.ones(3)
    with pytest.raises(ValueError):
        bad._c()
    rec = np.zeros(2, dtype=bubbles.RECORD)
    with pytest.raises(ValueError):
        bubbles.contact_times(rec, [1.0], 0.1)
