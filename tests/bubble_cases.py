"""Seeded 3-D level-set fields for the bubble-statistics tests: rotated ellipsoidal bubbles
with a smeared edge (PSI_TMP = 0 inside, 1 outside, fractions in between), velocity fields,
and a numpy restatement of BUBBLE_TRACKING / BUBBLE_EIGENV's sums (two_phase.f:6321-6705)
written independently of the C oracle, to check it.
"""
import numpy as np

from lica_boiling1d_b200.bubbles import BubbleGrid


def rotation(ax, ay, az):
    cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ ry @ rx


def ellipsoid_psi(grid: BubbleGrid, centre, axes, rot=np.eye(3), zshift=(0.0,)):
    """PSI_TMP of an ellipsoid (semi-axes `axes` along the columns of `rot`), edge smeared over
    about one cell; zshift lists copies displaced in z (periodic images)."""
    z, y, x = np.meshgrid(grid.zp, grid.yp, grid.xp, indexing="ij")
    h = min(grid.sdx[1], grid.sdy[1], grid.sdz[1])
    psi = np.ones(grid.field_shape)
    for dz in zshift:
        d = np.stack([x - centre[0], y - centre[1], z - centre[2] - dz], axis=-1) @ rot
        r = np.sqrt(((d / np.asarray(axes)) ** 2).sum(-1))
        phi = (r - 1.0) * min(axes)
        psi = np.minimum(psi, np.clip(0.5 + phi / (1.5 * h), 0.0, 1.0))
    # ghost layers: the reference never reads PSI_TMP there
    psi[0], psi[-1], psi[:, 0], psi[:, -1], psi[:, :, 0], psi[:, :, -1] = 1, 1, 1, 1, 1, 1
    return psi


def velocity(grid: BubbleGrid, seed):
    rng = np.random.default_rng(seed)
    return tuple(rng.standard_normal(grid.field_shape) for _ in range(3))


def numpy_tracking(grid: BubbleGrid, psi, u, v, w):
    """VOL, the centroid (x, y, z), the velocity (u, v, w) and the second-moment matrix about
    the centroid, as BUBBLE_TRACKING (icacy 1) and BUBBLE_EIGENV define them."""
    n1, n2, n3 = grid.n1m, grid.n2m, grid.n3m
    P = psi[1:n3 + 1, 1:n2 + 1, 1:n1 + 1]
    gas = P != 1.0
    vf = (1.0 - P) * grid.sdx[None, None, 1:n1 + 1] * grid.sdy[None, 1:n2 + 1, None] * grid.sdz[1:n3 + 1, None, None]
    vf = np.where(gas, vf, 0.0)
    iz = bool(gas[-1].any())
    zp = grid.zp[1:n3 + 1].copy()
    if grid.ipz == 1 and iz:
        zp = np.where(zp <= 0.5 * grid.zl, zp + grid.zl, zp)
    X = np.broadcast_to(grid.xp[None, None, 1:n1 + 1], P.shape)
    Y = np.broadcast_to(grid.yp[None, 1:n2 + 1, None], P.shape)
    Z = np.broadcast_to(zp[:, None, None], P.shape)
    ip = np.arange(2, n1 + 2)
    ip[-1] = 1 if grid.ipx else n1 + 1
    jp = np.arange(2, n2 + 2)
    jp[-1] = 1 if grid.ipy else n2 + 1
    kp = np.arange(2, n3 + 2)
    kp[-1] = 1 if grid.ipz else n3 + 1
    I, J, K = np.arange(1, n1 + 1), np.arange(1, n2 + 1), np.arange(1, n3 + 1)
    uc = 0.5 * (u[np.ix_(K, J, I)] + u[np.ix_(K, J, ip)])
    vc = 0.5 * (v[np.ix_(K, J, I)] + v[np.ix_(K, jp, I)])
    wc = 0.5 * (w[np.ix_(K, J, I)] + w[np.ix_(kp, J, I)])
    vol = vf.sum()
    if vol == 0.0:
        return {"vol": 0.0, "cen": np.zeros(3), "vel": np.zeros(3), "ami": np.zeros((3, 3)), "iz": iz}
    cen = np.array([(X * vf).sum(), (Y * vf).sum(), (Z * vf).sum()]) / vol
    vel = np.array([(uc * vf).sum(), (vc * vf).sum(), (wc * vf).sum()]) / vol
    D = [X - cen[0], Y - cen[1], Z - cen[2]]
    ami = np.array([[(D[a] * D[b] * vf).sum() for b in range(3)] for a in range(3)]) / vol
    return {"vol": vol, "cen": cen, "vel": vel, "ami": ami, "iz": iz}


def three_bubbles(n1=48, n2=40, n3=56, seed=0, ipz=0):
    """Three rotated ellipsoids of distinct axes in a 1.2 x 1.0 x 1.4 box, velocity noise."""
    grid = BubbleGrid.uniform(n1, n2, n3, 1.2, 1.0, 1.4, ipx=1, ipy=1, ipz=ipz)
    psi = np.stack([
        ellipsoid_psi(grid, (0.40, 0.45, 0.50), (0.22, 0.15, 0.09), rotation(0.3, 0.5, 0.2)),
        ellipsoid_psi(grid, (0.85, 0.55, 0.95), (0.14, 0.18, 0.26), rotation(-0.4, 0.1, 0.9)),
        ellipsoid_psi(grid, (0.60, 0.30, 0.25), (0.10, 0.16, 0.12), rotation(1.1, -0.7, 0.4)),
    ])
    return grid, psi, velocity(grid, seed)
