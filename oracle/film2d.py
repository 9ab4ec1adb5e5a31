"""ORACLE (test infrastructure only): CPU restatement, in numpy, of one RK3 time step of the
2-D film-boiling model run by lica_boiling1d_b200/csrc/film2d.cu.  Only tests/ and bench.py's
CPU leg use it.

The reference is a 1-D code; this step generalises its hot-path rows to 2-D (x periodic, y
the reference's wall-normal z):
  * RK3 substeps with RK3COEF's coefficients (1d.f:1310-1322), every right-hand side stored
    for the next substep (RK3ZO / the LS RK3 storage);
  * properties mixed linearly in the liquid fraction psi as in the reference's DEN/VIS/DENSC/
    TC = m + (p - m) * psi (1d.f:437-489, CAL_CONTINUITY), psi from the refined level set
    (the analogue of GRID_COUPLING / CAL_PSIF, two_phase.f:2503-5538) through a smoothed
    Heaviside (quintic, no transcendental functions);
  * momentum: explicit central convection, the full variable-viscosity stress and gravity
    (the 2-D analogue of RHSZ / LHSW, 1d.f:1603-1809, treated explicitly).  The pressure is
    the modified pressure p + rho_l g y, so the body force is g (rho_l / rho - 1) (zero in
    the liquid, buoyancy in the vapour): the liquid column's hydrostatic pressure would
    otherwise dominate p and put the projection's attainable relative residual (about
    5e-10 at a 1000:1 density ratio) above the 1e-10 tolerance;
  * projection, incremental: the predictor carries -alpha dt beta grad p of the current
    pressure, div(beta grad dp) = (div u* - S) / (alpha dt) is solved for the increment from
    zero with the 2-D multigrid's operator (mg2d.cpp; beta = 1/rho on faces by harmonic mean,
    Neumann bottom, p = 0 on the top face, x periodic), then u = u* - alpha dt beta grad dp
    and p += dp (PRESSURE_CORRECTION).  Solving for the whole pressure instead puts the
    buoyancy's divergence into every right-hand side and leaves the PCG short of 1e-10 at
    512 x 1536;
  * phase change: mdot = Ja / (Re Pr) * k * max(0, -grad(theta) . grad(psi)) and the volume
    source S = mdot (1/rho_v - 1/rho_l) (the smeared analogue of TEMP_GRAD / TF_GRAD /
    VOL_TOT_MFDOT and CAL_CONTINUITY2's source);
  * energy: central advection and conservative diffusion of theta = (T - T_sat) / dT_wall,
    theta = 1 on the wall face, zero gradient at the top, theta = 0 (saturation) in cells
    with psi > 1/2 (the analogue of PASSIVE_SCALAR / TEMPASSIGN);
  * level set: TRANSPORT_RK3 with the reference's HJWENO derivatives (two_phase.f:
    1133-1495, 2477-2500) in x and y, velocity bilinearly interpolated from the MAC faces to
    the refined centres (VEL_INTP's role), simple upwinding by the sign of each component;
  * reinitialisation: REINITIALIZATION's SSP-RK3 pseudo-time iterations with GODUNOV and
    Peng's smoothed sign (two_phase.f:2033-2474);
  * both on the band |phi| < 8 refined cells (BAND_GENERATION's role, two_phase.f:1622-2030):
    cells outside keep their value (the properties see phi only within one flow cell of the
    interface).
  * surface tension: CAL_CUR / CAL_CUR_INTEGRAL / INTER_CUR (two_phase.f:3317-4432) in 2-D:
    the curvature of the refined level set on the band by central differences, carried to the
    foot of each band cell on the interface (bilinear interpolation), averaged per flow face
    over the interface cells of the face's box, and applied as SURF CUR dpsi/dx / rho_f on the
    faces where psi jumps (SURF = 1/We).
Documented simplifications: the interface recession term of the phase change is not applied
(the interface moves with the one-fluid velocity, which carries the expansion flow of S),
and the viscous terms are explicit.

Every expression is written in the CUDA kernels' evaluation order (left to right, explicit
parentheses; the kernels are compiled without FMA contraction), so all fields agree bit for
bit except through the iterative pressure solve, which both sides converge to the same
relative residual.  film2d.cpp restates this file in C++/OpenMP (step_native): bit-identical to
step() wherever the multigrid's OpenMP reductions run serially (below 65536 cells), and the
fast CPU baseline.

Layout (row-major, x fastest): u (ny, nx) on the face west of cell i; v (ny + 1, nx) on the
face below cell row j (v[0] = 0 wall, v[ny] top); p, theta (ny, nx); phi (2 ny, 2 nx).
"""
import numpy as np

GAMMA = (0.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
RO = (0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0)

def default_props():
    """The 2-D film-boiling benchmark's liquid/vapour ratios (Welch and Wilson's case: rho 200/5,
    mu 0.1/0.005, k 40/1, c_p 400/200, h_fg 1e4, superheat 5 K): density 40, viscosity 20,
    conductivity 40, specific heat 2, Ja = c_p,v dT / h_fg = 0.1, Pr_v = 1, and Re = 69.2 and
    Fr = 1 on the velocity sqrt(g Lx) with Lx the most dangerous Rayleigh-Taylor wavelength
    (0.0787 m), We = rho_v U^2 Lx / sigma = 3.04 (sigma 0.1 N/m).  The pressure solves stop at
    a relative residual of 1e-10, or at FP64's attainable accuracy where that lies above it
    (LICA_STALLED): at 512 x 1536 the phase-change source leaves a pressure increment so large
    against its right-hand side (||A|| ||dp|| / ||f|| ~ 1e7) that rounding the exact increment to
    FP64 alone gives a relative residual of 1.6e-10, and the solves end near 3e-10 after about
    12 iterations.  At 64 x 192 the floor is 6e-12 and 1e-10 is met in 9."""
    return dict(re=69.2, visr=20.0, denr=40.0, prm=1.0, scr=2.0, tcr=40.0, jakob=0.1, fr=1.0, we=3.04,
                rtol=1e-10, nreinit=2)


class Derived:
    """Constants of the step (the same expressions as Const in film2d.cu)."""

    def __init__(self, nx, ny, props):
        P = props
        self.nx, self.ny = nx, ny
        self.h = 1.0 / nx
        self.hf = 0.5 * self.h
        self.ih = 1.0 / self.h
        self.ih2 = 2.0 / self.h
        self.inv2h = 0.5 / self.h
        self.ihsq = 1.0 / (self.h * self.h)
        self.ihf = 1.0 / self.hf
        self.eps_h = self.h
        self.inv2e = 1.0 / (2.0 * self.eps_h)
        self.denm = 1.0
        self.den_diff = P["denr"] - 1.0
        self.vism = 1.0 / P["re"]
        self.vis_diff = P["visr"] / P["re"] - 1.0 / P["re"]
        self.denscm = 1.0
        self.densc_diff = P["denr"] * P["scr"] - 1.0
        self.tcm = 1.0
        self.tc_diff = P["tcr"] - 1.0
        self.pei = 1.0 / (P["re"] * P["prm"])
        self.cmd = P["jakob"] * self.pei
        self.cvol = 1.0 / 1.0 - 1.0 / P["denr"]
        self.gravity = 0.0 if P["fr"] == 0.0 else 1.0 / (P["fr"] * P["fr"])
        self.denp = P["denr"]
        self.surf = 0.0 if P.get("we", 0.0) == 0.0 else 1.0 / P["we"]
        self.ih2f = 0.5 / self.hf
        self.ihfsq = 1.0 / (self.hf * self.hf)
        self.q4 = 0.25 * self.ihfsq
        self.nreinit = int(P["nreinit"])
        self.band = 8.0 * self.hf  # transport / reinitialisation band |phi| < band (BAND_GENERATION's role)
        self.rtol = P["rtol"]


def initial_state(nx, ny, y0_cells=64.0, amp_cells=4.0, props=None):
    """The film: interface y = y0 h + amp h cos(2 pi x) (Lx = 1, h = 1/nx), phi = y - y_i(x) on
    the refined centres (liquid where phi > 0); theta linear in the vapour from 1 at the wall to
    0 at the interface and 0 in the liquid; u = v = 0; p the discrete hydrostatic (modified)
    pressure of the initial density field, which balances the buoyancy g (rho_l / rho_f - 1) on
    every face with the projection's own face density rho_f = (rho_below + rho_above) / 2 (top
    face: p = 0 half a cell above the last row), so the first pressure solve starts from the
    balanced state.  Host numpy arrays."""
    h = 1.0 / nx
    hf = 0.5 * h
    xf = (np.arange(2 * nx) + 0.5) * hf
    yf = (np.arange(2 * ny) + 0.5) * hf
    yi_f = y0_cells * h + amp_cells * h * np.cos(2.0 * np.pi * xf)
    phi = np.ascontiguousarray(yf[:, None] - yi_f[None, :])
    xc = (np.arange(nx) + 0.5) * h
    yc = (np.arange(ny) + 0.5) * h
    yi_c = y0_cells * h + amp_cells * h * np.cos(2.0 * np.pi * xc)
    th = np.maximum(0.0, 1.0 - yc[:, None] / yi_c[None, :])
    z = np.zeros((ny, nx))
    P = default_props() if props is None else props
    g = 0.0 if P["fr"] == 0.0 else 1.0 / (P["fr"] * P["fr"])
    denp = P["denr"]
    # density per cell from the smoothed Heaviside of phi (the step's property rule)
    eps = h
    s = (phi + eps) * (1.0 / (2.0 * eps))
    H = np.where(phi <= -eps, 0.0, np.where(phi >= eps, 1.0, s * s * s * (10.0 + s * (-15.0 + 6.0 * s))))
    psi = 0.25 * ((H[0::2, 0::2] + H[0::2, 1::2]) + (H[1::2, 0::2] + H[1::2, 1::2]))
    den = 1.0 + (denp - 1.0) * psi
    p = np.zeros((ny, nx))
    p[ny - 1] = 0.0 - (0.5 * h) * (g * (denp - den[ny - 1]))
    for j in range(ny - 1, 0, -1):
        p[j - 1] = p[j] - h * (g * (denp - 0.5 * (den[j - 1] + den[j])))
    return dict(u=z.copy(), v=np.zeros((ny + 1, nx)), p=p, th=th, phi=phi)


def stable_dt(nx, props, cfl=0.2):
    """Explicit limits from rest: viscous and thermal diffusion (fastest phase) and the
    gravity wave time sqrt(h / g); cfl times the smallest."""
    D = Derived(nx, nx, props)
    nu = max(D.vism / D.denm, (D.vism + D.vis_diff) / (D.denm + D.den_diff))
    al = D.pei * max(D.tcm / D.denscm, (D.tcm + D.tc_diff) / (D.denscm + D.densc_diff))
    lim = [0.25 * D.h * D.h / nu, 0.25 * D.h * D.h / al]
    if D.gravity > 0.0:
        lim.append(np.sqrt(D.h / D.gravity))
    return cfl * min(lim)


# ----------------------------------------------------------------------------- helpers
def _e(a):
    return np.roll(a, -1, axis=1)


def _w(a):
    return np.roll(a, 1, axis=1)


def heaviside(x, D):
    s = (x + D.eps_h) * D.inv2e
    poly = s * s * s * (10.0 + s * (-15.0 + 6.0 * s))
    return np.where(x <= -D.eps_h, 0.0, np.where(x >= D.eps_h, 1.0, poly))


def properties(phi, D):
    """psi, den, vis, densc, tc per flow cell and the face coefficients bx, by = 1/rho."""
    H = heaviside(phi, D)
    psi = 0.25 * ((H[0::2, 0::2] + H[0::2, 1::2]) + (H[1::2, 0::2] + H[1::2, 1::2]))
    den = D.denm + D.den_diff * psi
    vis = D.vism + D.vis_diff * psi
    densc = D.denscm + D.densc_diff * psi
    tc = D.tcm + D.tc_diff * psi
    bx = 2.0 / (_w(den) + den)
    ny = den.shape[0]
    by = np.empty((ny + 1, den.shape[1]))
    by[0] = 1.0 / den[0]
    by[1:ny] = 2.0 / (den[:-1] + den[1:])
    by[ny] = 1.0 / den[ny - 1]
    return psi, den, vis, densc, tc, bx, by


def _rows_s(a, bottom):
    """a shifted so that row j holds a[j - 1]; row 0 holds `bottom`."""
    out = np.empty_like(a)
    out[1:] = a[:-1]
    out[0] = bottom
    return out


def _rows_n(a, top):
    """a shifted so that row j holds a[j + 1]; the last row holds `top`."""
    out = np.empty_like(a)
    out[:-1] = a[1:]
    out[-1] = top
    return out


def mass_source(th, psi, tc, D):
    """Volume source S = mdot (1/rho_v - 1/rho_l) per cell, and mdot."""
    ts = _rows_s(th, 2.0 - th[0])
    tn = _rows_n(th, th[-1])
    ps = _rows_s(psi, psi[0])
    pn = _rows_n(psi, psi[-1])
    gtx = (_e(th) - _w(th)) * D.inv2h
    gty = (tn - ts) * D.inv2h
    gpx = (_e(psi) - _w(psi)) * D.inv2h
    gpy = (pn - ps) * D.inv2h
    q = -(gtx * gpx + gty * gpy)
    md = (D.cmd * tc) * np.maximum(q, 0.0)
    return md * D.cvol, md


N_CUR = 4   # CAL_CUR(4, ...) (two_phase.f:2792): kappa on band layers 1..N_CUR+1, CURF on 1..N_CUR


def _nbrs(a):
    """E, W (x periodic), N, S (y indices clamped) and the four corners of a refined array."""
    nj = a.shape[0]
    idx = np.arange(nj)
    up = a[np.minimum(idx + 1, nj - 1)]
    dn = a[np.maximum(idx - 1, 0)]
    E, W = np.roll(a, -1, axis=1), np.roll(a, 1, axis=1)
    return E, W, up, dn, np.roll(up, -1, axis=1), np.roll(up, 1, axis=1), np.roll(dn, -1, axis=1), \
        np.roll(dn, 1, axis=1)


def curvature_refined(phi, D):
    """CAL_CUR's CURF_TMP (two_phase.f:3362-3397) in 2-D: kappa = -(GXX GZ^2 + GZZ GX^2 -
    2 GXZ GX GZ) / |grad phi|^3 from central differences on the refined grid, on the band
    layers 1..N_CUR+1 (|phi| < (N_CUR+1) hf), 0 elsewhere and where grad phi vanishes.  The
    reference's y terms are exactly zero for a field that does not vary in y; |g|^3 is
    evaluated as g2 sqrt(g2)."""
    E, W, N, S, NE, NW, SE, SW = _nbrs(phi)
    gx = 0.5 * (E - W) * D.ihf
    gz = 0.5 * (N - S) * D.ihf
    gxx = ((E - 2.0 * phi) + W) * D.ihf * D.ihf
    gzz = ((N - 2.0 * phi) + S) * D.ihf * D.ihf
    gxz = 0.25 * ((NE - NW) - (SE - SW)) * D.ihf * D.ihf
    g2 = gx * gx + gz * gz
    num = (gxx * (gz * gz) + gzz * (gx * gx)) - 2.0 * (gxz * gx * gz)
    ok = (np.abs(phi) < (N_CUR + 1) * D.hf) & (g2 > 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(ok, -num / (g2 * np.sqrt(g2)), 0.0)


def curvature_interface(phi, kt, D):
    """CAL_CUR's CURF (two_phase.f:3405-3458) in 2-D: kappa at the foot of each band cell
    (layers 1..N_CUR) on the interface, x_base = x - phi n, interpolated bilinearly from
    CURF_TMP (the reference's trilinear form with YD = 0); 0 off those layers."""
    nj, ni = phi.shape
    E, W, N, S = _nbrs(phi)[:4]
    dpx = 0.5 * (E - W) * D.ihf
    dpz = 0.5 * (N - S) * D.ihf
    g2 = dpx * dpx + dpz * dpz
    ok = (np.abs(phi) < N_CUR * D.hf) & (g2 > 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        amdpi = 1.0 / np.sqrt(g2)
    dis = phi * amdpi
    I = np.arange(ni)[None, :]
    J = np.arange(nj)[:, None]
    xp = (I + 0.5) * D.hf
    zp = (J + 0.5) * D.hf
    xb = xp - dis * (dpx * amdpi)
    zb = zp - dis * (dpz * amdpi)
    hx, hz = xb >= xp, zb >= zp
    xd = np.where(hx, (xb - xp) * D.ihf, (xb - (xp - D.hf)) * D.ihf)
    zd = np.where(hz, (zb - zp) * D.ihf, (zb - (zp - D.hf)) * D.ihf)
    Ie, Iw = (I + 1) % ni, (I - 1) % ni
    Jn, Js = np.minimum(J + 1, nj - 1), np.maximum(J - 1, 0)
    i1 = np.where(hx, I, Iw)
    i2 = np.where(hx, Ie, I)
    j1 = np.where(hz, J, Js)
    j2 = np.where(hz, Jn, J)
    with np.errstate(invalid="ignore"):
        c00 = kt[j1, i1] * (1.0 - xd) + kt[j1, i2] * xd
        c01 = kt[j2, i1] * (1.0 - xd) + kt[j2, i2] * xd
        out = c00 * (1.0 - zd) + c01 * zd
    return np.where(ok, out, 0.0)


def _box(val, cnt, rows, cols):
    """INTER_CUR's sums over the refined cells rows x cols (lists of index arrays), column by
    column and row by row within a column, as the reference's II / KK loops run."""
    s = np.zeros(val[rows[0], cols[0]].shape)
    v = np.zeros_like(s)
    for c in cols:
        for r in rows:
            s = s + val[r, c]
            v = v + cnt[r, c]
    return s, v


def face_curvature(phi, cf, psi, D):
    """CAL_CUR's face loops with CAL_CUR_INTEGRAL / INTER_CUR (two_phase.f:3547-3590,
    3654-4432) in 2-D: on every face where psi jumps, the mean of CURF over the refined cells
    of the face's box (centre to centre across the face, face to face along it) that are cut
    by the interface (0 < psi_f < 1, CURF /= 0); if none is, the box twice as wide across the
    face; 0 where psi does not jump.  On the uniform 2x refinement the boxes are whole refined
    cells, so every weight is 1.  Returns (cx on the u faces (ny, nx), cy on the v faces
    below each row (ny, nx), row 0 the wall: 0)."""
    ny, nx = psi.shape
    nxf = 2 * nx
    H = heaviside(phi, D)
    cnt = ((H > 0.0) & (H < 1.0) & (cf != 0.0)).astype(np.float64)
    val = np.where(cnt > 0.0, cf, 0.0)
    i = np.arange(nx)[None, :]
    j = np.arange(ny)[:, None]
    # u faces: x box refined columns 2i-1..2i (fallback 2i-2..2i+1), rows 2j..2j+1
    rows = [2 * j, 2 * j + 1]
    s, v = _box(val, cnt, rows, [(2 * i - 1) % nxf, (2 * i) % nxf])
    s2, v2 = _box(val, cnt, rows, [(2 * i + q) % nxf for q in (-2, -1, 0, 1)])
    with np.errstate(divide="ignore", invalid="ignore"):
        cur = np.where(v != 0.0, s / v, np.where(v2 != 0.0, s2 / v2, 0.0))
    cx = np.where((psi - _w(psi)) != 0.0, cur, 0.0)
    # v faces j = 1..ny-1: columns 2i..2i+1, rows 2j-1..2j (fallback 2j-2..2j+1)
    jj = np.maximum(j, 1)
    cols = [2 * i, 2 * i + 1]
    s, v = _box(val, cnt, [2 * jj - 1, 2 * jj], cols)
    s2, v2 = _box(val, cnt, [2 * jj + q for q in (-2, -1, 0, 1)], cols)
    with np.errstate(divide="ignore", invalid="ignore"):
        cur = np.where(v != 0.0, s / v, np.where(v2 != 0.0, s2 / v2, 0.0))
    cy = np.where((j >= 1) & ((psi - _rows_s(psi, psi[0])) != 0.0), cur, 0.0)
    return cx, cy


def curvature(phi, psi, D):
    """CAL_CUR in 2-D: (cx, cy) face curvatures from the refined level set."""
    kt = curvature_refined(phi, D)
    cf = curvature_interface(phi, kt, D)
    return face_curvature(phi, cf, psi, D)


def momentum_u(u, v, den, vis, D, psi=None, cx=None):
    ih = D.ih
    ue, uw = _e(u), _w(u)
    un = _rows_n(u, u[-1])
    us = _rows_s(u, -u[0])
    vw = _w(v)
    vn = 0.5 * (vw[1:] + v[1:])
    vs = 0.5 * (vw[:-1] + v[:-1])
    uci = 0.5 * (u + ue)
    ucm = 0.5 * (uw + u)
    conv = (uci * uci - ucm * ucm) * ih + (0.5 * (u + un) * vn - 0.5 * (us + u) * vs) * ih
    visw = _w(vis)
    vis_n = _rows_n(vis, vis[-1])
    vis_s = _rows_s(vis, vis[0])
    txe = 2.0 * vis * (ue - u) * ih
    txw = 2.0 * visw * (u - uw) * ih
    mun = 0.25 * ((visw + vis) + (_w(vis_n) + vis_n))
    mus = 0.25 * ((_w(vis_s) + vis_s) + (visw + vis))
    tyn = mun * ((un - u) * ih + (v[1:] - vw[1:]) * ih)
    tys = mus * ((u - us) * ih + (v[:-1] - vw[:-1]) * ih)
    rho = 0.5 * (_w(den) + den)
    visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho
    if cx is None:
        return visc - conv
    # surface tension SURF CUR dpsi/dx on the face (CAL_CUR's SUR_X, two_phase.f:3547-3556)
    return visc - conv + (D.surf * cx) * ((psi - _w(psi)) * ih) / rho


def momentum_v(u, v, den, vis, D, psi=None, cy=None):
    """Right-hand side on the faces j = 1..ny (returned as ny rows)."""
    ih = D.ih
    vc = v[1:]
    vsv = v[:-1]
    vnv = _rows_n(vc, vc[-1])
    ve, vw = _e(vc), _w(vc)
    ulo = u
    uhi = _rows_n(u, u[-1])
    ulo_e, uhi_e = _e(ulo), _e(uhi)
    vcj = 0.5 * (vc + vnv)
    vcm = 0.5 * (vsv + vc)
    conv = ((0.5 * (ulo_e + uhi_e)) * (0.5 * (vc + ve)) - (0.5 * (ulo + uhi)) * (0.5 * (vw + vc))) * ih + \
        (vcj * vcj - vcm * vcm) * ih
    mulo = vis
    muhi = _rows_n(vis, vis[-1])
    tyn = 2.0 * muhi * (vnv - vc) * ih
    tys = 2.0 * mulo * (vc - vsv) * ih
    mue = 0.25 * ((mulo + _e(mulo)) + (muhi + _e(muhi)))
    muw = 0.25 * ((_w(mulo) + mulo) + (_w(muhi) + muhi))
    txe = mue * ((ve - vc) * ih + (uhi_e - ulo_e) * ih)
    txw = muw * ((vc - vw) * ih + (uhi - ulo) * ih)
    dlo = den
    dhi = _rows_n(den, den[-1])
    rho = 0.5 * (dlo + dhi)
    visc = ((txe - txw) * ih + (tyn - tys) * ih) / rho
    if cy is None:
        return visc - conv + D.gravity * (D.denp / rho - 1.0)
    # the face above row j carries cy of row j + 1 (top face: no jump, 0)
    cf = _rows_n(cy, 0.0)
    pshi = _rows_n(psi, psi[-1])
    return visc - conv + D.gravity * (D.denp / rho - 1.0) + (D.surf * cf) * ((pshi - psi) * ih) / rho


def energy_rhs(th, u, v, densc, tc, D):
    te, tw = _e(th), _w(th)
    tn = _rows_n(th, th[-1])
    ts = _rows_s(th, 2.0 - th[0])
    uc = 0.5 * (u + _e(u))
    vc = 0.5 * (v[:-1] + v[1:])
    adv = uc * ((te - tw) * D.inv2h) + vc * ((tn - ts) * D.inv2h)
    ke = 0.5 * (tc + _e(tc))
    kw = 0.5 * (_w(tc) + tc)
    kn = 0.5 * (tc + _rows_n(tc, tc[-1]))
    ks = 0.5 * (_rows_s(tc, tc[0]) + tc)
    dif = ((ke * (te - th) - kw * (th - tw)) + (kn * (tn - th) - ks * (th - ts))) * D.ihsq
    return (D.pei * dif) / densc - adv


def refined_velocity(u, v):
    """u, v bilinearly interpolated to the refined cell centres (2 ny, 2 nx)."""
    ny, nx = u.shape
    ug = np.empty((ny + 2, nx))  # rows -1 .. ny
    ug[1:-1] = u
    ug[0] = -u[0]
    ug[-1] = u[-1]
    J = np.arange(2 * ny)
    jp, b = J // 2, J % 2
    # u: rows r0 = jp - 1 + b, r1 = r0 + 1 (ghost-shifted by +1), weight on r1: 0.75 (b=0) / 0.25
    r0 = jp - 1 + b + 1
    wy_u = np.where(b == 0, 0.75, 0.25)[:, None]
    I = np.arange(2 * nx)
    m, a = I // 2, I % 2
    c0 = m
    c1 = (m + 1) % nx
    wx_u = np.where(a == 0, 0.25, 0.75)[None, :]
    a00 = ug[r0][:, c0]
    a10 = ug[r0][:, c1]
    a01 = ug[r0 + 1][:, c0]
    a11 = ug[r0 + 1][:, c1]
    uf = (1.0 - wy_u) * ((1.0 - wx_u) * a00 + wx_u * a10) + wy_u * ((1.0 - wx_u) * a01 + wx_u * a11)
    # v: columns c0 = m - 1 + a, c1 = c0 + 1 (periodic), weight on c1: 0.75 (a=0) / 0.25;
    # rows r0 = jp, r1 = jp + 1, weight on r1: 0.25 (b=0) / 0.75
    vc0 = (m - 1 + a) % nx
    vc1 = (m + a) % nx
    wx_v = np.where(a == 0, 0.75, 0.25)[None, :]
    wy_v = np.where(b == 0, 0.25, 0.75)[:, None]
    b00 = v[jp][:, vc0]
    b10 = v[jp][:, vc1]
    b01 = v[jp + 1][:, vc0]
    b11 = v[jp + 1][:, vc1]
    vf = (1.0 - wy_v) * ((1.0 - wx_v) * b00 + wx_v * b10) + wy_v * ((1.0 - wx_v) * b01 + wx_v * b11)
    return uf, vf


def hjweno(a, b, cc, dd):
    eps = 1e-6
    s1 = 13.0 * (a - b) * (a - b) + 3.0 * (a - 3.0 * b) * (a - 3.0 * b)
    s2 = 13.0 * (b - cc) * (b - cc) + 3.0 * (b + cc) * (b + cc)
    s3 = 13.0 * (cc - dd) * (cc - dd) + 3.0 * (3.0 * cc - dd) * (3.0 * cc - dd)
    a1 = 1.0 / ((eps + s1) * (eps + s1))
    a2 = 6.0 / ((eps + s2) * (eps + s2))
    a3 = 3.0 / ((eps + s3) * (eps + s3))
    w1 = a1 / (a1 + a2 + a3)
    w3 = a3 / (a1 + a2 + a3)
    return (1.0 / 3.0) * w1 * (a - 2.0 * b + cc) + (1.0 / 6.0) * (w3 - 0.5) * (b - 2.0 * cc + dd)


def _weno(dp, take):
    """One-sided WENO5 derivatives from the face differences dp, take(k) = dp shifted so that
    element i holds dp[i + k]."""
    v1, v2, v3, v4, v5 = take(-3), take(-2), take(-1), take(0), take(1)
    dm = (1.0 / 12.0) * (-v2 + 7.0 * v3 + 7.0 * v4 - v5) - hjweno(v2 - v1, v3 - v2, v4 - v3, v5 - v4)
    q1, q2, q3, q4, q5 = take(2), take(1), take(0), take(-1), take(-2)
    dpl = (1.0 / 12.0) * (-q5 + 7.0 * q4 + 7.0 * q3 - q2) + hjweno(q1 - q2, q2 - q3, q3 - q4, q4 - q5)
    return dm, dpl


def face_diffs(phi, D):
    """dpx[J, I] = (phi[J, I+1] - phi[J, I]) / hf (periodic); dpy[J, I] = (phi[J+1, I] -
    phi[J, I]) / hf for J = 0..NJ-2, extended by constant slope (dpy[J] = dpy[0] below,
    dpy[NJ-2] above)."""
    dpx = (np.roll(phi, -1, axis=1) - phi) * D.ihf
    dpy = (phi[1:] - phi[:-1]) * D.ihf
    return dpx, dpy


def _take_x(dpx):
    return lambda k: np.roll(dpx, -k, axis=1)


def _take_y(dpy, nj):
    # element J holds dpy[clamp(J + k, 0, nj - 2)]
    idx = np.arange(nj)

    def take(k):
        return dpy[np.clip(idx + k, 0, nj - 2)]
    return take


def weno_xy(phi, D):
    nj = phi.shape[0]
    dpx, dpy = face_diffs(phi, D)
    dmx, dplx = _weno(dpx, _take_x(dpx))
    dmy, dply = _weno(dpy, _take_y(dpy, nj))
    return dmx, dplx, dmy, dply, dpx, dpy


def ls_rhs(phi, uf, vf, D):
    dmx, dplx, dmy, dply, _, _ = weno_xy(phi, D)
    px = np.where(uf >= 0.0, dmx, dplx)
    py = np.where(vf >= 0.0, dmy, dply)
    return -(uf * px + vf * py)


def godunov(sg, ap, am):
    aplus, aminus = sg * ap, sg * am
    return np.where((aplus >= 0.0) & (aminus >= 0.0), am,
                    np.where((aplus <= 0.0) & (aminus <= 0.0), ap,
                             np.where((aplus > 0.0) & (aminus < 0.0), 0.0,
                                      np.where(aplus + aminus > 0.0, am, ap))))


def reinit_stage(phi, a0, D):
    """One stage on the band |a0| < D.band; cells outside keep phi."""
    nj = phi.shape[0]
    dmx, dplx, dmy, dply, dpx, dpy = weno_xy(phi, D)
    tky = _take_y(dpy, nj)
    dx = 0.5 * (np.roll(dpx, 1, axis=1) + dpx)
    dz = 0.5 * (tky(-1) + tky(0))
    dal = dx * dx + dz * dz
    sg = a0 / np.sqrt(a0 * a0 + dal * (D.hf * D.hf))
    ax = godunov(sg, dplx, dmx)
    az = godunov(sg, dply, dmy)
    drhs = sg * (1.0 - np.sqrt(ax * ax + az * az))
    return np.where(np.abs(a0) < D.band, phi + (0.5 * D.hf) * drhs, phi)


def reinitialize(phi, D):
    a0 = phi.copy()
    band = np.abs(a0) < D.band
    for _ in range(D.nreinit):
        rk = phi
        phi = reinit_stage(phi, a0, D)
        phi = reinit_stage(phi, a0, D)
        phi = np.where(band, 0.75 * rk + 0.25 * phi, phi)
        phi = reinit_stage(phi, a0, D)
        phi = np.where(band, (1.0 / 3.0) * rk + (2.0 / 3.0) * phi, phi)
    return phi


def step(state, dt, props, mg_solve, mg_levels=6):
    """One RK3 step (three substeps, then the reinitialisation).  mg_solve(f, bx, by, h, p0)
    returns (p, iterations, rel, status).  Returns (new state, info)."""
    ny, nx = state["p"].shape
    D = Derived(nx, ny, props)
    u, v, p, th, phi = (np.array(state[k], dtype=np.float64, copy=True) for k in ("u", "v", "p", "th", "phi"))
    ru = np.zeros_like(u)
    rv = np.zeros((ny, nx))
    rth = np.zeros_like(th)
    rphi = np.zeros_like(phi)
    info = dict(iterations=[], rel=[], status=[], mdot_total=[])
    for k in (1, 2, 3):
        gam, ro = GAMMA[k], RO[k]
        alpha = gam + ro
        adt = alpha * dt
        iadt = 1.0 / (alpha * dt)
        psi, den, vis, densc, tc, bx, by = properties(phi, D)
        S, md = mass_source(th, psi, tc, D)
        cx, cy = curvature(phi, psi, D)
        nu = momentum_u(u, v, den, vis, D, psi, cx)
        nv = momentum_v(u, v, den, vis, D, psi, cy)
        # predictor with the current pressure gradient (p = 0 on the top face)
        us = u + dt * (gam * nu + ro * ru) - adt * (bx * ((p - _w(p)) * D.ih))
        vs = np.zeros_like(v)
        vs[1:ny] = v[1:ny] + dt * (gam * nv[:-1] + ro * rv[:-1]) - adt * (by[1:ny] * ((p[1:] - p[:-1]) * D.ih))
        vs[ny] = v[ny] + dt * (gam * nv[-1] + ro * rv[-1]) - adt * (by[ny] * ((0.0 - p[ny - 1]) * D.ih2))
        ru, rv = nu, nv
        f = ((_e(us) - us) * D.ih + (vs[1:] - vs[:-1]) * D.ih - S) * iadt
        # the pressure increment, from zero
        dp, it, rel, st = mg_solve(f, bx, by, D.h, np.zeros_like(p))
        info["iterations"].append(it)
        info["rel"].append(rel)
        info["status"].append(st)
        info["mdot_total"].append(float(md.sum()) * D.h * D.h)
        info["S"], info["mdot"] = S, md
        u = us - adt * (bx * ((dp - _w(dp)) * D.ih))
        v = vs.copy()
        v[1:ny] = vs[1:ny] - adt * (by[1:ny] * ((dp[1:] - dp[:-1]) * D.ih))
        v[ny] = vs[ny] - adt * (by[ny] * ((0.0 - dp[ny - 1]) * D.ih2))
        p = p + dp
        e = energy_rhs(th, u, v, densc, tc, D)
        thn = th + dt * (gam * e + ro * rth)
        rth = e
        th = np.where(psi > 0.5, 0.0, thn)
        uf, vf = refined_velocity(u, v)
        band = np.abs(phi) < D.band
        L = np.where(band, ls_rhs(phi, uf, vf, D), 0.0)
        phi = np.where(band, phi + dt * (gam * L + ro * rphi), phi)
        rphi = L
    phi = reinitialize(phi, D)
    return dict(u=u, v=v, p=p, th=th, phi=phi), info


def oracle_mg(levels, rtol=1e-10, ncoarse=2):
    """The oracle's 2-D multigrid (oracle/mg2d.cpp) as step()'s pressure solver, with the GPU
    multigrid's cycle: symmetric smoothing and piecewise-constant prolongation (flags 5)."""
    from . import oracle as orc

    def solve(f, bx, by, h, p0):
        p, cyc, rel, _, st = orc.mg_solve(f, bx, by, h, h, nlevels=levels, ncoarse=ncoarse, p0=p0, rtol=rtol,
                                          max_cycles=200, sym=5)
        return p, cyc, rel, st
    return solve


def step_native(state, dt, props, levels, native=False):
    """The same step through the C++/OpenMP restatement (film2d.cpp, bit-identical to step());
    returns (new state, info with iterations, rel, status, S, mdot)."""
    import ctypes as C
    from . import oracle as orc
    L = orc.lib(native)
    D = C.POINTER(C.c_double)
    I = C.POINTER(C.c_int)
    f = L.orc_film2d_step
    f.argtypes = [C.c_int, C.c_int, D, C.c_double, C.c_int, C.c_int, C.c_double] + [D] * 5 + [I, D, I, D, D]
    ny, nx = state["p"].shape
    out = {k: np.array(state[k], dtype=np.float64, copy=True, order="C") for k in ("u", "v", "p", "th", "phi")}
    P = np.array([props[k] for k in ("re", "visr", "denr", "prm", "scr", "tcr", "jakob", "fr")] +
                 [props.get("we", 0.0)], dtype=np.float64)
    its = (C.c_int * 3)()
    rels = (C.c_double * 3)()
    sts = (C.c_int * 3)()
    S = np.zeros((ny, nx))
    md = np.zeros((ny, nx))
    ptr = lambda a: a.ctypes.data_as(D)  # noqa: E731
    f(nx, ny, ptr(P), props["rtol"], int(props["nreinit"]), levels, dt, ptr(out["u"]), ptr(out["v"]), ptr(out["p"]),
      ptr(out["th"]), ptr(out["phi"]), its, rels, sts, ptr(S), ptr(md))
    return out, dict(iterations=list(its), rel=list(rels), status=list(sts), S=S, mdot=md)


def divergence(u, v, h):
    return (_e(u) - u) / h + (v[1:] - v[:-1]) / h
