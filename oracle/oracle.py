"""ctypes bindings to the oracle (test infrastructure only).

The oracle is the CPU restatement that the CUDA path is checked against.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this module; the
product package never does.
"""
import ctypes as C

import numpy as np

from . import build as _build

_LIBS = {}

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_INT = C.POINTER(C.c_int)


def lib(native: bool = False):
    key = bool(native)
    if key not in _LIBS:
        L = C.CDLL(_build.build(native=native))
        L.orc_mg_solve.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double] + [C.c_int] * 7 + \
            [_D, _D, _D, _D, C.c_double, C.c_int, _INT, _D, _D]
        L.orc_mg_precond.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double] + [C.c_int] * 6 + [_D] * 4
        L.orc_mg_apply.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _D, _D, _D]
        L.orc_mg_smooth.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _D, _D, _D, C.c_int,
                                    C.c_int]
        L.orc_trdiag3.argtypes = [_D, _D, _D, _D, _D] + [C.c_int64] * 5
        L.orc_trdiag3p.argtypes = [_D, _D, _D, _D] + [C.c_int64] * 5
        L.orc_poisson1d.argtypes = [C.c_int64] * 6 + [_D, _D, _D, _I64, _D, _D, _D]
        L.orc_lvs_init.argtypes = [C.c_int, C.c_double, C.c_double, _D, _INT, _D, _D, _D]
        L.orc_lvs_transport.argtypes = [C.c_int, C.c_double, _D, _INT, _D, _D, _D, _D, C.c_int, C.c_double,
                                        C.c_double, C.c_int, C.c_int, _D, C.c_double, C.c_int, _D, _D, _D]
        L.orc_lvs_transport_geo.argtypes = L.orc_lvs_transport.argtypes + [C.c_void_p]
        L.orc_lvs_alphi_bc.argtypes = [C.c_int, C.c_double, _D]
        L.orc_lvs_band.argtypes = [C.c_int, C.c_double, _D, _INT]
        L.orc_lvs_reinit.argtypes = [C.c_int, C.c_double, _D, _INT, C.c_int]
        L.orc_col_init.argtypes = [C.c_int, C.c_double, C.c_double, _D, _INT] + [_D] * 6 + [_INT] + [_D] * 5 + \
            [_INT, _D]
        L.orc_col_resume.argtypes = [C.c_int, C.c_double, _D, _INT, _D, _D, _D]
        L.orc_col_step.argtypes = [C.c_int, C.c_double, _D, _INT] + [_D] * 6 + [_INT] + [_D] * 5 + [_INT, _D, _D]
        L.orc_col_init_geo.argtypes = L.orc_col_init.argtypes + [C.c_void_p]
        L.orc_col_step_geo.argtypes = L.orc_col_step.argtypes + [C.c_void_p]
        L.orc_col_last_place.restype = C.c_double
        L.orc_col_last_place.argtypes = []
        L.orc_reinitialization.argtypes = [C.c_int, C.c_double, _D, _INT, C.c_int]
        L.orc_grid_coupling.argtypes = [C.c_int, C.c_double, C.c_int, _D, _INT, _D, _D]
        L.orc_col_temp_grad.argtypes = [C.c_int, C.c_double, _D, _INT, C.c_double, _D, _D, _D, _INT, _D, _D, _D,
                                        _INT, _D]
        L.orc_col_pressure_correction.argtypes = [C.c_int, C.c_double, _D, _INT, C.c_double, _D, _D, _D, _D]
        L.orc_jacobi3.argtypes = [_D, _D, C.c_double]
        L.orc_bubble_tracking.argtypes = [C.c_int] * 6 + [C.c_double] + [_D] * 6 + [C.c_int, C.c_int] + [_D] * 4 + \
            [C.c_double, C.c_int, C.c_void_p]
        _LIBS[key] = L
    return _LIBS[key]


def _p(a):
    return a.ctypes.data_as(_D if a.dtype == np.float64 else _I64)


METHODS = {"vcycle": 0, "defect": 1, "pcg": 2}


def mg_solve(f, bx, by, hx, hy, *, nlevels=6, nu1=2, nu2=2, ncoarse=2, sym=5, method="pcg", rtol=1e-10,
             max_cycles=100, mixed=False, p0=None, native=False):
    """Multigrid solve of A p = f (see oracle/mg2d.cpp).  sym: the cycle flags (1 symmetric
    smoothing, 2 R = P^T/4 of bilinear P, 4 piecewise-constant P, 8 y-line relaxation); the
    default 5 is the GPU multigrid's cycle.  Returns (p, cycles, rel, hist, status)."""
    ny, nx = f.shape
    f = np.ascontiguousarray(f, dtype=np.float64)
    bx = np.ascontiguousarray(bx, dtype=np.float64)
    by = np.ascontiguousarray(by, dtype=np.float64)
    assert bx.shape == (ny, nx) and by.shape == (ny + 1, nx)
    p = np.zeros((ny, nx)) if p0 is None else np.array(p0, dtype=np.float64, copy=True, order="C")
    cyc = C.c_int(0)
    rel = C.c_double(0.0)
    hist = np.full(max_cycles + 1, np.nan)
    st = lib(native).orc_mg_solve(nx, ny, hx, hy, nlevels, nu1, nu2, ncoarse, int(sym), METHODS[method],
                                  int(mixed), _p(f), _p(bx), _p(by), _p(p), rtol, max_cycles, C.byref(cyc),
                                  C.byref(rel), _p(hist))
    return p, cyc.value, rel.value, hist[: cyc.value + 1], st


def mg_apply(u, bx, by, hx, hy):
    ny, nx = u.shape
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty_like(u)
    lib().orc_mg_apply(nx, ny, hx, hy, _p(np.ascontiguousarray(bx)), _p(np.ascontiguousarray(by)), _p(u),
                       _p(out))
    return out


def mg_smooth(u, f, bx, by, hx, hy, nsweeps, reverse=False):
    ny, nx = u.shape
    u = np.array(u, dtype=np.float64, copy=True, order="C")
    lib().orc_mg_smooth(nx, ny, hx, hy, _p(np.ascontiguousarray(bx)), _p(np.ascontiguousarray(by)),
                        _p(np.ascontiguousarray(f)), _p(u), nsweeps, int(reverse))
    return u


def mg_precond(r, bx, by, hx, hy, *, nlevels=6, nu1=2, nu2=2, ncoarse=2, sym=5, mixed=False):
    """z = M r, one V-cycle preconditioner application (sym: the cycle flags of mg_solve)."""
    ny, nx = r.shape
    z = np.empty((ny, nx))
    st = lib().orc_mg_precond(nx, ny, hx, hy, nlevels, nu1, nu2, ncoarse, int(sym), int(mixed),
                              _p(np.ascontiguousarray(bx)), _p(np.ascontiguousarray(by)),
                              _p(np.ascontiguousarray(r, dtype=np.float64)), _p(z))
    assert st == 0, st
    return z


def trdiag3(A, B, C_, R, l1, l2, ll1, ll2):
    """TRDIAG3 on Fortran-ordered (ld, n) arrays; returns (R_out, UU)."""
    A, B, C_ = (np.asfortranarray(x, dtype=np.float64) for x in (A, B, C_))
    R = np.array(R, dtype=np.float64, order="F", copy=True)
    UU = np.zeros_like(R, order="F")
    st = lib().orc_trdiag3(_p(A), _p(B), _p(C_), _p(R), _p(UU), l1, l2, ll1, ll2, A.shape[0])
    assert st == 0
    return R, UU


def trdiag3p(A, B, C_, F, j1, j2, l1, l2):
    A, B, C_ = (np.asfortranarray(x, dtype=np.float64) for x in (A, B, C_))
    F = np.array(F, dtype=np.float64, order="F", copy=True)
    st = lib().orc_trdiag3p(_p(A), _p(B), _p(C_), _p(F), j1, j2, l1, l2, A.shape[0])
    assert st == 0
    return F


def poisson1d(geom, p, divgsum, denf_zi):
    """POISSON (1d.f:3492) on Fortran-layout arrays; geom is a dict of GEOM arrays."""
    m1, m2, m3 = geom["m1"], geom["m2"], geom["m3"]
    p = np.array(p, dtype=np.float64, order="F", copy=True)
    st = lib().orc_poisson1d(m1, m2, m3, geom["n1m"], geom["n2m"], geom["n3m"], _p(geom["vvdz"]),
                             _p(geom["ssdz"]), _p(geom["fixkl"]), _p(geom["kpv"]), _p(p),
                             _p(np.asfortranarray(divgsum)), _p(np.asfortranarray(denf_zi)))
    assert st == 0
    return p


# ---------------------------------------------------------------------------------------
# Level set of one 1-D column (oracle/lvs1d.cpp).  State dict:
#   phi (nf+7,) f64 at [k+2], layer (nf+7,) int32, psif (nf+2,), wo (n+2,), vol_tot_ori float
# ---------------------------------------------------------------------------------------

def _pi(a):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_INT)


def lvs_init(n, length, z0):
    """LVSINIT for a planar interface at z0 (vapour below).  Returns the state dict."""
    nf = 2 * n
    st = {"n": n, "length": float(length), "phi": np.zeros(nf + 7), "layer": np.zeros(nf + 7, np.int32),
          "psif": np.zeros(nf + 2), "wo": np.zeros(n + 2)}
    vol = C.c_double(0.0)
    rc = lib().orc_lvs_init(n, length, z0, _p(st["phi"]), _pi(st["layer"]), _p(st["psif"]), _p(st["wo"]),
                            C.byref(vol))
    assert rc == 0
    st["vol_tot_ori"] = vol.value
    return st


def lvs_copy(st):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}


def lvs_transport(st, w, mflvs, *, iphs, denr, dtconst, first, m_step, vol_tot_iphs, mglobal, psi_cn, psi_zn,
                  geo=None):
    """TRANSPORT + GRID_COUPLING(0) on a copy of st (geo: a stretched flow grid as col_geo
    takes it).  Returns (state, psi_cn, psi_zn, stats)."""
    st = lvs_copy(st)
    n = st["n"]
    w = np.ascontiguousarray(w, dtype=np.float64)
    mf = np.ascontiguousarray(mflvs, dtype=np.float64)
    assert w.shape == (n + 2,) and mf.shape == (2 * n + 7,)
    pc = np.array(psi_cn, dtype=np.float64, copy=True)
    pz = np.array(psi_zn, dtype=np.float64, copy=True)
    stats = np.zeros(4)
    vol = C.c_double(st["vol_tot_ori"])
    args = (n, st["length"], _p(st["phi"]), _pi(st["layer"]), _p(st["psif"]), _p(st["wo"]), _p(w), _p(mf),
            int(iphs), float(denr), float(dtconst), int(first), int(m_step), C.byref(vol), float(vol_tot_iphs),
            int(mglobal), _p(pc), _p(pz), _p(stats))
    if geo is None:
        rc = lib().orc_lvs_transport(*args)
    else:
        g = col_geo(geo)
        rc = lib().orc_lvs_transport_geo(*args, C.byref(g))
    if rc == 2:
        raise OverflowError("band left the stored range k = -2..nf+4")
    assert rc == 0
    st["vol_tot_ori"] = vol.value
    return st, pc, pz, stats


def lvs_alphi_bc(n, length, phi):
    phi = np.array(phi, dtype=np.float64, copy=True)
    lib().orc_lvs_alphi_bc(n, length, _p(phi))
    return phi


def lvs_band(n, length, phi, layer):
    phi = np.array(phi, dtype=np.float64, copy=True)
    layer = np.array(layer, dtype=np.int32, copy=True)
    lib().orc_lvs_band(n, length, _p(phi), _pi(layer))
    return phi, layer


def lvs_reinit(n, length, phi, layer, ilimit):
    phi = np.array(phi, dtype=np.float64, copy=True)
    lib().orc_lvs_reinit(n, length, _p(phi), _pi(np.ascontiguousarray(layer, dtype=np.int32)), ilimit)
    return phi


# ---------------------------------------------------------------------------------------
# 1-D column time step (oracle/column1d.cpp).  State dict of one column with the arrays of
# lica_col_state: w p t psi_cn psi_zn wo (n+2), phi mflvs (nf+7), layer (nf+7 int32),
# psif sfgas sfgas2 (nf+2), imask (n+2 int32), scal (5), stats (8).
# ---------------------------------------------------------------------------------------
COL_PROPS = ("re", "visr", "denr", "weber", "fr", "prm", "scr", "tcr", "t_sat", "jakob", "cflmax", "dt0")
COL_ORDER = ("w", "p", "t", "psi_cn", "psi_zn", "phi", "layer", "psif", "wo", "mflvs", "sfgas", "sfgas2", "imask",
             "scal")


def _col_props(props):
    return (np.array([float(getattr(props, k)) for k in COL_PROPS]),
            np.array([int(props.iphs), int(props.mglobal)], np.int32))


def _col_args(st):
    return [_pi(st[k]) if st[k].dtype == np.int32 else _p(st[k]) for k in COL_ORDER]


def col_empty(n):
    nf = 2 * n
    sf, sp, sq = n + 2, nf + 7, nf + 2
    st = {k: np.zeros(sf) for k in ("w", "p", "t", "psi_cn", "psi_zn", "wo")}
    st.update({"phi": np.zeros(sp), "mflvs": np.zeros(sp), "layer": np.zeros(sp, np.int32), "psif": np.zeros(sq),
               "sfgas": np.zeros(sq), "sfgas2": np.zeros(sq), "imask": np.zeros(sf, np.int32), "scal": np.zeros(5),
               "stats": np.zeros(8)})
    return st


def col_init(n, length, z0, props):
    st = col_empty(n)
    pr, ip = _col_props(props)
    rc = lib().orc_col_init(n, length, z0, _p(pr), _pi(ip), *_col_args(st))
    if rc:
        raise ValueError(f"orc_col_init returned {rc}")
    return st


def col_step(st, n, length, props, native=False):
    """One time step in place.  Returns the status (0 ok, 1 TEMP_EXTP not converged,
    2 band overflow)."""
    pr, ip = _col_props(props)
    return lib(native).orc_col_step(n, length, _p(pr), _pi(ip), *_col_args(st), _p(st["stats"]))


def col_history_record(st, time_before, native=False):
    """The reference's per-step interface record for the step col_step just took on this
    thread: (TIME before the step, place of 0interface.dat (chphase.f:1419-1438), the vapour
    volume VOL_TOT_IPHS (chphase.f:1457), DT)."""
    return (time_before, lib(native).orc_col_last_place(), float(st["scal"][4]), float(st["scal"][0]))


# ---------------------------------------------------------------------------------------
# Single routines of the column step (the per-subroutine drop-ins' checkers)
# ---------------------------------------------------------------------------------------
def reinitialization(n, length, phi, layer, ilimit):
    """REINITIALIZATION (two_phase.f:2033-2474) of one column: phi (nf+7) in place."""
    lib().orc_reinitialization(n, length, _p(phi), _pi(layer), int(ilimit))
    return phi


def grid_coupling(n, length, ini, psif, layer, psi_cn, psi_zn):
    """GRID_COUPLING(INI_PSI) (two_phase.f:4863-5118) of one column: psi_cn, psi_zn in place."""
    lib().orc_grid_coupling(n, length, int(ini), _p(psif), _pi(layer), _p(psi_cn), _p(psi_zn))
    return psi_cn, psi_zn


def col_temp_grad(n, length, props, dtconst, t, psi_cn, phi, layer, vol):
    """TEMP_GRAD (chphase.f:55-368) of one column: returns (iterations, mflvs, sfgas, sfgas2,
    imask, VOL_TOT_IPHS); iterations -1 when TEMP_EXTP did not converge."""
    pr, ip = _col_props(props)
    nf = 2 * n
    mflvs, sfgas, sfgas2 = np.zeros(nf + 7), np.zeros(nf + 2), np.zeros(nf + 2)
    imask = np.zeros(n + 2, np.int32)
    v = np.array([float(vol)])
    it = lib().orc_col_temp_grad(n, length, _p(pr), _pi(ip), float(dtconst), _p(np.ascontiguousarray(t)),
                                 _p(np.ascontiguousarray(psi_cn)), _p(np.ascontiguousarray(phi)),
                                 _pi(np.ascontiguousarray(layer)), _p(mflvs), _p(sfgas), _p(sfgas2), _pi(imask), _p(v))
    return it, mflvs, sfgas, sfgas2, imask, float(v[0])


def col_pressure_correction(n, length, props, dtconst, w, p, denf_zi, sfgas):
    """PRESSURE_CORRECTION (1d.f:3403-3488) of one column: w, p in place."""
    pr, ip = _col_props(props)
    lib().orc_col_pressure_correction(n, length, _p(pr), _pi(ip), float(dtconst), _p(w), _p(p),
                                      _p(np.ascontiguousarray(denf_zi)), _p(np.ascontiguousarray(sfgas)))
    return w, p


# ---------------------------------------------------------------------------------------
# Stretched columns: the geometry (GEOMETRIC arrays, GEOM_COUPLING z tables) of ColGeo
# ---------------------------------------------------------------------------------------
class _ColGeo(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("z", "zp", "sdz", "vdz", "ssdz", "vvdz", "kcou1", "kcou2", "kcoump1",
                                           "kcoump2", "kcou_vel", "kcoump_vel")]


def col_geo(geo):
    """A ColGeo over the arrays of geo (a dict of z, zp, sdz, vdz, ssdz, vvdz (float64, n+2)
    and kcou1, kcou2, kcoump1, kcoump2, kcou_vel, kcoump_vel (int32)); keeps them alive."""
    arrs = {k: np.ascontiguousarray(geo[k], dtype=np.int32 if k.startswith("kcou") else np.float64)
            for k in _ColGeo._fields_ and [f[0] for f in _ColGeo._fields_]}
    g = _ColGeo(*[arrs[f[0]].ctypes.data for f in _ColGeo._fields_])
    g._keep = arrs
    return g


def col_init_geo(n, length, z0, props, geo):
    st = col_empty(n)
    pr, ip = _col_props(props)
    g = col_geo(geo)
    rc = lib().orc_col_init_geo(n, length, z0, _p(pr), _pi(ip), *_col_args(st), C.byref(g))
    if rc:
        raise ValueError(f"orc_col_init_geo returned {rc}")
    return st


def col_step_geo(st, n, length, props, geo, native=False):
    """One time step of a stretched column in place (geo as col_geo takes it)."""
    pr, ip = _col_props(props)
    g = col_geo(geo)
    return lib(native).orc_col_step_geo(n, length, _p(pr), _pi(ip), *_col_args(st), _p(st["stats"]), C.byref(g))


# one record of BUBBLE_TRACKING per level set (the layout of lica_bub_record)
BUB_RECORD = np.dtype([("time", "f8"), ("llvs", "i8"), ("col", "f8", 9), ("vel", "f8", 3), ("vol", "f8"),
                       ("ami", "f8", 3), ("iz_periodic", "i8")])


def jacobi3(a, abserr=1e-12):
    """Jacobi_bub on a symmetric 3x3 matrix: (a after the rotations, eigenvectors as columns)."""
    a = np.array(a, dtype=np.float64, order="C", copy=True)
    x = np.empty((3, 3))
    lib().orc_jacobi3(_p(a), _p(x), abserr)
    return a, x


def bubble_tracking(grid, psi_tmp, u, v, w, *, time=0.0, icacy=1, llvs0=1):
    """BUBBLE_TRACKING + BUBBLE_EIGENV for each field of psi_tmp (nlvs, n3m+2, n2m+2, n1m+2);
    grid: dict with n1m, n2m, n3m, ipx, ipy, ipz, zl and sdx, sdy, sdz, xp, yp, zp (Fortran
    index as offset).  Returns the records (BUB_RECORD)."""
    psi = np.ascontiguousarray(psi_tmp, dtype=np.float64)
    nlvs = psi.shape[0]
    shape = (grid["n3m"] + 2, grid["n2m"] + 2, grid["n1m"] + 2)
    assert psi.shape[1:] == shape
    u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
    assert u.shape == v.shape == w.shape == shape
    geo = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in ("sdx", "sdy", "sdz", "xp", "yp", "zp")]
    out = np.zeros(nlvs, dtype=BUB_RECORD)
    lib().orc_bubble_tracking(grid["n1m"], grid["n2m"], grid["n3m"], grid["ipx"], grid["ipy"], grid["ipz"],
                              grid["zl"], *[_p(a) for a in geo], nlvs, llvs0, _p(psi), _p(u), _p(v), _p(w),
                              time, icacy, out.ctypes.data_as(C.c_void_p))
    return out
