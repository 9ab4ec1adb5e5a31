"""Non-uniform grids: the reference's grid generator and its metrics, through the library's
host code (lica_grid_*).

``read_grid_in`` parses the generator's input file (grid.in: the flow grid's sections
for directions 1-3, the level-set grid's for 4-6), ``generate`` builds the coordinates of
every direction section by section (UNIFORM, GEOPRO, HYPTAN; grid.f:118-128),
``write_grid_dat`` writes them as grid.f writes grid.dat (grid.f:229-243), and
``metrics`` is GEOMETRIC (1d.f:4808-4882) for one direction.  ``poisson.column_geometry``
turns a column's faces into the arrays of the POISSON drop-in, and
``poisson.stretched_system`` writes a 2-D pressure system on a stretched wall-normal grid
for the multigrid.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native

_D = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(_D)


@dataclass
class Section:
    idir: int      # 1-3: flow x, y, z; 4-6: level-set x, y, z
    xyzi: float
    xyzf: float
    ngi: int
    ngf: int
    iopt: int      # 1 uniform, 2 geometric progression, 3 hyperbolic tangent
    fac1: float    # ER or GAM
    fac2: float    # YESEXP or XSI


def _tokens(line):
    return line.replace(",", " ").split()


def read_grid_in(path):
    """The generator's input (grid.f:31-52, list-directed reads: a DUMMY line is skipped
    whole; blank lines are skipped).  Returns dict(ispare=[4 ints], flow=dict(n=(N1,N2,N3),
    length=(XL,YL,ZL), sections=[Section]), levelset=dict(...))."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    it = iter(lines)

    def record():
        for ln in it:
            if ln.strip():
                return ln
        raise ValueError(f"{path}: unexpected end of file")

    def block():
        record()                                       # ##...GRID## label
        record()                                       # NSECT N1 N2 N3 XL YL ZL labels
        tok = _tokens(record())
        nsect, n1, n2, n3 = (int(t) for t in tok[:4])
        xl, yl, zl = (float(t.replace("d", "e").replace("D", "E")) for t in tok[4:7])
        record()                                       # column labels
        secs = []
        for _ in range(nsect):
            t = _tokens(record())
            secs.append(Section(int(t[0]), float(t[1]), float(t[2]), int(t[3]), int(t[4]), int(t[5]), float(t[6]),
                                float(t[7])))
        return dict(n=(n1, n2, n3), length=(xl, yl, zl), sections=secs)

    record()                                           # ISPARE labels
    ispare = [int(t) for t in _tokens(record())[:4]]
    flow = block()
    ls = block()
    return dict(ispare=ispare, flow=flow, levelset=ls)


def section(s, out):
    """Fill out[N - 1], N = s.ngi..s.ngf, with the section's coordinates."""
    native.check(native.lib().lica_grid_section(s.iopt, s.xyzi, s.xyzf, s.ngi, s.ngf, s.fac1, s.fac2, _p(out)),
                 "lica_grid_section")


def generate(spec):
    """Coordinates of the six directions of a read_grid_in spec: dict idir -> array of the
    direction's points (index N - 1).  Spare cells for an immersed pipe (ISPARE /= 0) are
    not supported."""
    if any(spec["ispare"]):
        raise NotImplementedError("ISPARE spare cells (the immersed-boundary pipe) are not supported")
    sizes = dict(zip((1, 2, 3), spec["flow"]["n"]))
    sizes.update(zip((4, 5, 6), spec["levelset"]["n"]))
    out = {d: np.full(sizes[d], np.nan) for d in sizes}
    for s in spec["flow"]["sections"] + spec["levelset"]["sections"]:
        if s.ngf > sizes[s.idir]:
            raise ValueError(f"section of direction {s.idir} ends at {s.ngf} > {sizes[s.idir]}")
        section(s, out[s.idir])
    for d, a in out.items():
        if np.isnan(a).any():
            raise ValueError(f"direction {d}: points not covered by any section")
    return out


def _es(x, w, d):
    m, e = ("%.*E" % (d, x)).split("E")
    e = int(e)
    s = m + ("E%+03d" % e if abs(e) <= 99 else "%+04d" % e)
    return s.rjust(w) if len(s) <= w else "*" * w


def _put(values, per, fmt):
    out = []
    for i in range(0, len(values), per):
        out.append("".join(fmt(v) for v in values[i:i + per]) + "\n")
    return "".join(out) if out else "\n"


def write_grid_dat(path, spec, coords):
    """grid.dat as grid.f writes it (FORMATs 111 3I23, 112 3F23.15, 113 5ES23.15)."""
    i23 = lambda v: ("%d" % v).rjust(23)       # noqa: E731
    f23 = lambda v: ("%.15f" % v).rjust(23)    # noqa: E731
    es23 = lambda v: _es(float(v), 23, 15)     # noqa: E731
    o = []
    for blk, dirs in (("flow", (1, 2, 3)), ("levelset", (4, 5, 6))):
        o.append(_put(list(spec[blk]["n"]), 3, i23))
        o.append(_put(list(spec[blk]["length"]), 3, f23))
        for d in dirs:
            o.append(_put(list(coords[d]), 5, es23))
    with open(path, "w") as f:
        f.write("".join(o))


def metrics(z):
    """GEOMETRIC for faces z (z[0] = Z(1) ... z[n-1] = Z(n)): dict of SDZ, VDZ, SSDZ, VVDZ,
    ZP as arrays indexed by the Fortran index 0..n."""
    z = np.asarray(z, dtype=np.float64)
    n = len(z)
    zf = np.concatenate([[0.0], z])                       # zf[k] = Z(k)
    outs = {k: np.zeros(n + 1) for k in ("sdz", "vdz", "ssdz", "vvdz", "zp")}
    native.check(native.lib().lica_grid_metrics(n, _p(zf), *(_p(outs[k]) for k in ("sdz", "vdz", "ssdz", "vvdz",
                                                                                    "zp"))),
                 "lica_grid_metrics")
    return outs


def coupling_z(z, zf):
    """GEOM_COUPLING's z tables (lica_grid_coupling_z) for flow faces z (Z(1)..Z(N3)) and
    uniform refined faces zf (ZF(1)..ZF(N3F)): dict of int32 arrays kcou1, kcou2 (index K+1,
    K = -1..N3+2), kcoump1, kcoump2 (K+1, K = -1..N3+1), kcou_vel, kcoump_vel (K = 1..N3F)."""
    z = np.concatenate([[0.0], np.asarray(z, dtype=np.float64)])
    zf = np.concatenate([[0.0], np.asarray(zf, dtype=np.float64)])
    n3, n3f = len(z) - 1, len(zf) - 1
    out = dict(kcou1=np.zeros(n3 + 4, np.int32), kcou2=np.zeros(n3 + 4, np.int32),
               kcoump1=np.zeros(n3 + 3, np.int32), kcoump2=np.zeros(n3 + 3, np.int32),
               kcou_vel=np.zeros(n3f + 1, np.int32), kcoump_vel=np.zeros(n3f + 1, np.int32))
    I32 = C.POINTER(C.c_int32)
    native.check(native.lib().lica_grid_coupling_z(n3, _p(z), n3f, _p(zf), *(out[k].ctypes.data_as(I32) for k in (
        "kcou1", "kcou2", "kcoump1", "kcoump2", "kcou_vel", "kcoump_vel"))), "lica_grid_coupling_z")
    return out


def column_geometry(faces, length):
    """The wall-normal geometry of a 1-D column of n = len(faces) - 1 flow cells on the
    given faces Z(1..n+1) (a stretched grid), against the uniform level-set grid of 2n cells
    over the same length: GEOMETRIC's arrays z, zp, sdz, vdz, ssdz, vvdz (float64, n+2,
    Fortran index; z[k] = Z(k)) and GEOM_COUPLING's z tables kcou1, kcou2, kcoump1, kcoump2,
    kcou_vel, kcoump_vel (int32) -- the layout of lica_col_geometry.  Host code only."""
    faces = np.asarray(faces, dtype=np.float64)
    n = len(faces) - 1
    nf = 2 * n
    zf = np.arange(nf + 1, dtype=np.float64) * (float(length) / nf)   # ZF(k) = (k - 1) hf
    geo = metrics(faces)
    geo["z"] = np.concatenate([[0.0], faces])
    geo.update(coupling_z(faces, zf))
    return geo
