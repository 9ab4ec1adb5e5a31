"""Host-side mirror of the reference's time loop for 1-D boiling columns.

``Columns`` holds the state of a batch of independent columns (the reference's MAIN
state for its 1-D case: W, P, T, PSI_CN, PSI_ZN, the level-set band, the phase-change
fields and DT/TIME/M) in the layout of ``lica_col_state`` (include/lica_gpu.h), as numpy
arrays (host) or torch CUDA tensors (device).  ``Columns.steps`` advances every column by
whole RK3 time steps of MAIN (1d.f:190-250) in one persistent GPU launch.

Column arrays, nf = 2 n refined cells:
  w, p, t, psi_cn, psi_zn, wo : (ncol, n+2), index k = 0..n+1
  phi, mflvs : (ncol, nf+7) at k+2, k = -2..nf+4;  layer : int32, same shape
  psif, sfgas, sfgas2 : (ncol, nf+2) at k;  imask : int32 (ncol, n+2)
  scal : (ncol, 5) DT, TIME, M, VOL_TOT_ORI, VOL_TOT_IPHS;  stats : (ncol, 8)
"""
import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import native

PHASES = ("dt", "continuity", "energy", "temp_grad", "temp_extp", "continuity2", "rhsz", "lhsw", "pressure",
          "convrge", "transport")

STATS = ("cfl", "divergence", "extension_iterations", "levelset_subcycles", "mass_corrections", "interface_height",
         "vapour_volume", "dt")


@dataclass
class ColumnProps:
    """lica.in properties of the two-phase / heat block (INPUT_SIMULATION, 1d.f:346-379).
    Defaults: the shipped case."""
    re: float = 1.42e-2
    visr: float = 22.22
    denr: float = 1605.36
    weber: float = 7.36e-8
    fr: float = 9.7
    prm: float = 1.0231
    scr: float = 2.077
    tcr: float = 27.16
    t_sat: float = 1.0
    jakob: float = 0.009
    cflmax: float = 0.5
    dt0: float = 2.5e-6
    iphs: int = 1
    mglobal: int = 1

    def c(self):
        return native.ColProps(*[getattr(self, f.name) for f in fields(self)])


def _shapes(ncol, n):
    nf = 2 * n
    sf, sp, sq = n + 2, nf + 7, nf + 2
    return {"w": (sf, np.float64), "p": (sf, np.float64), "t": (sf, np.float64), "psi_cn": (sf, np.float64),
            "psi_zn": (sf, np.float64), "phi": (sp, np.float64), "layer": (sp, np.int32), "psif": (sq, np.float64),
            "wo": (sf, np.float64), "mflvs": (sp, np.float64), "sfgas": (sq, np.float64),
            "sfgas2": (sq, np.float64), "imask": (sf, np.int32), "scal": (5, np.float64), "stats": (8, np.float64)}


class ColumnGeometry:
    """The flow grid of a stretched column: n cells on the faces Z(1..n+1) = faces (rising
    from 0 to the column length, no cell narrower than length / 2n) under the uniform
    level-set grid of 2n cells -- GEOMETRIC's arrays and GEOM_COUPLING's z tables
    (lica_col_geometry), and their checked device copy (lica_gpu_column_geometry_create),
    made on first use."""

    def __init__(self, faces):
        from .grid import column_geometry
        faces = np.ascontiguousarray(faces, dtype=np.float64)
        self.n, self.length = len(faces) - 1, float(faces[-1])
        self.faces = faces
        self.arrays = column_geometry(faces, self.length)
        self._h = None

    @staticmethod
    def tanh(n, length, gam):
        """HYPTAN clustering at both walls (grid.f:383-420, XSI = 0.5): n cells."""
        from .grid import Section, section
        faces = np.zeros(n + 1)
        section(Section(3, 0.0, float(length), 1, n + 1, 3, float(gam), 0.5), faces)
        return ColumnGeometry(faces)

    def c(self):
        """The lica_col_geometry of the host arrays (valid while self lives)."""
        return native.ColGeometry(*[self.arrays[k].ctypes.data for k in native.GEO_FIELDS])

    def handle(self):
        if self._h is None:
            h = C.c_void_p()
            g = self.c()
            native.check(native.lib().lica_gpu_column_geometry_create(C.byref(h), self.n, self.length, C.byref(g)),
                         "lica_gpu_column_geometry_create")
            self._h = _GeoHandle(h.value)
        return self._h.ptr


class Columns:
    """State of ncol columns of n flow cells over a column of the given length; geometry:
    a ColumnGeometry all the columns share (a stretched flow grid), or None (uniform)."""

    def __init__(self, n, length, arrays, geometry=None):
        self.n, self.length = int(n), float(length)
        self.arrays = arrays
        self.ncol = arrays["w"].shape[0]
        self.geometry = geometry
        if geometry is not None and (geometry.n != self.n or abs(geometry.length - self.length) > 1e-12 * self.length):
            raise ValueError("the geometry's size or length differs from the columns'")

    def __getattr__(self, k):
        a = self.__dict__.get("arrays")
        if a is not None and k in a:
            return a[k]
        raise AttributeError(k)

    @property
    def on_device(self):
        return not isinstance(self.arrays["w"], np.ndarray)

    @staticmethod
    def empty(ncol, n, length, geometry=None):
        return Columns(n, length, {k: np.zeros((ncol, m), dt) for k, (m, dt) in _shapes(ncol, n).items()}, geometry)

    @staticmethod
    def film(n, length, z0s, props, geometry=None):
        """Columns each holding a vapour film of thickness z0 at the wall (MAKEFLD +
        LVSINIT + GRID_COUPLING(1), lica_gpu_column_init; lica_gpu_column_init_geometry
        on a stretched grid)."""
        z0s = np.atleast_1d(np.asarray(z0s, dtype=np.float64))
        cols = Columns.empty(len(z0s), n, length, geometry)
        cp = props.c()
        g = geometry.c() if geometry is not None else None
        for c, z0 in enumerate(z0s):
            st = native.ColState(*[cols.arrays[k][c].ctypes.data for k in native.COL_FIELDS])
            if g is None:
                rc = native.lib().lica_gpu_column_init(n, length, float(z0), C.byref(cp), C.byref(st))
            else:
                rc = native.lib().lica_gpu_column_init_geometry(n, length, float(z0), C.byref(cp), C.byref(g),
                                                                C.byref(st))
            native.check(rc, "lica_gpu_column_init")
        return cols

    def to(self, device):
        """A copy on a torch device, or on the host (numpy) for device=None."""
        import torch
        out = {}
        for k, v in self.arrays.items():
            if device is None:
                out[k] = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v.copy()
            else:
                out[k] = torch.as_tensor(v if isinstance(v, np.ndarray) else v.cpu().numpy(), device=device).clone()
        return Columns(self.n, self.length, out, self.geometry)

    def _state(self, ptr):
        return native.ColState(*[ptr(self.arrays[k]) for k in native.COL_FIELDS])

    def steps(self, nsteps, props, stream=None, scratch=None, threads=0):
        """Advance every column by nsteps time steps.  Returns the per-column status
        (numpy for host state; a CUDA tensor for device state, filled when the stream
        reaches it)."""
        L = native.lib()
        cp = props.c()
        if not self.on_device:
            for k, (m, dt) in _shapes(self.ncol, self.n).items():
                a = self.arrays[k]
                if a.dtype != dt or not a.flags.c_contiguous or a.shape != (self.ncol, m):
                    raise TypeError(f"{k}: need a C-contiguous {np.dtype(dt).name} array of shape {(self.ncol, m)}")
            status = np.zeros(self.ncol, np.int32)
            st = self._state(lambda a: a.ctypes.data)
            sp = status.ctypes.data_as(C.POINTER(C.c_int32))
            if self.geometry is None:
                rc = L.lica_gpu_column_steps(self.ncol, self.n, self.length, C.byref(cp), C.byref(st), int(nsteps), sp)
            else:
                rc = L.lica_gpu_column_steps_geometry(self.geometry.handle(), self.ncol, C.byref(cp), C.byref(st),
                                                      int(nsteps), sp)
            native.check(rc, "column steps", ok=(0, 1, 2, 4))
            return status
        import torch
        dev = self.arrays["w"].device
        status = torch.zeros(self.ncol, dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        st = self._state(lambda a: a.data_ptr())
        scr = C.c_void_p(scratch.data_ptr() if scratch is not None else None)
        if self.geometry is None:
            rc = L.lica_gpu_column_steps_device(self.ncol, self.n, self.length, C.byref(cp), C.byref(st), int(nsteps),
                                                int(threads), scr, C.c_void_p(status.data_ptr()),
                                                C.c_void_p(s.cuda_stream))
        else:
            rc = L.lica_gpu_column_steps_geometry_device(self.geometry.handle(), self.ncol, C.byref(cp), C.byref(st),
                                                         int(nsteps), int(threads), scr,
                                                         C.c_void_p(status.data_ptr()), C.c_void_p(s.cuda_stream))
        native.check(rc, "column steps")
        return status


def scratch_bytes(ncol, n):
    return int(native.lib().lica_gpu_column_scratch_bytes(ncol, n))


def profile(prof):
    """Collect per-phase SM cycles into prof (an int64 CUDA tensor of len(PHASES) * ncol,
    zeroed by the caller) during later steps; None turns the profile off."""
    native.check(native.lib().lica_gpu_column_profile_device(C.c_void_p(prof.data_ptr() if prof is not None else None)),
                 "column profile")


HISTORY = ("time", "place", "vapour_volume", "dt")


def history(hist):
    """Record the reference's per-step interface history (0interface.dat's TIME and place,
    chphase.f:1419-1438; VOL_TOT_IPHS, chphase.f:1457; and DT) of later step launches into
    hist, a float64 CUDA tensor of shape (ncol, capacity, 4): step s of a launch goes to
    hist[c, s].  None turns it off."""
    if hist is None:
        rc = native.lib().lica_gpu_column_history_device(None, 0)
    else:
        if hist.dim() != 3 or hist.shape[2] != len(HISTORY) or not hist.is_contiguous():
            raise ValueError("hist: need a contiguous (ncol, capacity, 4) tensor")
        rc = native.lib().lica_gpu_column_history_device(C.c_void_p(hist.data_ptr()), int(hist.shape[1]))
    native.check(rc, "column history")


_FLOW = ("w", "p", "t", "psi_cn", "psi_zn", "wo", "imask")
_PHI = ("phi", "layer", "mflvs")
_PSIF = ("psif", "sfgas", "sfgas2")
_INT = ("layer", "imask")


class ColumnBatch:
    """Columns of uneven size, length and properties, packed back to back
    (lica_gpu_column_batch_*).  Flat arrays: the flow kind (w, p, t, psi_cn, psi_zn, wo,
    imask), the phi kind (phi, layer, mflvs), the psif kind (psif, sfgas, sfgas2); scal
    (ncol, 5) and stats (ncol, 8).  ``offsets[c]`` = the column's start in each kind."""

    def __init__(self, n, length, props, arrays=None, _handle=None):
        self.n = np.asarray(n, dtype=np.int32)
        self.length = np.asarray(length, dtype=np.float64)
        self.props = list(props)
        self.ncol = len(self.n)
        if _handle is None:
            h = C.c_void_p()
            cp = (native.ColProps * self.ncol)(*[p.c() for p in self.props])
            native.check(native.lib().lica_gpu_column_batch_create(
                C.byref(h), self.ncol, self.n.ctypes.data_as(C.POINTER(C.c_int32)),
                self.length.ctypes.data_as(C.POINTER(C.c_double)), cp), "column batch")
            _handle = _Handle(h)
        self._h = _handle
        off = np.zeros(3 * self.ncol, np.int64)
        tot = np.zeros(4, np.int64)
        native.check(native.lib().lica_gpu_column_batch_layout(self._h.ptr, off.ctypes.data_as(C.POINTER(C.c_int64)),
                                                               tot.ctypes.data_as(C.POINTER(C.c_int64))), "layout")
        self.offsets = off.reshape(self.ncol, 3)
        self.totals = tot
        if arrays is None:
            arrays = {}
            for k in _FLOW:
                arrays[k] = np.zeros(tot[0], np.int32 if k in _INT else np.float64)
            for k in _PHI:
                arrays[k] = np.zeros(tot[1], np.int32 if k in _INT else np.float64)
            for k in _PSIF:
                arrays[k] = np.zeros(tot[2], np.float64)
            arrays["scal"] = np.zeros((self.ncol, 5))
            arrays["stats"] = np.zeros((self.ncol, 8))
        self.arrays = arrays

    @staticmethod
    def films(n, length, z0, props):
        """Each column with a vapour film of thickness z0[c] at the wall (lica_gpu_column_init)."""
        b = ColumnBatch(n, length, props)
        for c in range(b.ncol):
            st = b._column_state(c, lambda a: a.ctypes.data)
            native.check(native.lib().lica_gpu_column_init(int(b.n[c]), float(b.length[c]), float(z0[c]),
                                                           C.byref(b.props[c].c()), C.byref(st)), "column init")
        return b

    def _column_state(self, c, ptr):
        of, op, oq = (int(x) for x in self.offsets[c])
        isz = {np.dtype(np.int32): 4, np.dtype(np.float64): 8}

        def at(k, o):
            a = self.arrays[k]
            return ptr(a) + o * (4 if k in _INT else 8)
        f = {k: at(k, of) for k in _FLOW}
        f.update({k: at(k, op) for k in _PHI})
        f.update({k: at(k, oq) for k in _PSIF})
        f["scal"] = ptr(self.arrays["scal"]) + 8 * 5 * c
        f["stats"] = ptr(self.arrays["stats"]) + 8 * 8 * c
        del isz
        return native.ColState(*[f[k] for k in native.COL_FIELDS])

    def column(self, c):
        """Host copy of column c's arrays in lica_col_state shapes."""
        host = self if isinstance(self.arrays["w"], np.ndarray) else self.to(None)
        n = int(self.n[c])
        of, op, oq = (int(x) for x in self.offsets[c])
        out = {k: host.arrays[k][of:of + n + 2].copy() for k in _FLOW}
        out.update({k: host.arrays[k][op:op + 2 * n + 7].copy() for k in _PHI})
        out.update({k: host.arrays[k][oq:oq + 2 * n + 2].copy() for k in _PSIF})
        out["scal"] = host.arrays["scal"][c].copy()
        out["stats"] = host.arrays["stats"][c].copy()
        return out

    def to(self, device):
        import torch
        out = {}
        for k, v in self.arrays.items():
            if device is None:
                out[k] = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v.copy()
            else:
                out[k] = torch.as_tensor(v if isinstance(v, np.ndarray) else v.cpu().numpy(), device=device).clone()
        return ColumnBatch(self.n, self.length, self.props, out, self._h)

    def steps(self, nsteps, threads=0, stream=None, scratch=None, tri_cap=-1):
        """nsteps time steps of every column (device state).  threads: the CTA width (64,
        128 or 256), or 0 for the autotuner's launch shape for this batch on this GPU (timed
        once on a copy of the state, then cached; see autotune.py); tri_cap: the longest
        column whose Thomas arrays live in shared memory (-1: as the CTAs per SM allow, 0:
        none).  Returns the per-column status."""
        import torch
        if threads == 0:
            from . import autotune
            threads, tri_cap = autotune.tune(self)[0]
        dev = self.arrays["w"].device
        status = torch.zeros(self.ncol, dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        st = native.ColState(*[self.arrays[k].data_ptr() for k in native.COL_FIELDS])
        native.check(native.lib().lica_gpu_column_batch_steps_ex_device(
            self._h.ptr, C.byref(st), int(nsteps), int(threads), int(tri_cap),
            C.c_void_p(scratch.data_ptr() if scratch is not None else None), C.c_void_p(status.data_ptr()),
            C.c_void_p(s.cuda_stream)), "column batch steps")
        return status


class _Handle:
    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            native.lib().lica_gpu_column_batch_destroy(self.ptr)
        except Exception:
            pass


class _GeoHandle:
    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            native.lib().lica_gpu_column_geometry_destroy(self.ptr)
        except Exception:
            pass


def uneven_batch(ncol, seed=0, nmin=128, nmax=2048, h=1.0 / 512):
    """Seeded batch of independent boiling columns: n uniform in [nmin, nmax] flow cells of
    size h, film 0.1 of the column, wall superheat uniform 2-20 K (Jakob number 0.009 per
    10 K), liquid/vapour density ratio uniform 100-1600; other properties of the shipped
    case.  Returns (n, length, z0, props)."""
    rng = np.random.default_rng(seed)
    n = rng.integers(nmin, nmax + 1, ncol).astype(np.int32)
    length = n * h
    z0 = 0.1 * length + 0.37 * h
    sup = rng.uniform(2.0, 20.0, ncol)
    denr = rng.uniform(100.0, 1600.0, ncol)
    props = [ColumnProps(denr=float(d), jakob=0.009 * float(t) / 10.0) for d, t in zip(denr, sup)]
    return n, length, z0, props
