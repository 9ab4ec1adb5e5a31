"""Bubble statistics of several level sets on a 3-D grid, on the GPU.

``track`` is BUBBLE_TRACKING(LLVS, PSI_TMP, U, V, W) (two_phase.f:6321-6555) with
BUBBLE_EIGENV (6558-6705) and Jacobi_bub (two_phase.f:19-97) for every level set of a batch
in one launch (``lica_gpu_bubble_tracking[_device]`` in include/lica_gpu.h).  Each record
holds what the reference appends to 0bub_tracking.dat -- TIME, LLVS and nine columns (the
centroid, the velocity, the aspect ratio and two angles; cylindrical with icacy = 2) -- and
VELVS(LLVS, 1:3), plus the gas volume, the eigenvalues and IZ_PERIODIC.

Fields are (n3m+2, n2m+2, n1m+2) arrays in C order, i.e. the Fortran (0:N1, 0:N2, 0:N3)
arrays as they lie in memory; ``psi_tmp`` stacks nlvs of them.  numpy arrays take the host
path (copies in and out); torch CUDA tensors the device path.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native

RECORD = np.dtype([("time", "f8"), ("llvs", "i8"), ("col", "f8", 9), ("vel", "f8", 3), ("vol", "f8"),
                   ("ami", "f8", 3), ("iz_periodic", "i8")])

GRID_ARRAYS = ("sdx", "sdy", "sdz", "xp", "yp", "zp")


@dataclass
class BubbleGrid:
    """The flow grid BUBBLE_TRACKING reads: cells per direction, periodic flags, the z
    period ZL and the cell widths and centres SDX, XP (0:N1), SDY, YP (0:N2), SDZ, ZP (0:N3)."""
    n1m: int
    n2m: int
    n3m: int
    sdx: np.ndarray
    sdy: np.ndarray
    sdz: np.ndarray
    xp: np.ndarray
    yp: np.ndarray
    zp: np.ndarray
    ipx: int = 1
    ipy: int = 1
    ipz: int = 0
    zl: float = 0.0

    @staticmethod
    def uniform(n1m, n2m, n3m, xl, yl, zl, *, ipx=1, ipy=1, ipz=0):
        """Uniform cells over [0, xl] x [0, yl] x [0, zl] (the ghost entries repeat the first
        cell's width, the ghost centres continue the spacing)."""
        arrays = {}
        for name, n, length in (("x", n1m, xl), ("y", n2m, yl), ("z", n3m, zl)):
            h = length / n
            arrays["sd" + name] = np.full(n + 2, h)
            arrays[name + "p"] = (np.arange(n + 2) - 0.5) * h
        return BubbleGrid(n1m, n2m, n3m, ipx=ipx, ipy=ipy, ipz=ipz, zl=float(zl), **arrays)

    @property
    def field_shape(self):
        return (self.n3m + 2, self.n2m + 2, self.n1m + 2)

    def as_dict(self):
        d = {k: getattr(self, k) for k in ("n1m", "n2m", "n3m", "ipx", "ipy", "ipz", "zl")}
        d.update({k: np.ascontiguousarray(getattr(self, k), dtype=np.float64) for k in GRID_ARRAYS})
        return d

    def _c(self):
        arrs = [np.ascontiguousarray(getattr(self, k), dtype=np.float64) for k in GRID_ARRAYS]
        for k, a, n in zip(GRID_ARRAYS, arrs, (self.n1m, self.n2m, self.n3m) * 2):
            if a.shape != (n + 2,):
                raise ValueError(f"{k}: shape {a.shape}, expected ({n + 2},)")
        g = native.BubGrid(self.n1m, self.n2m, self.n3m, int(self.ipx), int(self.ipy), int(self.ipz), float(self.zl),
                           *[a.ctypes.data for a in arrs])
        return g, arrs


class BubbleTracker:
    """A device copy of the grid with room for max_lvs level sets per call."""

    def __init__(self, grid: BubbleGrid, max_lvs: int):
        self.grid = grid
        self.max_lvs = int(max_lvs)
        g, keep = grid._c()
        h = C.c_void_p()
        native.check(native.lib().lica_gpu_bubble_grid_create(C.byref(h), C.byref(g), self.max_lvs),
                     "lica_gpu_bubble_grid_create")
        del keep
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            native.lib().lica_gpu_bubble_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def track(self, psi_tmp, u, v, w, *, time=0.0, icacy=1, llvs0=1, out=None, stream=None):
        """Device path: psi_tmp (nlvs, *field_shape), u, v, w torch CUDA float64 tensors.
        Enqueues on the stream (default: torch's current one) and returns the records as a
        uint8 CUDA tensor of nlvs * RECORD.itemsize bytes (``records(...)`` reads them)."""
        import torch
        nlvs = psi_tmp.shape[0]
        fs = self.grid.field_shape
        if tuple(psi_tmp.shape[1:]) != fs or any(tuple(a.shape) != fs for a in (u, v, w)):
            raise ValueError(f"fields must be {fs}")
        for a in (psi_tmp, u, v, w):
            if not (a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()):
                raise ValueError("fields must be contiguous float64 CUDA tensors")
        if out is None:
            out = torch.empty(nlvs * RECORD.itemsize, dtype=torch.uint8, device=psi_tmp.device)
        st = stream if stream is not None else torch.cuda.current_stream(psi_tmp.device)
        native.check(native.lib().lica_gpu_bubble_tracking_device(
            self._h, nlvs, int(llvs0), C.c_void_p(psi_tmp.data_ptr()), C.c_void_p(u.data_ptr()),
            C.c_void_p(v.data_ptr()), C.c_void_p(w.data_ptr()), float(time), int(icacy),
            C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream)), "lica_gpu_bubble_tracking_device")
        return out


def records(raw):
    """The records of a ``BubbleTracker.track`` result (after the stream has finished)."""
    return np.frombuffer(raw.cpu().numpy().tobytes(), dtype=RECORD)


def track(grid: BubbleGrid, psi_tmp, u, v, w, *, time=0.0, icacy=1, llvs0=1):
    """Host path: numpy fields in, records (RECORD) out."""
    fs = grid.field_shape
    psi = np.ascontiguousarray(psi_tmp, dtype=np.float64)
    if psi.ndim != 4 or psi.shape[1:] != fs:
        raise ValueError(f"psi_tmp must be (nlvs, {fs[0]}, {fs[1]}, {fs[2]})")
    u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
    if any(a.shape != fs for a in (u, v, w)):
        raise ValueError(f"u, v, w must be {fs}")
    g, keep = grid._c()
    out = np.zeros(psi.shape[0], dtype=RECORD)
    p = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in (psi, u, v, w)]
    native.check(native.lib().lica_gpu_bubble_tracking(C.byref(g), psi.shape[0], int(llvs0), *p, float(time),
                                                        int(icacy), out.ctypes.data_as(C.c_void_p)),
                 "lica_gpu_bubble_tracking")
    del keep
    return out


def format_records(recs):
    """The lines BUBBLE_TRACKING appends to 0bub_tracking.dat (FORMAT 1ES15.7, 1I5, 9ES15.7)."""
    lines = []
    for r in recs:
        lines.append("%15.7E%5d" % (r["time"], r["llvs"]) + "".join("%15.7E" % c for c in r["col"]))
    return lines


def append_records(path, recs):
    """Append the records to a 0bub_tracking.dat file as BUBBLE_TRACKING does (OPEN with
    POSITION='APPEND', one WRITE per level set; two_phase.f:6440-6443)."""
    with open(path, "a") as fh:
        for line in format_records(recs):
            fh.write(line + "\n")


def contact_times(recs, vol_tot_ori, surf_j):
    """CAL_TCON (two_phase.f:7304-7343) for every pair of the records' level sets: T_CON(L, LL)
    = SURF_J * |VELVS(L) - VELVS(LL)|^2 * DCHAR with DCHAR = 0.5 (6 VOLS / 3.14159)^(1/3) and
    VOLS = min(VOL_TOT_ORI(L), VOL_TOT_ORI(LL)) -- the reference's constants, in its order.
    vol_tot_ori: the original volume of each record's level set.  Returns an nlvs x nlvs
    array (zero on the diagonal)."""
    vel = np.asarray(recs["vel"], dtype=np.float64)
    vol = np.asarray(vol_tot_ori, dtype=np.float64)
    nl = vel.shape[0]
    if vol.shape != (nl,):
        raise ValueError(f"vol_tot_ori must hold {nl} volumes")
    out = np.zeros((nl, nl))
    for a in range(nl):
        for b in range(nl):
            if a == b:
                continue
            vols = min(vol[b], vol[a])
            dchar = 0.5 * ((6 * vols / 3.14159) ** (1.0 / 3.0))
            d = vel[a] - vel[b]
            urel = ((d[0] ** 2 + d[1] ** 2) + d[2] ** 2) ** 0.5
            out[a, b] = surf_j * (urel ** 2) * dchar
    return out
