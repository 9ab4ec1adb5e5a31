"""Host-side mirror of the reference's level-set transport for 1-D columns.

``transport`` is TRANSPORT (two_phase.f:701-984) followed by GRID_COUPLING(0)
(two_phase.f:4863-5118), the pair MAIN calls once per RK3 substep (1d.f:242-244), run on
the GPU for a batch of independent columns through the C ABI
(``lica_gpu_lvs_transport[_device]`` in include/lica_gpu.h).  ``ColumnBatch`` holds the
per-column level-set state with the layout that entry point takes; its arrays are numpy
(host path: every call copies in and out, like the Fortran subroutine it replaces) or
torch CUDA tensors (device path: state stays in HBM).

The refined grid of a column has nf = 2 n cells; phi and layer hold k = -2..nf+4 at
index k+2, psif holds k = 1..nf at index k, the flow-face arrays k = 0..n+1 at index k.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)

FIELDS = ("phi", "layer", "psif", "wo", "vol_tot_ori", "psi_cn", "psi_zn")


def _shapes(ncol, n):
    nf = 2 * n
    return {"phi": (ncol, nf + 7), "layer": (ncol, nf + 7), "psif": (ncol, nf + 2), "wo": (ncol, n + 2),
            "vol_tot_ori": (ncol,), "psi_cn": (ncol, n + 2), "psi_zn": (ncol, n + 2), "w": (ncol, n + 2),
            "mflvs": (ncol, nf + 7), "vol_tot_iphs": (ncol,), "status": (ncol,), "stats": (ncol, 4)}


@dataclass
class ColumnBatch:
    """Level-set state of ncol columns of n flow cells over a column of the given length."""
    n: int
    length: float
    phi: object
    layer: object
    psif: object
    wo: object
    vol_tot_ori: object
    psi_cn: object
    psi_zn: object

    @property
    def ncol(self):
        return self.phi.shape[0]

    @staticmethod
    def from_arrays(n, length, **arrays):
        return ColumnBatch(n=n, length=float(length), **{k: arrays[k] for k in FIELDS})

    def to(self, device):
        """A copy on a torch device ('cuda'), or on the host as numpy with device=None."""
        import torch
        out = {}
        for k in FIELDS:
            v = getattr(self, k)
            if device is None:
                out[k] = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.array(v, copy=True)
            else:
                out[k] = torch.as_tensor(np.asarray(v) if not isinstance(v, torch.Tensor) else v, device=device).clone()
        return ColumnBatch(n=self.n, length=self.length, **out)


def _params(iphs, first, m_step, mglobal, denr, dtconst):
    return native.LvsParams(int(iphs), int(first), int(m_step), int(mglobal), float(denr), float(dtconst))


def _check(batch, arrays):
    sh = _shapes(batch.ncol, batch.n)
    for name, a in arrays.items():
        if tuple(a.shape) != sh[name]:
            raise ValueError(f"{name}: shape {tuple(a.shape)}, expected {sh[name]}")


def transport(batch, w, mflvs, vol_tot_iphs, *, iphs, denr, dtconst, first, m_step, mglobal=1, stream=None,
              geometry=None):
    """One TRANSPORT + GRID_COUPLING(0) of every column, updating ``batch`` in place.

    w: W on the flow faces (ncol, n+2); mflvs: interfacial mass flux per refined cell
    (ncol, nf+7), used when iphs = 1; vol_tot_iphs: (ncol,).  Returns (status, stats):
    per-column lica_status and [subcycles, max |grad phi|, min |grad phi|, IMASS].
    Host batches take numpy arrays; device batches take CUDA tensors (and a torch
    stream, default: the current one).  geometry: a column.ColumnGeometry of the batch's
    n and length for stretched flow grids (lica_gpu_lvs_transport_geometry[_device])."""
    if geometry is not None and (geometry.n != batch.n or abs(geometry.length - batch.length) > 1e-12 * batch.length):
        raise ValueError("the geometry's size or length differs from the batch's")
    prm = _params(iphs, first, m_step, mglobal, denr, dtconst)
    L = native.lib()
    st_arrays = {k: getattr(batch, k) for k in FIELDS}
    _check(batch, {**st_arrays, "w": w, "mflvs": mflvs, "vol_tot_iphs": vol_tot_iphs})
    if isinstance(batch.phi, np.ndarray):
        for k, a in st_arrays.items():
            want = np.int32 if k == "layer" else np.float64
            if a.dtype != want or not a.flags.c_contiguous:
                raise TypeError(f"{k}: need a C-contiguous {want.__name__} array")
        w = np.ascontiguousarray(w, dtype=np.float64)
        mflvs = np.ascontiguousarray(mflvs, dtype=np.float64)
        vi = np.ascontiguousarray(vol_tot_iphs, dtype=np.float64)
        status = np.zeros(batch.ncol, np.int32)
        stats = np.zeros((batch.ncol, 4))
        d = lambda a: a.ctypes.data_as(_D)  # noqa: E731
        args = (d(batch.phi), batch.layer.ctypes.data_as(_I32), d(batch.psif), d(batch.wo), d(w), d(mflvs),
                d(batch.vol_tot_ori), d(vi), d(batch.psi_cn), d(batch.psi_zn), status.ctypes.data_as(_I32),
                d(stats), C.byref(prm))
        if geometry is None:
            rc = L.lica_gpu_lvs_transport(batch.ncol, batch.n, batch.length, *args)
        else:
            rc = L.lica_gpu_lvs_transport_geometry(geometry.handle(), batch.ncol, *args)
        native.check(rc, "TRANSPORT", ok=(0, 2))
        return status, stats
    import torch
    for k, a in st_arrays.items():
        want = torch.int32 if k == "layer" else torch.float64
        if a.dtype != want or not a.is_cuda or not a.is_contiguous():
            raise TypeError(f"{k}: need a contiguous CUDA {want} tensor")
    for name, a in (("w", w), ("mflvs", mflvs), ("vol_tot_iphs", vol_tot_iphs)):
        if a.dtype != torch.float64 or not a.is_cuda or not a.is_contiguous():
            raise TypeError(f"{name}: need a contiguous CUDA float64 tensor")
    dev = batch.phi.device
    status = torch.zeros(batch.ncol, dtype=torch.int32, device=dev)
    stats = torch.zeros((batch.ncol, 4), dtype=torch.float64, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    args = (batch.phi.data_ptr(), batch.layer.data_ptr(), batch.psif.data_ptr(), batch.wo.data_ptr(), w.data_ptr(),
            mflvs.data_ptr(), batch.vol_tot_ori.data_ptr(), vol_tot_iphs.data_ptr(), batch.psi_cn.data_ptr(),
            batch.psi_zn.data_ptr(), status.data_ptr(), stats.data_ptr(), C.byref(prm), C.c_void_p(s.cuda_stream))
    if geometry is None:
        rc = L.lica_gpu_lvs_transport_device(batch.ncol, batch.n, batch.length, *args)
    else:
        rc = L.lica_gpu_lvs_transport_geometry_device(geometry.handle(), batch.ncol, *args)
    native.check(rc, "TRANSPORT")
    return status, stats
