"""Host-side mirror of the reference's single subroutines of the step, one call each, for
batches of 1-D columns (the C ABI's per-routine drop-ins, include/lica_gpu.h):

    reinitialization   REINITIALIZATION(NN1, NN2, ILIMIT, LLVS)   two_phase.f:2033-2474
    grid_coupling      GRID_COUPLING(INI_PSI, ...)                two_phase.f:4863-5118
    temp_grad          TEMP_GRAD(PSI_CN)                          chphase.f:55-368
    pressure_correction PRESSURE_CORRECTION(U, V, W, P, ...)      1d.f:3403-3488

Arrays are (ncol, m) in the column layout of ``column.Columns`` (flow n+2, phi-like nf+7 at
k+2, psif-like nf+2 at k): numpy arrays go through the host entry points (copied in and
out), torch CUDA tensors through the _device ones on the current stream.  Each routine runs
the fused step's own device code.
"""
import ctypes as C

import numpy as np

from . import native


def _is_np(a):
    return isinstance(a, np.ndarray)


def _np(a, dt, shape, name):
    if a.dtype != dt or not a.flags.c_contiguous or a.shape != shape:
        raise TypeError(f"{name}: need a C-contiguous {np.dtype(dt).name} array of shape {shape}")
    return a.ctypes.data_as(C.POINTER(C.c_int32 if dt == np.int32 else C.c_double))


def _dev(a, dt, shape, name):
    import torch
    want = torch.int32 if dt == np.int32 else torch.float64
    if not (a.is_cuda and a.dtype == want and a.is_contiguous() and tuple(a.shape) == shape):
        raise TypeError(f"{name}: need a contiguous CUDA {want} tensor of shape {shape}")
    return C.c_void_p(a.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def reinitialization(n, length, phi, layer, ilimit, status=None):
    """ILIMIT reinitialisation iterations of the band (layers 1..N_MAX-1) of every column;
    phi in place.  Returns the per-column status."""
    ncol, nf = phi.shape[0], 2 * n
    L = native.lib()
    if _is_np(phi):
        st = np.zeros(ncol, np.int32)
        rc = L.lica_gpu_reinitialization(ncol, n, length, _np(phi, np.float64, (ncol, nf + 7), "phi"),
                                         _np(layer, np.int32, (ncol, nf + 7), "layer"), int(ilimit),
                                         st.ctypes.data_as(C.POINTER(C.c_int32)))
        native.check(rc, "lica_gpu_reinitialization", ok=(0, 2, 4))
        return st
    import torch
    st = torch.zeros(ncol, dtype=torch.int32, device=phi.device) if status is None else status
    rc = L.lica_gpu_reinitialization_device(ncol, n, length, _dev(phi, np.float64, (ncol, nf + 7), "phi"),
                                            _dev(layer, np.int32, (ncol, nf + 7), "layer"), int(ilimit),
                                            C.c_void_p(st.data_ptr()), _stream())
    native.check(rc, "lica_gpu_reinitialization_device")
    return st


def grid_coupling(n, length, ini_psi, psif, layer, psi_cn, psi_zn):
    """PSI_CN / PSI_ZN of every column from PSIF (in place)."""
    ncol, nf = psif.shape[0], 2 * n
    L = native.lib()
    if _is_np(psif):
        lay = None if layer is None else _np(layer, np.int32, (ncol, nf + 7), "layer")
        rc = L.lica_gpu_grid_coupling(ncol, n, length, int(ini_psi), _np(psif, np.float64, (ncol, nf + 2), "psif"),
                                      lay, _np(psi_cn, np.float64, (ncol, n + 2), "psi_cn"),
                                      _np(psi_zn, np.float64, (ncol, n + 2), "psi_zn"))
    else:
        lay = C.c_void_p(None) if layer is None else _dev(layer, np.int32, (ncol, nf + 7), "layer")
        rc = L.lica_gpu_grid_coupling_device(ncol, n, length, int(ini_psi),
                                             _dev(psif, np.float64, (ncol, nf + 2), "psif"), lay,
                                             _dev(psi_cn, np.float64, (ncol, n + 2), "psi_cn"),
                                             _dev(psi_zn, np.float64, (ncol, n + 2), "psi_zn"), _stream())
    native.check(rc, "lica_gpu_grid_coupling")


def temp_grad(n, length, props, dtconst, t, psi_cn, phi, layer, vol_tot_iphs):
    """TEMP_GRAD of every column.  Returns dict(mflvs, sfgas, sfgas2, imask, vol_tot_iphs,
    iterations, status), numpy or CUDA tensors like the inputs; vol_tot_iphs (ncol,) is
    updated in place too."""
    ncol, nf = t.shape[0], 2 * n
    cp = props.c()
    L = native.lib()
    if _is_np(t):
        out = dict(mflvs=np.zeros((ncol, nf + 7)), sfgas=np.zeros((ncol, nf + 2)), sfgas2=np.zeros((ncol, nf + 2)),
                   imask=np.zeros((ncol, n + 2), np.int32), iterations=np.zeros(ncol, np.int32),
                   status=np.zeros(ncol, np.int32))
        rc = L.lica_gpu_temp_grad(ncol, n, length, C.byref(cp), float(dtconst),
                                  _np(t, np.float64, (ncol, n + 2), "t"),
                                  _np(psi_cn, np.float64, (ncol, n + 2), "psi_cn"),
                                  _np(phi, np.float64, (ncol, nf + 7), "phi"),
                                  _np(layer, np.int32, (ncol, nf + 7), "layer"),
                                  *(_np(out[k], out[k].dtype, out[k].shape, k) for k in ("mflvs", "sfgas", "sfgas2",
                                                                                          "imask")),
                                  _np(vol_tot_iphs, np.float64, (ncol,), "vol_tot_iphs"),
                                  _np(out["iterations"], np.int32, (ncol,), "iterations"),
                                  _np(out["status"], np.int32, (ncol,), "status"))
        native.check(rc, "lica_gpu_temp_grad", ok=(0, 1, 2))
    else:
        import torch
        dev = t.device
        out = dict(mflvs=torch.zeros((ncol, nf + 7), dtype=torch.float64, device=dev),
                   sfgas=torch.zeros((ncol, nf + 2), dtype=torch.float64, device=dev),
                   sfgas2=torch.zeros((ncol, nf + 2), dtype=torch.float64, device=dev),
                   imask=torch.zeros((ncol, n + 2), dtype=torch.int32, device=dev),
                   iterations=torch.zeros(ncol, dtype=torch.int32, device=dev),
                   status=torch.zeros(ncol, dtype=torch.int32, device=dev))
        ptr = lambda a: C.c_void_p(a.data_ptr())  # noqa: E731
        rc = L.lica_gpu_temp_grad_device(ncol, n, length, C.byref(cp), float(dtconst),
                                         _dev(t, np.float64, (ncol, n + 2), "t"),
                                         _dev(psi_cn, np.float64, (ncol, n + 2), "psi_cn"),
                                         _dev(phi, np.float64, (ncol, nf + 7), "phi"),
                                         _dev(layer, np.int32, (ncol, nf + 7), "layer"),
                                         ptr(out["mflvs"]), ptr(out["sfgas"]), ptr(out["sfgas2"]), ptr(out["imask"]),
                                         _dev(vol_tot_iphs, np.float64, (ncol,), "vol_tot_iphs"),
                                         ptr(out["iterations"]), ptr(out["status"]), C.c_void_p(None), _stream())
        native.check(rc, "lica_gpu_temp_grad_device")
    out["vol_tot_iphs"] = vol_tot_iphs
    return out


def pressure_correction(n, length, props, dtconst, w, p, denf_zi, sfgas):
    """DIVGS + POISSON + UCALC + the P(1) shift of every column; w, p in place."""
    ncol, nf = w.shape[0], 2 * n
    cp = props.c()
    L = native.lib()
    if _is_np(w):
        rc = L.lica_gpu_pressure_correction(ncol, n, length, C.byref(cp), float(dtconst),
                                            _np(w, np.float64, (ncol, n + 2), "w"),
                                            _np(p, np.float64, (ncol, n + 2), "p"),
                                            _np(denf_zi, np.float64, (ncol, n + 2), "denf_zi"),
                                            _np(sfgas, np.float64, (ncol, nf + 2), "sfgas"))
        native.check(rc, "lica_gpu_pressure_correction")
        return
    import torch
    st = torch.zeros(ncol, dtype=torch.int32, device=w.device)
    rc = L.lica_gpu_pressure_correction_device(ncol, n, length, C.byref(cp), float(dtconst),
                                               _dev(w, np.float64, (ncol, n + 2), "w"),
                                               _dev(p, np.float64, (ncol, n + 2), "p"),
                                               _dev(denf_zi, np.float64, (ncol, n + 2), "denf_zi"),
                                               _dev(sfgas, np.float64, (ncol, nf + 2), "sfgas"),
                                               C.c_void_p(st.data_ptr()), C.c_void_p(None), _stream())
    native.check(rc, "lica_gpu_pressure_correction_device")
