"""Host-side mirror of the reference's pressure-Poisson interface.

* ``poisson``, ``trdiag3``, ``trdiag3p``: the reference subroutines POISSON
  (1d.f:3492-3578), TRDIAG3 (1d.f:3783-3811) and TRDIAG3P (1d.f:3929-3983) with the
  same arrays in the same Fortran layout (numpy, order='F'), run on the GPU through
  the C ABI.  Like the Fortran originals they update their output arrays in place.
* ``MultigridPoisson``: the 2-D variable-coefficient pressure Poisson solved by
  multigrid-preconditioned CG on the GPU (the reference has no multigrid; its
  operator is generalised from 1d.f:3535-3541).  Accepts device tensors (torch, on
  CUDA) or host numpy arrays.
"""
import ctypes as C

import numpy as np

from . import native

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


def _fptr(a):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1), "float64 Fortran-ordered array"
    return a.ctypes.data_as(_D)


def trdiag3(A, B, Cc, R, UU, l1, l2, ll1, ll2):
    """TRDIAG3(A,B,C,R,UU,L1,L2,LL1,LL2) on (ld, n) float64 Fortran arrays, in place.
    R and UU may be the same array (as LHSW passes GK twice, 1d.f:1790)."""
    ld = A.shape[0]
    for x in (A, B, Cc, R, UU):
        assert x.shape[0] == ld and x.flags.f_contiguous and x.dtype == np.float64
    native.check(native.lib().lica_gpu_trdiag3(_fptr(A), _fptr(B), _fptr(Cc), _fptr(R), _fptr(UU), l1, l2, ll1,
                                               ll2, ld), "TRDIAG3")


def trdiag3p(A, B, Cc, F, j1, j2, l1, l2):
    """TRDIAG3P(A,B,C,F,J1,J2,L1,L2): periodic systems, solution overwrites F."""
    ld = A.shape[0]
    for x in (A, B, Cc, F):
        assert x.shape[0] == ld and x.flags.f_contiguous and x.dtype == np.float64
    native.check(native.lib().lica_gpu_trdiag3p(_fptr(A), _fptr(B), _fptr(Cc), _fptr(F), j1, j2, l1, l2, ld),
                 "TRDIAG3P")


def poisson(geom, P, DIVGSUM, DENF_ZI):
    """POISSON(P,DIVGSUM,DENF_XI,DENF_YI,DENF_ZI,...) for the 1-D column.

    geom holds the GEOM module arrays as the Fortran code allocates them:
    m1, m2, m3, n1m, n2m, n3m, VVDZ(1:m3) as ``vvdz``, SSDZ(0:m3) as ``ssdz``,
    FIXKL(1:m3-1) as ``fixkl``, KPV(0:m3+1) as ``kpv`` (int64).  P is updated in place."""
    g = geom
    native.check(native.lib().lica_gpu_poisson(
        g["m1"], g["m2"], g["m3"], g["n1m"], g["n2m"], g["n3m"], _fptr(g["vvdz"]), _fptr(g["ssdz"]),
        _fptr(g["fixkl"]), g["kpv"].ctypes.data_as(_I64), _fptr(P), _fptr(DIVGSUM), _fptr(DENF_ZI)), "POISSON")


def uniform_column_geometry(n3m, zl=1.0, m1=2, m2=2):
    """GEOM arrays of a uniform 1-D column (GEOMETRIC 1d.f:4808-4866, INDICES
    1d.f:4975-5029) with IPZ != 1: VDZ(1) = VDZ(N3) = SDZ/2, FIXKL(1) = 1."""
    m3 = n3m + 1
    sdz = zl / n3m
    vvdz = np.empty(m3)
    vvdz[:] = 1.0 / sdz
    vvdz[0] = 1.0 / (0.5 * sdz)
    vvdz[m3 - 1] = 1.0 / (0.5 * sdz)
    ssdz = np.zeros(m3 + 1)
    ssdz[1:n3m + 1] = 1.0 / sdz
    fixkl = np.zeros(m3 - 1)
    fixkl[0] = 1.0
    kpv = np.arange(1, m3 + 3, dtype=np.int64)
    return dict(m1=m1, m2=m2, m3=m3, n1m=m1 - 1, n2m=m2 - 1, n3m=n3m, vvdz=vvdz, ssdz=ssdz, fixkl=fixkl, kpv=kpv)


def column_geometry(z, m1=2, m2=2):
    """GEOM arrays of a 1-D column on the faces z[0..n3m] (Z(1)..Z(N3), any spacing), for
    lica_gpu_poisson: VVDZ and SSDZ from GEOMETRIC (1d.f:4808-4882, lica_grid_metrics),
    FIXKL(1) = 1 and KPV(K) = K + 1 for IPZ != 1 (INDICES 1d.f:4975-5029)."""
    from .grid import metrics
    z = np.asarray(z, dtype=np.float64)
    n3m = len(z) - 1
    m3 = n3m + 1
    g = metrics(z)
    vvdz = np.ascontiguousarray(g["vvdz"][1:m3 + 1])
    ssdz = np.zeros(m3 + 1)
    ssdz[1:n3m + 1] = g["ssdz"][1:n3m + 1]
    fixkl = np.zeros(m3 - 1)
    fixkl[0] = 1.0
    kpv = np.arange(1, m3 + 3, dtype=np.int64)
    return dict(m1=m1, m2=m2, m3=m3, n1m=m1 - 1, n2m=m2 - 1, n3m=n3m, vvdz=vvdz, ssdz=ssdz, fixkl=fixkl, kpv=kpv)


def stretched_system(yface, bx, by, f):
    """(bx', by', f') of a pressure system on the stretched wall-normal faces yface[0..ny]
    (lica_mg_stretched_system): solve them with MultigridPoisson(nx, ny, hx, 1.0)."""
    ny, nx = f.shape
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (yface, bx, by, f)]
    assert arrs[0].shape == (ny + 1,) and arrs[1].shape == (ny, nx) and arrs[2].shape == (ny + 1, nx)
    out = [np.empty_like(arrs[1]), np.empty_like(arrs[2]), np.empty_like(arrs[3])]
    native.check(native.lib().lica_mg_stretched_system(nx, ny, *(a.ctypes.data_as(_D) for a in arrs + out)),
                 "lica_mg_stretched_system")
    return tuple(out)


PRECISION = {"fp64": 0, "mixed": 1}
SMOOTHER = {"rb": 0, "yline": 1}   # red-black points; y-line zebra (stretched wall grids, FP64)


class MultigridPoisson:
    """PCG with a symmetric V(nu1,nu2) multigrid preconditioner (C ABI lica_mg_*), red-black
    point smoothing or (smoother="yline") y-line zebra relaxation.

    Arrays: p, f of shape (ny, nx); bx (ny, nx) = beta on the face left of each cell
    (x periodic); by (ny+1, nx) = beta on the face below each row, row ny the top wall
    (p = 0 on that face), row 0 unused (Neumann bottom)."""

    def __init__(self, nx, ny, hx, hy, *, nlevels=6, nu1=2, nu2=2, ncoarse=2, precision="fp64", use_graph=True,
                 smoother="rb"):
        self.nx, self.ny, self.hx, self.hy = nx, ny, hx, hy
        self.options = native.MgOptions(nlevels, nu1, nu2, ncoarse, PRECISION[precision], int(use_graph),
                                        SMOOTHER[smoother])
        h = C.c_void_p()
        native.check(native.lib().lica_mg_create(C.byref(h), nx, ny, hx, hy, C.byref(self.options)),
                     "lica_mg_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            native.lib().lica_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_shapes(self, p, f, bx, by):
        assert tuple(p.shape) == (self.ny, self.nx) and tuple(f.shape) == (self.ny, self.nx)
        assert tuple(bx.shape) == (self.ny, self.nx) and tuple(by.shape) == (self.ny + 1, self.nx)

    def solve(self, p, f, bx, by, rtol=1e-10, max_iters=200, stream=None):
        """Solve A p = f in place on p.  Torch CUDA tensors run device-resident on the
        given (default: current) stream; numpy arrays go through the host entry point.
        Returns (iterations, rel_residual, status)."""
        self._check_shapes(p, f, bx, by)
        res = native.MgResult()
        if isinstance(p, np.ndarray):
            for a in (p, f, bx, by):
                assert a.dtype == np.float64 and a.flags.c_contiguous
            sp = None
            if stream is not None:
                sp = stream.cuda_stream
            code = native.lib().lica_mg_solve_host(self._h, p.ctypes.data_as(_D), f.ctypes.data_as(_D),
                                                   bx.ctypes.data_as(_D), by.ctypes.data_as(_D), rtol, max_iters,
                                                   C.byref(res), sp)
        else:
            import torch
            for a in (p, f, bx, by):
                assert a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()
            s = stream if stream is not None else torch.cuda.current_stream()
            code = native.lib().lica_mg_solve_device(self._h, p.data_ptr(), f.data_ptr(), bx.data_ptr(),
                                                     by.data_ptr(), rtol, max_iters, C.byref(res), s.cuda_stream)
        native.check(code, "lica_mg_solve", ok=(0, 1, 8))
        return res.iterations, res.rel_residual, res.status

    def solve_batch(self, ps, fs, bxs, bys, rtol=1e-10, max_iters=200):
        """Independent solves A p_k = f_k from host arrays (lica_mg_solve_host_batch): the
        upload of the next system and the download of the previous one overlap each solve
        (pinned arrays give the overlap).  Solves in place on each p_k; returns a list of
        (iterations, rel_residual, status)."""
        cnt = len(ps)
        if not (len(fs) == len(bxs) == len(bys) == cnt):
            raise ValueError("ps, fs, bxs, bys must have the same length")
        for k in range(cnt):
            self._check_shapes(ps[k], fs[k], bxs[k], bys[k])
            for a in (ps[k], fs[k], bxs[k], bys[k]):
                assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous

        def ptrs(arrs):
            return (C.c_void_p * cnt)(*[a.ctypes.data for a in arrs])
        res = (native.MgResult * cnt)()
        code = native.lib().lica_mg_solve_host_batch(self._h, cnt, ptrs(ps), ptrs(fs), ptrs(bxs), ptrs(bys), rtol,
                                                     max_iters, res)
        native.check(code, "lica_mg_solve_host_batch", ok=(0, 1, 8))
        return [(r.iterations, r.rel_residual, r.status) for r in res]

    KERNEL_CLASSES = ("down0", "down", "up0", "up", "cta", "pupdate", "xupdate", "setup")

    def profile(self, enable=True):
        """Time each kernel class with CUDA events (solves run as separate launches)."""
        native.check(native.lib().lica_mg_profile(self._h, int(enable)), "lica_mg_profile")

    def profile_read(self):
        out = {}
        for k, name in enumerate(self.KERNEL_CLASSES):
            ms, n = C.c_double(), C.c_int64()
            native.check(native.lib().lica_mg_profile_read(self._h, k, C.byref(ms), C.byref(n)), "profile_read")
            out[name] = (ms.value, n.value)
        return out

    def precond(self, z, r, bx, by, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        native.check(native.lib().lica_mg_precond_device(self._h, z.data_ptr(), r.data_ptr(), bx.data_ptr(),
                                                         by.data_ptr(), s.cuda_stream), "lica_mg_precond")

    def apply(self, out, u, bx, by, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        native.check(native.lib().lica_mg_apply_device(self._h, out.data_ptr(), u.data_ptr(), bx.data_ptr(),
                                                       by.data_ptr(), s.cuda_stream), "lica_mg_apply")
