"""ctypes binding of the C ABI in include/lica_gpu.h (liblica_gpu.so, built in-tree).

There is no CPU fallback: if the library is missing this module raises at import, and
every entry point runs CUDA kernels.
"""
import ctypes as C
import os

from . import build as _build

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class MgOptions(C.Structure):
    _fields_ = [("nlevels", C.c_int32), ("nu1", C.c_int32), ("nu2", C.c_int32), ("ncoarse", C.c_int32),
                ("precision", C.c_int32), ("use_graph", C.c_int32), ("smoother", C.c_int32)]


class MgResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("rel_residual", C.c_double)]


class LvsParams(C.Structure):
    _fields_ = [("iphs", C.c_int32), ("first", C.c_int32), ("m_step", C.c_int32), ("mglobal", C.c_int32),
                ("denr", C.c_double), ("dtconst", C.c_double)]


_I32 = C.POINTER(C.c_int32)


class ColProps(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("re", "visr", "denr", "weber", "fr", "prm", "scr", "tcr", "t_sat",
                                           "jakob", "cflmax", "dt0")] + [("iphs", C.c_int32), ("mglobal", C.c_int32)]


COL_FIELDS = ("w", "p", "t", "psi_cn", "psi_zn", "phi", "layer", "psif", "wo", "mflvs", "sfgas", "sfgas2", "imask",
              "scal", "stats")


class ColState(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in COL_FIELDS]


GEO_FIELDS = ("z", "zp", "sdz", "vdz", "ssdz", "vvdz", "kcou1", "kcou2", "kcoump1", "kcoump2", "kcou_vel",
              "kcoump_vel")


class ColGeometry(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in GEO_FIELDS]


class FldInfo(C.Structure):
    _fields_ = [("ihist", C.c_int64), ("m", C.c_int64), ("time", C.c_double), ("dt", C.c_double),
                ("qvol_ori", C.c_double), ("ips", C.c_int32), ("ipx", C.c_int32), ("ipy", C.c_int32),
                ("ipz", C.c_int32), ("pra", C.c_double)] + \
        [(k, C.c_double) for k in ("denr", "visr", "fr", "surf_j", "fk", "re_air", "prm", "scr", "tcr")] + \
        [("n_max", C.c_int32), ("contact", C.c_int32), ("contact_old", C.c_int32), ("lvson", C.c_int32),
         ("vol_tot_ori", C.c_double), ("contact_start", C.c_double), ("contact_time", C.c_double),
         ("t_con", C.c_double)]


class FldOptions(C.Structure):
    _fields_ = [("ireset", C.c_int32), ("idtold", C.c_int32), ("ipzero", C.c_int32)]


class Film2DProps(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("re", "visr", "denr", "prm", "scr", "tcr", "jakob", "fr", "we",
                                          "rtol")] + \
        [("max_iters", C.c_int32), ("nreinit", C.c_int32)]


class Film2DStats(C.Structure):
    _fields_ = [("iterations", C.c_int32 * 3), ("status", C.c_int32 * 3), ("rel_residual", C.c_double * 3),
                ("guess_rel", C.c_double * 3)]


class BubGrid(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("n1m", "n2m", "n3m", "ipx", "ipy", "ipz")] + [("zl", C.c_double)] + \
        [(k, C.c_void_p) for k in ("sdx", "sdy", "sdz", "xp", "yp", "zp")]


# every symbol include/lica_gpu.h declares, with its ctypes signature
SIGNATURES = {
    "lica_last_error": (C.c_char_p, []),
    "lica_kernel_launch_count": (C.c_int64, []),
    "lica_debug_poison_shared": (C.c_int, [C.c_double, C.c_void_p]),
    "lica_gpu_trdiag3": (C.c_int, [_D, _D, _D, _D, _D] + [C.c_int64] * 5),
    "lica_gpu_trdiag3p": (C.c_int, [_D, _D, _D, _D] + [C.c_int64] * 5),
    "lica_gpu_trdiag3_device": (C.c_int, [C.c_void_p] * 5 + [C.c_int64] * 5 + [C.c_void_p]),
    "lica_gpu_trdiag3p_device": (C.c_int, [C.c_void_p] * 4 + [C.c_int64] * 5 + [C.c_void_p]),
    "lica_gpu_trdiag3_noalloc_device": (C.c_int, [C.c_void_p] * 5 + [C.c_int64] * 5 + [C.c_void_p]),
    "lica_gpu_poisson": (C.c_int, [C.c_int64] * 6 + [_D, _D, _D, _I64, _D, _D, _D]),
    "lica_mg_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_double, C.c_double,
                                 C.POINTER(MgOptions)]),
    "lica_mg_destroy": (C.c_int, [C.c_void_p]),
    "lica_mg_solve_host_batch": (C.c_int, [C.c_void_p, C.c_int32] + [C.POINTER(C.c_void_p)] * 4 +
                                 [C.c_double, C.c_int32, C.POINTER(MgResult)]),
    "lica_mg_solve_device": (C.c_int, [C.c_void_p] * 5 + [C.c_double, C.c_int32, C.POINTER(MgResult),
                                                           C.c_void_p]),
    "lica_mg_solve_host": (C.c_int, [C.c_void_p, _D, _D, _D, _D, C.c_double, C.c_int32, C.POINTER(MgResult),
                                      C.c_void_p]),
    "lica_mg_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "lica_mg_profile_read": (C.c_int, [C.c_void_p, C.c_int32, _D, _I64]),
    "lica_mg_precond_device": (C.c_int, [C.c_void_p] * 6),
    "lica_mg_apply_device": (C.c_int, [C.c_void_p] * 6),
    "lica_gpu_lvs_transport": (C.c_int, [C.c_int32, C.c_int32, C.c_double, _D, _I32, _D, _D, _D, _D, _D, _D, _D,
                                         _D, _I32, _D, C.POINTER(LvsParams)]),
    "lica_gpu_lvs_transport_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double] + [C.c_void_p] * 12 +
                                      [C.POINTER(LvsParams), C.c_void_p]),
    "lica_gpu_column_init": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.POINTER(ColProps),
                                       C.POINTER(ColState)]),
    "lica_grid_section": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                    _D]),
    "lica_grid_metrics": (C.c_int, [C.c_int32, _D, _D, _D, _D, _D, _D]),
    "lica_grid_coupling_z": (C.c_int, [C.c_int32, _D, C.c_int32, _D] + [_I32] * 6),
    "lica_mg_stretched_system": (C.c_int, [C.c_int32, C.c_int32, _D, _D, _D, _D, _D, _D, _D]),
    "lica_fld_name": (C.c_int, [C.c_int64, C.c_char_p, C.c_int32]),
    "lica_col_fld_write": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(ColProps), C.POINTER(ColState),
                                     C.POINTER(FldInfo)]),
    "lica_col_fld_dims": (C.c_int, [C.c_char_p, _I32]),
    "lica_col_fld_read": (C.c_int, [C.c_char_p, C.c_int32, C.c_double, C.POINTER(ColProps), C.POINTER(FldOptions),
                                    C.POINTER(ColState), C.POINTER(FldInfo)]),
    "lica_gpu_column_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
    "lica_gpu_column_profile_device": (C.c_int, [C.c_void_p]),
    "lica_gpu_column_history_device": (C.c_int, [C.c_void_p, C.c_int32]),
    "lica_gpu_column_steps_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps),
                                               C.POINTER(ColState), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                               C.c_void_p]),
    "lica_gpu_column_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, _I32, _D, C.POINTER(ColProps)]),
    "lica_gpu_column_batch_destroy": (C.c_int, [C.c_void_p]),
    "lica_gpu_column_batch_layout": (C.c_int, [C.c_void_p, _I64, _I64]),
    "lica_gpu_column_batch_steps_device": (C.c_int, [C.c_void_p, C.POINTER(ColState), C.c_int32, C.c_int32,
                                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "lica_gpu_column_batch_steps_ex_device": (C.c_int, [C.c_void_p, C.POINTER(ColState), C.c_int32, C.c_int32,
                                                        C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "lica_gpu_column_steps": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps), C.POINTER(ColState),
                                        C.c_int32, _I32]),
    "lica_gpu_column_init_geometry": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.POINTER(ColProps),
                                                C.POINTER(ColGeometry), C.POINTER(ColState)]),
    "lica_gpu_column_geometry_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_double,
                                                  C.POINTER(ColGeometry)]),
    "lica_gpu_column_geometry_destroy": (C.c_int, [C.c_void_p]),
    "lica_gpu_column_steps_geometry_device": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ColProps),
                                                        C.POINTER(ColState), C.c_int32, C.c_int32, C.c_void_p,
                                                        C.c_void_p, C.c_void_p]),
    "lica_gpu_column_steps_geometry": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ColProps), C.POINTER(ColState),
                                                 C.c_int32, _I32]),
    "lica_gpu_lvs_transport_geometry": (C.c_int, [C.c_void_p, C.c_int32, _D, _I32, _D, _D, _D, _D, _D, _D, _D, _D,
                                                  _I32, _D, C.POINTER(LvsParams)]),
    "lica_gpu_lvs_transport_geometry_device": (C.c_int, [C.c_void_p, C.c_int32] + [C.c_void_p] * 12 +
                                               [C.POINTER(LvsParams), C.c_void_p]),
    "lica_gpu_reinitialization": (C.c_int, [C.c_int32, C.c_int32, C.c_double, _D, _I32, C.c_int32, _I32]),
    "lica_gpu_reinitialization_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                                   C.c_int32, C.c_void_p, C.c_void_p]),
    "lica_gpu_grid_coupling": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_int32, _D, _I32, _D, _D]),
    "lica_gpu_grid_coupling_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_int32] + [C.c_void_p] * 5),
    "lica_gpu_temp_grad": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps), C.c_double, _D, _D, _D,
                                     _I32, _D, _D, _D, _I32, _D, _I32, _I32]),
    "lica_gpu_temp_grad_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps), C.c_double] +
                                  [C.c_void_p] * 13),
    "lica_gpu_pressure_correction": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps), C.c_double,
                                               _D, _D, _D, _D]),
    "lica_gpu_pressure_correction_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.POINTER(ColProps),
                                                      C.c_double] + [C.c_void_p] * 7),
    "lica_unet_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_int32, C.c_uint64]),
    "lica_unet_destroy": (C.c_int, [C.c_void_p]),
    "lica_unet_param_count": (C.c_int64, [C.c_void_p]),
    "lica_unet_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "lica_unet_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "lica_unet_guess_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "lica_unet_guess_checked_device": (C.c_int, [C.c_void_p] * 5 + [C.c_double, C.c_double, C.c_void_p, _D,
                                                                      C.c_void_p]),
    "lica_unet_grad_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                        C.POINTER(C.c_float), C.c_int64, C.c_void_p]),
    "lica_unet_train_step_device": (C.c_int, [C.c_void_p] + [C.c_void_p] * 5 + [C.c_double, C.c_double, C.c_float,
                                                                              C.POINTER(C.c_double), C.c_void_p]),
    "lica_unet_conv3x3_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                           C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                           C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "lica_film2d_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(Film2DProps), C.c_int32,
                                     C.c_int32]),
    "lica_film2d_destroy": (C.c_int, [C.c_void_p]),
    "lica_film2d_set_guess": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lica_film2d_set_warm_start": (C.c_int, [C.c_void_p, C.c_int32]),
    "lica_film2d_capture_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lica_film2d_step_device": (C.c_int, [C.c_void_p] * 6 + [C.c_double, C.POINTER(Film2DStats), C.c_void_p]),
    "lica_film2d_mdot_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lica_gpu_bubble_grid_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(BubGrid), C.c_int32]),
    "lica_gpu_bubble_grid_destroy": (C.c_int, [C.c_void_p]),
    "lica_gpu_bubble_tracking_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32] + [C.c_void_p] * 4 +
                                        [C.c_double, C.c_int32, C.c_void_p, C.c_void_p]),
    "lica_gpu_bubble_tracking": (C.c_int, [C.POINTER(BubGrid), C.c_int32, C.c_int32] + [_D] * 4 +
                                 [C.c_double, C.c_int32, C.c_void_p]),
}

STATUS = {0: "LICA_OK", 1: "LICA_NOT_CONVERGED", 2: "LICA_BAND_OVERFLOW", 3: "LICA_NAN", 4: "LICA_BAD_ARG",
          5: "LICA_ERR_CUDA", 6: "LICA_ERR_NOMEM", 7: "LICA_ERR_IO", 8: "LICA_STALLED"}


class LicaError(RuntimeError):
    def __init__(self, code, where):
        msg = lib().lica_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(code, code)} {msg}")
        self.code = code


_lib = None


def lib_path() -> str:
    return _build.LIB


def lib():
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise ImportError(f"lica CUDA library not built: {path} is missing (run __graft_entry__.build())")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, where, ok=(0,)):
    if code not in ok:
        raise LicaError(code, where)
    return code


def launch_count() -> int:
    return int(lib().lica_kernel_launch_count())


def poison_shared(value=float("nan"), stream=None):
    """Fill every SM's shared memory with value and wait for it (diagnostic; see
    lica_debug_poison_shared)."""
    import torch
    check(lib().lica_debug_poison_shared(float(value), stream), "lica_debug_poison_shared")
    torch.cuda.synchronize()
