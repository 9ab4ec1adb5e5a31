"""The C-ABI library loads and exports every symbol include/lica_gpu.h declares (no
compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from lica_boiling1d_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "lica_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(lica_\w+)\s*\(", txt)))


def test_header_declares_expected_entry_points():
    syms = declared_symbols()
    for s in ("lica_gpu_poisson", "lica_gpu_trdiag3", "lica_gpu_trdiag3p", "lica_mg_create", "lica_mg_solve_device",
              "lica_mg_solve_host"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) == set(native.SIGNATURES), set(declared_symbols()) ^ set(native.SIGNATURES)


def test_fortran_module_is_current_and_complete():
    """include/lica_gpu.f90 is what include/make_fortran_module.py writes from the header
    (not compiled here: the image has no Fortran compiler), with one bind(c) interface of
    the right arity per declared entry point."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_fortran_module",
                                                  os.path.join(ROOT, "include", "make_fortran_module.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    text = gen.generate()
    assert open(os.path.join(ROOT, "include", "lica_gpu.f90")).read() == text
    _, _, _, funcs = gen.parse(open(os.path.join(ROOT, "include", "lica_gpu.h")).read())
    assert sorted(f for f, _, _ in funcs) == declared_symbols()
    flat = re.sub(r"&\s*\n\s*", "", text)
    for name, _, params in funcs:
        m = re.search(r"function %s\(([^)]*)\)\s*bind\(c, name=\"%s\"\)" % (name, name), flat)
        assert m, name
        args = [a.strip() for a in m.group(1).split(",") if a.strip()]
        assert args == [p for p, _ in params], name
    assert all(len(line) <= 100 for line in text.splitlines())


def test_new_entry_points_refuse_bad_arguments_before_any_device_work():
    """The geometry, y-line and batch-shape entry points check their arguments on the host
    and return LICA_BAD_ARG (4) before touching a device, so these calls run without a GPU."""
    import ctypes as C
    L = native.lib()
    bad = 4
    st = native.ColState()
    props = native.ColProps()
    status = (C.c_int32 * 4)()
    # a null geometry handle
    assert L.lica_gpu_column_steps_geometry_device(None, 1, C.byref(props), C.byref(st), 1, 0, None,
                                                   C.cast(status, C.c_void_p), None) == bad
    assert L.lica_gpu_column_steps_geometry(None, 1, C.byref(props), C.byref(st), 1, status) == bad
    prm = native.LvsParams(1, 1, 1, 1, 1000.0, 1e-3)
    args = [None] * 12
    assert L.lica_gpu_lvs_transport_geometry_device(None, 1, *args, C.byref(prm), None) == bad
    # a geometry with null arrays, and a null output handle
    g = native.ColGeometry()
    h = C.c_void_p()
    assert L.lica_gpu_column_geometry_create(C.byref(h), 64, 1.0, C.byref(g)) == bad and not h.value
    assert L.lica_gpu_column_geometry_create(None, 64, 1.0, C.byref(g)) == bad
    # y-line smoothing is FP64 only; unknown smoothers are refused
    for prec, sm in ((1, 1), (0, 2)):
        o = native.MgOptions(6, 2, 2, 1, prec, 1, sm)
        assert L.lica_mg_create(C.byref(h), 1024, 1024, 1.0 / 1024, 1.0 / 1024, C.byref(o)) == bad
