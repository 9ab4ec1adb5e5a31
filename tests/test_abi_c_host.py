"""The C ABI from a compiled host: tests/abi/host_restart.c, built with gcc against
include/lica_gpu.h and linked to the library, drives the host entry points (column
initial state, fld restart files, grid sections and metrics) the way a Fortran or C solver
would.  No GPU."""
import os
import shutil
import subprocess

import pytest

from lica_boiling1d_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_compiled_host_drives_restart_and_grid_entry_points(tmp_path):
    lib = build.build()
    exe = str(tmp_path / "host_restart")
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi", "host_restart.c"), lib, "-Wl,-rpath," + libdir,
                    "-Wl,--allow-shlib-undefined", "-lm", "-o", exe], check=True)
    out = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_compiled_host_drives_gpu_entry_points(tmp_path):
    """tests/abi/host_gpu.c: POISSON, the 2-D multigrid solve, whole column steps, the
    single-routine drop-ins and the bubble statistics, called from C with host arrays through
    the header alone."""
    lib = build.build()
    exe = str(tmp_path / "host_gpu")
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-O1", "-Wall", "-Werror", "-D_DEFAULT_SOURCE", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi", "host_gpu.c"), lib, "-Wl,-rpath," + libdir,
                    "-Wl,--allow-shlib-undefined", "-lm", "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr
