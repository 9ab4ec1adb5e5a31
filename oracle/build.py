"""Build recipe for the oracle (test infrastructure, not the product).

Compiles the C++ restatement under oracle/ into oracle/_build/liblica_oracle.so.
FP64 semantics are kept strict: no fast-math and no FMA contraction, so the CUDA
kernels (built with -fmad=false) can be compared bit for bit where the algorithm
allows it.  ``native=True`` builds an -march=native copy for CPU-baseline timing on
the machine that runs it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["mg2d.cpp", "tridiag.cpp", "lvs1d.cpp", "column1d.cpp", "film2d.cpp", "bubble3d.cpp"]


def lib_path(native: bool = False) -> str:
    return os.path.join(HERE, "_build", "native" if native else "portable", "liblica_oracle.so")


def build(native: bool = False, force: bool = False) -> str:
    out = lib_path(native)
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    if not force and os.path.exists(out):
        mt = os.path.getmtime(out)
        hdrs = [os.path.join(HERE, h) for h in os.listdir(HERE) if h.endswith(".hpp")]
        if all(os.path.getmtime(s) <= mt for s in srcs + hdrs + [__file__]):
            return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    arch = "-march=native" if native else "-march=x86-64-v2"
    opt = "-O3" if native else "-O2"
    cmd = ["g++", "-std=c++17", opt, arch, "-fno-fast-math", "-ffp-contract=off", "-fopenmp",
           "-fPIC", "-shared", "-o", out + ".tmp"] + srcs
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(native="--native" in sys.argv, force=True))
