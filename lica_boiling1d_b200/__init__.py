"""B200 (sm_100a) hot path of the lica two-phase boiling solver.

The CUDA kernels live in csrc/ and are reached through the C ABI declared in
include/lica_gpu.h (liblica_gpu.so, built in-tree by build.py).  Importing the
package does not load the library; the first call into ``native.lib()`` does, and it
raises if the library is missing -- there is no CPU fallback.
"""
from . import build  # noqa: F401

__all__ = ["build", "native", "poisson", "inputs"]
