"""phist_b200 -- B200 kernel library behind PHIST's phist_kernels C API.

The product is the shared library lib/libphist_kernels_b200.so (CUDA for
sm_100a, C ABI in include/phist_b200_kernels.h).  This package holds its
sources (csrc/), its build script (build.py), a ctypes binding that mirrors
PHIST's Python binding (kernels.py), a small object layer (objects.py) and the
seeded synthetic problem generators (generators.py).
"""
import os

LIBPATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libphist_kernels_b200.so")


def load():
    """Import the ctypes binding (raises ImportError if the library is not built)."""
    from . import kernels
    return kernels
