"""Build libphist_kernels_b200.so (sm_100a) in-tree with nvcc.

    python -m phist_b200.build          # or phist_b200.build.build()

The CUDA sources under phist_b200/csrc/ are compiled for sm_100a only and
linked into one shared library, phist_b200/lib/libphist_kernels_b200.so,
whose exported symbols are the C ABI declared in include/phist_b200_kernels.h.
Object files are rebuilt only when a source or header is newer.

build_solvers() then compiles PHIST's unchanged solver layers against that
library, together with this package's FP32 correction solver and the drivers
(phist_b200/solvers/Makefile), when the PHIST sources are reachable
(the PHIST_SRC environment variable names the PHIST source tree); without
them the prebuilt outputs in phist_b200/lib are used.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILDDIR = os.path.join(HERE, "_build")
LIBNAME = "libphist_kernels_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

SOURCES = ["pb_runtime.cu", "pb_api_D.cu", "pb_api_S.cu", "pb_api_mixed.cu", "pb_matfuncs.cu",
           "pb_noalloc.cu", "pb_carpcg.cu", "pb_tune.cu",
           "pb_gmres.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
              "--expt-relaxed-constexpr", "-diag-suppress", "550,177"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".cuh", ".hpp", ".inc", ".h"))]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src):
    obj = os.path.join(BUILDDIR, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + _headers()
    if not _stale(obj, deps):
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj


def build(verbose=False):
    """Compile every CUDA source for sm_100a and link the shared library."""
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if _stale(LIBPATH, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIBPATH] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    if verbose:
        print("built", LIBPATH)
    return LIBPATH


def openblas_path():
    """The LAPACK/BLAS the solver layers link: $OPENBLAS, else the OpenBLAS
    that the installed scipy bundles (exports LAPACKE_* and BLAS under the
    scipy_ prefix, 32-bit integers)"""
    env = os.environ.get("OPENBLAS")
    if env:
        return env
    try:
        import glob

        import scipy
        libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        cand = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so")))
        return cand[0] if cand else None
    except ImportError:
        return None


def build_solvers(verbose=False):
    """make -C phist_b200/solvers (PHIST solver layers + drivers), if the
    PHIST sources are present; returns True when they were built"""
    src = os.environ.get("PHIST_SRC", "")
    if not src or not os.path.isdir(os.path.join(src, "src", "jada")):
        return False
    blas = openblas_path()
    if not blas:
        raise RuntimeError("no OpenBLAS shared library found (scipy's bundled libscipy_openblas); "
                           "set OPENBLAS to its path")
    env = dict(os.environ, PHIST_SRC=src)
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "solvers"), "CXX_=g++", "CC_=gcc",
                    "OPENBLAS=" + blas], check=True, env=env)
    if verbose:
        print("built PHIST solver layers into", LIBDIR)
    return True


if __name__ == "__main__":
    build(verbose=True)
    build_solvers(verbose=True)
    sys.exit(0)
