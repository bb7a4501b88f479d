"""The C ABI: the built library loads on a CPU-only machine and exports every
entry point that include/*.h declares; the ctypes binding covers them; and
without a GPU the library refuses to run instead of computing on the host."""
import ctypes as ct
import os
import re
import subprocess

import pytest

from conftest import ROOT, have_gpu

HEADER = os.path.join(ROOT, "include", "phist_b200_kernels.h")


def declared_functions():
    out = subprocess.run(["gcc", "-E", "-P", "-x", "c", HEADER], capture_output=True, text=True,
                         check=True).stdout
    names = set()
    for decl in out.replace("\n", " ").split(";"):
        decl = decl.strip()
        if decl.startswith("typedef") or "(" not in decl:
            continue
        m = re.match(r"^(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", decl)
        if m:
            names.add(m.group(1))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_header_compiles_as_c_and_cxx():
    for lang in ("c", "c++"):
        subprocess.run(["gcc", "-fsyntax-only", "-Wall", "-Werror", "-x", lang, HEADER], check=True)


def test_library_exports_every_declared_symbol(lib_built):
    from phist_b200 import LIBPATH
    decl = declared_functions()
    assert len(decl) > 200
    exp = exported_symbols(LIBPATH)
    missing = sorted(decl - exp)
    assert not missing, missing


def test_binding_declares_only_exported(lib_built):
    from phist_b200 import LIBPATH
    from phist_b200 import kernels as K
    exp = exported_symbols(LIBPATH)
    names = set(K.declared_names())
    assert names <= exp, sorted(names - exp)
    # every declared C function is reachable from Python
    assert declared_functions() <= names | {"phist_b200_problem_rowfunc"}


def test_reference_api_surface_present(lib_built):
    """the entry points PHIST's solver layers call on the hot path"""
    from phist_b200 import LIBPATH
    exp = exported_symbols(LIBPATH)
    for n in ["sparseMat_times_mvec", "sparseMat_times_mvec_vadd_mvec", "sparseMat_times_mvec_add_mvec",
              "fused_spmv_mvdot", "fused_spmv_mvTmv", "fused_spmv_mvdot_mvadd", "fused_spmv_pair",
              "mvecT_times_mvec", "mvec_times_sdMat", "mvec_times_sdMat_inplace",
              "mvec_times_sdMat_add_mvec_times_sdMat", "fused_mvsd_mvTmv", "fused_mvsdi_mvTmv",
              "mvec_dot_mvec", "mvec_norm2", "mvec_vadd_mvec", "carp_setup", "carp_sweep",
              "carp_destroy", "mvec_QR", "mvec_view_block", "sdMat_from_device"]:
        for p in ("D", "S"):
            assert "phist_%s%s" % (p, n) in exp


def test_kernel_lib_name(lib_built):
    from phist_b200 import kernels as K
    assert K.phist_kernel_lib() == b"b200"
    assert K.phist_sizeof_lidx() == 4 and K.phist_sizeof_gidx() == 8


@pytest.mark.skipif(have_gpu(), reason="only meaningful without a GPU")
def test_no_gpu_means_error_not_fallback(lib_built):
    from phist_b200 import kernels as K
    os.environ["PHIST_B200_QUIET"] = "1"
    iflag = K.iflag_of(K.phist_kernels_init, None, None)
    assert iflag == K.PHIST_FUNCTIONAL_ERROR
    comm = ct.c_void_p()
    assert K.iflag_of(K.phist_comm_create, ct.byref(comm)) < 0
