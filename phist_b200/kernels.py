"""ctypes binding of libphist_kernels_b200.so.

Mirrors PHIST's own Python binding (python/phist_kernels.py in the PHIST
sources): the library is loaded with RTLD_GLOBAL, every C entry point is
declared with its argument types and made available as a module attribute of
the same name (``phist_DsparseMat_times_mvec`` etc.), handles are opaque
``c_void_p`` subclasses and the last argument is always ``int* iflag``.

On top of the raw entry points, ``chk(fn, *args)`` calls a function with a
fresh iflag and raises ``PhistError`` on a negative status, the way
PHIST_CHK_IERR propagates errors (src/tools/phist_macros.h:111-133).

There is no fallback: if the CUDA library is missing this module raises at
import time, and every compute call fails when no GPU is present.
"""
import ctypes as _ct
import os as _os

import numpy as _np

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIBPATH = _os.path.join(_HERE, "lib", "libphist_kernels_b200.so")

if not _os.path.exists(LIBPATH):
    raise ImportError(
        "libphist_kernels_b200.so is not built (%s); run `python -m phist_b200.build`" % LIBPATH)
_lib = _ct.CDLL(LIBPATH, mode=_ct.RTLD_GLOBAL)

# status codes (src/tools/phist_defs.h:53-71)
PHIST_SUCCESS = 0
PHIST_FUNCTIONAL_ERROR = -1
PHIST_MEM_ALLOC_FAILED = -44
PHIST_INVALID_INPUT = -55
PHIST_CAUGHT_EXCEPTION = -77
PHIST_BAD_CAST = -88
PHIST_NOT_IMPLEMENTED = -99
# input flags (src/kernels/phist_kernel_flags.h)
PHIST_ROBUST_REDUCTIONS = 1
PHIST_NO_GLOBAL_REDUCTION = 2
PHIST_SPARSEMAT_PERM_LOCAL = 1
PHIST_SPARSEMAT_OPT_CARP = 32
PHIST_SDMAT_RUN_ON_HOST = 1024
PHIST_SDMAT_RUN_ON_DEVICE = 2048
PHIST_MVEC_RUN_ON_DEVICE = 2048


class PhistError(RuntimeError):
    def __init__(self, fname, code):
        RuntimeError.__init__(self, "%s returned iflag=%d" % (fname, code))
        self.code = code
        self.fname = fname


c_int = _ct.c_int
c_int_p = _ct.POINTER(_ct.c_int)
lidx = _ct.c_int32
gidx = _ct.c_int64
lidx_p = _ct.POINTER(lidx)
gidx_p = _ct.POINTER(gidx)
vp = _ct.c_void_p
vpp = _ct.POINTER(_ct.c_void_p)
c_char_p = _ct.c_char_p
u64 = _ct.c_uint64

ROWFUNC = _ct.CFUNCTYPE(c_int, gidx, lidx_p, gidx_p, vp, vp)
ROWFUNC_CTOR = _ct.CFUNCTYPE(c_int, vp, vpp)
ELEMFUNC = _ct.CFUNCTYPE(c_int, gidx, lidx, vp, vp)


def _declare(name, argtypes, restype=None):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = argtypes
    globals()[name] = f
    return f


def declared_names():
    """All entry points this module declares (C symbol names)."""
    return sorted(_DECLARED)


_DECLARED = []


def _d(name, argtypes, restype=None):
    _DECLARED.append(name)
    return _declare(name, argtypes, restype)


# ---------------------------------------------------------------- untyped
_d("phist_kernels_init", [c_int_p, vp, c_int_p])
_d("phist_kernels_finalize", [c_int_p])
_d("phist_kernels_common_init", [c_int_p, vp, c_int_p])
_d("phist_kernels_common_finalize", [c_int_p])
_d("phist_kernel_lib", [], c_char_p)
_d("phist_sizeof_lidx", [], c_int)
_d("phist_sizeof_gidx", [], c_int)
_d("phist_comm_create", [vpp, c_int_p])
_d("phist_comm_delete", [vp, c_int_p])
_d("phist_comm_get_rank", [vp, c_int_p, c_int_p])
_d("phist_comm_get_size", [vp, c_int_p, c_int_p])
_d("phist_comm_get_mpi_comm", [vp, c_int_p, c_int_p])
_d("phist_map_create", [vpp, vp, gidx, c_int_p])
_d("phist_map_delete", [vp, c_int_p])
_d("phist_map_get_comm", [vp, vpp, c_int_p])
_d("phist_map_get_local_length", [vp, lidx_p, c_int_p])
_d("phist_map_get_global_length", [vp, gidx_p, c_int_p])
_d("phist_map_get_ilower", [vp, gidx_p, c_int_p])
_d("phist_map_get_iupper", [vp, gidx_p, c_int_p])
_d("phist_maps_compatible", [vp, vp, c_int_p])
_d("phist_context_create", [vpp, vp, vp, vp, vp, c_int_p])
_d("phist_context_delete", [vp, c_int_p])
for _b in ("load", "store", "copy", "triad"):
    _d("phist_bench_stream_" + _b, [_ct.POINTER(_ct.c_double), _ct.POINTER(_ct.c_double), c_int_p])
_d("phist_b200_set_sell_params", [c_int, _ct.c_int64, c_int_p])
_d("phist_b200_synchronize", [c_int_p])
_d("phist_b200_selftest_bounded_wait", [c_int_p])
_d("phist_b200_lane_count", [c_int_p, c_int_p])
_d("phist_b200_device_memory", [_ct.POINTER(u64), _ct.POINTER(u64), c_int_p])
_d("phist_b200_set_spmv_config", [c_int, c_int, c_int, c_int_p])
_d("phist_b200_set_spmv_staged", [c_int, c_int_p])
_d("phist_b200_set_spmv_prefetch", [c_int, c_int_p])
_d("phist_b200_set_graphs", [c_int, c_int_p])
_d("phist_b200_set_option", [_ct.c_char_p, c_int, c_int_p])
_d("phist_b200_launch_count", [_ct.POINTER(u64), c_int_p])
_d("phist_b200_get_stream", [vpp, c_int_p])
_d("phist_b200_problem_create", [c_char_p, c_int, gidx_p, lidx_p], vp)
_d("phist_b200_problem_rowfunc", [gidx, lidx_p, vp, vp, vp], c_int)
_d("phist_b200_Dcreate_problem", [vpp, vp, c_char_p, c_int_p])
_d("phist_b200_Screate_problem", [vpp, vp, c_char_p, c_int_p])
_d("phist_b200_mvec_DtoS", [vp, vp, c_int_p])
_d("phist_b200_mvec_StoD", [vp, vp, c_int_p])
_d("phist_b200_sparseMat_DtoS", [vp, vpp, c_int_p])
_d("phist_b200_DcarpCG_batch",
   [vp, c_int, vp, vp, vp, c_int, _ct.c_double, c_int, c_int, c_int, _ct.c_double, vp, vp, c_int_p])
_d("phist_b200_DcarpCG_tune_block", [vp, c_int, c_int, c_int, c_int_p, vp, c_int_p])
_d("phist_b200_DmvecT_times_mvec_noalloc",
   [gidx, c_int, c_int, _ct.c_double, vp, gidx, vp, gidx, _ct.c_double, vp, gidx, vp, c_int_p])

# ---------------------------------------------------------------- typed
for _P, _ST in (("D", _ct.c_double), ("S", _ct.c_float)):
    p = "phist_" + _P
    x = "phist_b200_" + _P
    S = _ST
    Sp = _ct.POINTER(_ST)
    Spp = _ct.POINTER(Sp)
    _d(p + "type_avail", [c_int_p])
    for _r in ("read_mm", "read_hb", "read_bin"):
        _d(p + "sparseMat_" + _r, [vpp, vp, c_char_p, c_int_p])
        _d(p + "sparseMat_" + _r + "_with_context", [vpp, vp, c_char_p, c_int_p])
    for _m in ("row", "col", "domain", "range"):
        _d(p + "sparseMat_get_%s_map" % _m, [vp, vpp, c_int_p])
    _d(p + "sparseMat_get_context", [vp, vpp, c_int_p])
    _d(p + "sparseMat_local_nnz", [vp, _ct.POINTER(_ct.c_int64), c_int_p])
    _d(p + "sparseMat_global_nnz", [vp, _ct.POINTER(_ct.c_int64), c_int_p])
    _d(p + "sparseMat_global_nrows", [vp, gidx_p, c_int_p])
    _d(p + "sparseMat_global_ncols", [vp, gidx_p, c_int_p])
    _d(p + "sparseMat_delete", [vp, c_int_p])
    _d(p + "sparseMat_create_fromRowFunc", [vpp, vp, gidx, gidx, lidx, vp, vp, c_int_p])
    _d(p + "sparseMat_create_fromRowFuncAndContext", [vpp, vp, lidx, vp, vp, c_int_p])
    _d(p + "sparseMat_create_fromRowFuncWithConstructor", [vpp, vp, gidx, gidx, lidx, vp, vp, vp, c_int_p])
    _d(p + "sparseMat_create_fromRowFuncWithConstructorAndContext", [vpp, vp, lidx, vp, vp, vp, c_int_p])
    _d(x + "sparseMat_create_fromCRS", [vpp, vp, gidx, gidx, vp, vp, vp, c_int_p])
    _d(x + "sparseMat_sell_info", [vp, c_int_p, _ct.POINTER(_ct.c_int64), _ct.POINTER(_ct.c_int64),
                                   _ct.POINTER(_ct.c_int64), vp, c_int_p])
    _d(x + "sparseMat_autotune", [vp, c_int, vp, c_int, vp, c_int_p])
    _d(x + "jadaCorrection_gmres", [vp, vp, vp, vp, c_int, vp, vp, c_int, c_int, vp, c_int_p])
    _d(x + "jadaCorrection_minres", [vp, vp, vp, vp, c_int, vp, vp, c_int, c_int, vp, c_int_p])
    _d(x + "sparseMat_get_tuning", [vp, c_int_p, _ct.POINTER(_ct.c_int64), vp, vp, vp, c_int_p])
    _d(p + "mvec_create", [vpp, vp, c_int, c_int_p])
    _d(p + "mvec_clone_shape", [vpp, vp, c_int_p])
    _d(p + "mvec_delete", [vp, c_int_p])
    _d(p + "mvec_get_map", [vp, vpp, c_int_p])
    _d(p + "mvec_num_vectors", [vp, c_int_p, c_int_p])
    _d(p + "mvec_my_length", [vp, lidx_p, c_int_p])
    _d(p + "mvec_global_length", [vp, gidx_p, c_int_p])
    _d(p + "mvec_get_comm", [vp, vpp, c_int_p])
    _d(p + "mvec_get_data", [vp, vp, lidx, c_int, c_int_p])
    _d(p + "mvec_set_data", [vp, vp, lidx, c_int, c_int_p])
    _d(p + "mvec_extract_view", [vp, Spp, lidx_p, c_int_p])
    _d(p + "mvec_extract_const_view", [vp, Spp, lidx_p, c_int_p])
    _d(x + "mvec_device_view", [vp, Spp, lidx_p, c_int_p])
    _d(p + "mvec_to_device", [vp, c_int_p])
    _d(p + "mvec_from_device", [vp, c_int_p])
    _d(p + "mvec_write_bin", [vp, c_char_p, c_int_p])
    _d(p + "mvec_read_bin", [vp, c_char_p, c_int_p])
    _d(p + "mvec_to_mvec", [vp, vp, c_int_p])
    _d(p + "mvec_view_block", [vp, vpp, c_int, c_int, c_int_p])
    _d(p + "mvec_get_block", [vp, vp, c_int, c_int, c_int_p])
    _d(p + "mvec_set_block", [vp, vp, c_int, c_int, c_int_p])
    _d(p + "mvec_gather_mvecs", [vp, vpp, c_int, c_int_p])
    _d(p + "mvec_scatter_mvecs", [vp, vpp, c_int, c_int_p])
    _d(p + "mvec_put_value", [vp, S, c_int_p])
    _d(p + "mvec_put_func", [vp, vp, vp, c_int_p])
    _d(p + "mvec_random", [vp, c_int_p])
    _d(p + "mvec_print", [vp, c_int_p])
    _d(p + "mvec_norm2", [vp, Sp, c_int_p])
    _d(p + "mvec_normalize", [vp, Sp, c_int_p])
    _d(p + "mvec_scale", [vp, S, c_int_p])
    _d(p + "mvec_vscale", [vp, Sp, c_int_p])
    _d(p + "mvec_add_mvec", [S, vp, S, vp, c_int_p])
    _d(p + "mvec_vadd_mvec", [Sp, vp, S, vp, c_int_p])
    _d(p + "mvec_times_mvec_elemwise", [S, vp, vp, c_int_p])
    _d(p + "mvec_dot_mvec", [vp, vp, Sp, c_int_p])
    _d(p + "mvecT_times_mvec", [S, vp, vp, S, vp, c_int_p])
    _d(p + "mvec_times_sdMat", [S, vp, vp, S, vp, c_int_p])
    _d(p + "mvec_times_sdMat_inplace", [vp, vp, c_int_p])
    _d(p + "mvec_times_sdMat_add_mvec_times_sdMat", [vp, vp, vp, vp, c_int_p])
    _d(p + "fused_mvsd_mvTmv", [S, vp, vp, S, vp, vp, c_int_p])
    _d(p + "fused_mvsdi_mvTmv", [S, vp, vp, vp, S, vp, c_int_p])
    _d(p + "sparseMat_times_mvec_communicate", [vp, vp, c_int_p])
    _d(p + "sparseMat_times_mvec", [S, vp, vp, S, vp, c_int_p])
    _d(p + "sparseMatT_times_mvec", [S, vp, vp, S, vp, c_int_p])
    _d(p + "sparseMat_times_mvec_add_mvec", [S, vp, S, vp, S, vp, c_int_p])
    _d(p + "sparseMat_times_mvec_vadd_mvec", [S, vp, Sp, vp, S, vp, c_int_p])
    _d(p + "fused_spmv_mvdot", [S, vp, vp, S, vp, Sp, Sp, c_int_p])
    _d(p + "fused_spmv_mvdot_mvadd", [S, vp, vp, S, vp, S, S, vp, Sp, Sp, c_int_p])
    _d(p + "fused_spmv_mvTmv", [S, vp, vp, S, vp, vp, vp, c_int_p])
    _d(p + "fused_spmv_pair", [S, Sp, vp, Sp, vp, vp, S, vp, c_int_p])
    _d(p + "mvec_QR", [vp, vp, c_int_p])
    _d(p + "sdMat_create", [vpp, c_int, c_int, vp, c_int_p])
    _d(p + "sdMat_delete", [vp, c_int_p])
    _d(p + "sdMat_get_nrows", [vp, c_int_p, c_int_p])
    _d(p + "sdMat_get_ncols", [vp, c_int_p, c_int_p])
    _d(p + "sdMat_extract_view", [vp, Spp, lidx_p, c_int_p])
    _d(p + "sdMat_extract_const_view", [vp, Spp, lidx_p, c_int_p])
    _d(p + "sdMat_extract_error", [vp, Spp, c_int_p])
    _d(p + "sdMat_to_device", [vp, c_int_p])
    _d(p + "sdMat_from_device", [vp, c_int_p])
    _d(p + "sdMat_sync_values", [vp, vp, c_int_p])
    _d(p + "sdMat_write_bin", [vp, c_char_p, c_int_p])
    _d(p + "sdMat_read_bin", [vp, c_char_p, c_int_p])
    _d(p + "sdMat_view_block", [vp, vpp, c_int, c_int, c_int, c_int, c_int_p])
    _d(p + "sdMat_get_block", [vp, vp, c_int, c_int, c_int, c_int, c_int_p])
    _d(p + "sdMat_set_block", [vp, vp, c_int, c_int, c_int, c_int, c_int_p])
    _d(p + "sdMat_set_data", [vp, vp, lidx, c_int, c_int_p])
    _d(p + "sdMat_get_data", [vp, vp, lidx, c_int, c_int_p])
    _d(p + "sdMat_random", [vp, c_int_p])
    _d(p + "sdMat_put_value", [vp, S, c_int_p])
    _d(p + "sdMat_identity", [vp, c_int_p])
    _d(p + "sdMat_print", [vp, c_int_p])
    _d(p + "sdMat_add_sdMat", [S, vp, S, vp, c_int_p])
    _d(p + "sdMatT_add_sdMat", [S, vp, S, vp, c_int_p])
    _d(p + "sdMat_times_sdMat", [S, vp, vp, S, vp, c_int_p])
    _d(p + "sdMatT_times_sdMat", [S, vp, vp, S, vp, c_int_p])
    _d(p + "sdMat_times_sdMatT", [S, vp, vp, S, vp, c_int_p])
    _d(p + "carp_setup", [vp, c_int, Sp, vpp, c_int_p])
    _d(p + "carp_setup_rc", [vp, c_int, Sp, Sp, vpp, c_int_p])
    _d(p + "carp_sweep", [vp, Sp, vp, vp, vp, Sp, c_int_p])
    _d(p + "carp_sweep_rc", [vp, Sp, Sp, vp, vp, vp, vp, Sp, c_int_p])
    _d(p + "carp_sweep_aug", [vp, Sp, vp, vp, vp, vp, vp, Sp, c_int_p])
    _d(p + "carp_sweep_aug_rc", [vp, Sp, Sp, vp, vp, vp, vp, vp, vp, vp, Sp, c_int_p])
    _d(p + "carp_destroy", [vp, vp, c_int_p])
    _d(x + "carp_color_order", [vp, vp, c_int_p, vp, c_int_p])


def chk(fn, *args, flags=0):
    """Call ``fn(*args, &iflag)`` with iflag=flags on entry; raise on iflag<0."""
    iflag = c_int(flags)
    ret = fn(*args, _ct.byref(iflag))
    if iflag.value < 0:
        raise PhistError(getattr(fn, "__name__", str(fn)), iflag.value)
    return ret


def iflag_of(fn, *args, flags=0):
    """Call ``fn(*args, &iflag)`` and return iflag (no exception)."""
    iflag = c_int(flags)
    fn(*args, _ct.byref(iflag))
    return iflag.value


def ptr(a):
    """ctypes void pointer to a contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(vp)


def sptr(a, dtype):
    """typed scalar-array pointer for numpy array a (float64 / float32)."""
    ctype = _ct.c_double if dtype == _np.float64 else _ct.c_float
    return a.ctypes.data_as(_ct.POINTER(ctype))
