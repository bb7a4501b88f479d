"""Small object layer over the C ABI (used by the tests, the bench and smoke).

Every method calls the phist_* C entry points of libphist_kernels_b200.so
through ``phist_b200.kernels``; nothing here computes on the host except data
marshalling.
"""
import ctypes as ct

import numpy as np

from . import kernels as K

_P = {np.float64: "D", np.float32: "S"}


def _pfx(dtype):
    return _P[np.dtype(dtype).type]


def fn(dtype, name):
    return getattr(K, "phist_" + _pfx(dtype) + name)


def xfn(dtype, name):
    return getattr(K, "phist_b200_" + _pfx(dtype) + name)


class Session:
    """phist_kernels_init + one comm object (one process, one GPU)."""
    _inst = None

    def __init__(self):
        K.chk(K.phist_kernels_init, None, None)
        self.comm = ct.c_void_p()
        K.chk(K.phist_comm_create, ct.byref(self.comm))

    @classmethod
    def get(cls):
        if cls._inst is None:
            cls._inst = Session()
        return cls._inst


class Map:
    def __init__(self, n, session=None):
        s = session or Session.get()
        self.h = ct.c_void_p()
        self.n = n
        K.chk(K.phist_map_create, ct.byref(self.h), s.comm, n)

    def delete(self):
        if self.h:
            K.chk(K.phist_map_delete, self.h)
            self.h = ct.c_void_p()


class Mvec:
    def __init__(self, map_h, nvec, dtype=np.float64, _handle=None, nrows=None):
        self.dtype = np.dtype(dtype)
        self.nvec = nvec
        self.h = ct.c_void_p() if _handle is None else _handle
        if _handle is None:
            K.chk(fn(dtype, "mvec_create"), ct.byref(self.h), map_h, nvec)
        n = K.lidx()
        K.chk(fn(dtype, "mvec_my_length"), self.h, ct.byref(n))
        self.nrows = n.value
        self._view = _handle is not None

    def set(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.shape == (self.nrows, self.nvec), (a.shape, self.nrows, self.nvec)
        K.chk(fn(self.dtype, "mvec_set_data"), self.h, K.ptr(a), self.nvec, 1)
        return self

    def get(self):
        a = np.empty((self.nrows, self.nvec), self.dtype)
        K.chk(fn(self.dtype, "mvec_get_data"), self.h, K.ptr(a), self.nvec, 1)
        return a

    def view(self, jmin, jmax):
        v = ct.c_void_p()
        K.chk(fn(self.dtype, "mvec_view_block"), self.h, ct.byref(v), jmin, jmax)
        return Mvec(None, jmax - jmin + 1, self.dtype, _handle=v)

    def delete(self):
        if self.h:
            K.chk(fn(self.dtype, "mvec_delete"), self.h)
            self.h = ct.c_void_p()


class SdMat:
    def __init__(self, nrows, ncols, dtype=np.float64, session=None, _handle=None):
        s = session or Session.get()
        self.dtype = np.dtype(dtype)
        self.nrows, self.ncols = nrows, ncols
        self.h = ct.c_void_p() if _handle is None else _handle
        if _handle is None:
            K.chk(fn(dtype, "sdMat_create"), ct.byref(self.h), nrows, ncols, s.comm)

    def set(self, a):
        a = np.asfortranarray(a, dtype=self.dtype)
        assert a.shape == (self.nrows, self.ncols)
        K.chk(fn(self.dtype, "sdMat_set_data"), self.h, K.ptr(a), max(self.nrows, 1), 0)
        return self

    def get(self):
        a = np.zeros((self.nrows, self.ncols), self.dtype, order="F")
        K.chk(fn(self.dtype, "sdMat_get_data"), self.h, K.ptr(a), max(self.nrows, 1), 0)
        return np.ascontiguousarray(a)

    def host(self):
        """the host copy as it is right now (no download)"""
        p = ct.POINTER(ct.c_double if self.dtype == np.float64 else ct.c_float)()
        lda = K.lidx()
        K.chk(fn(self.dtype, "sdMat_extract_view"), self.h, ct.byref(p), ct.byref(lda))
        out = np.zeros((self.nrows, self.ncols), self.dtype)
        for j in range(self.ncols):
            for i in range(self.nrows):
                out[i, j] = p[i + j * lda.value]
        return out

    def delete(self):
        if self.h:
            K.chk(fn(self.dtype, "sdMat_delete"), self.h)
            self.h = ct.c_void_p()


class SparseMat:
    def __init__(self, h, dtype):
        self.h = h
        self.dtype = np.dtype(dtype)
        n = K.gidx()
        K.chk(fn(dtype, "sparseMat_global_nrows"), h, ct.byref(n))
        self.nrows = n.value
        K.chk(fn(dtype, "sparseMat_global_ncols"), h, ct.byref(n))
        self.ncols = n.value
        nnz = ct.c_int64()
        K.chk(fn(dtype, "sparseMat_local_nnz"), h, ct.byref(nnz))
        self.nnz = nnz.value
        m = ct.c_void_p()
        K.chk(fn(dtype, "sparseMat_get_row_map"), h, ct.byref(m))
        self.row_map = m
        m2 = ct.c_void_p()
        K.chk(fn(dtype, "sparseMat_get_domain_map"), h, ct.byref(m2))
        self.domain_map = m2

    @classmethod
    def from_crs(cls, rowptr, col, val, ncols=None, dtype=np.float64, flags=0, session=None):
        s = session or Session.get()
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, dtype)
        n = len(rowptr) - 1
        h = ct.c_void_p()
        K.chk(xfn(dtype, "sparseMat_create_fromCRS"), ct.byref(h), s.comm, n,
              n if ncols is None else ncols, K.ptr(rowptr), K.ptr(col), K.ptr(val), flags=flags)
        return cls(h, dtype)

    @classmethod
    def from_problem(cls, problem, dtype=np.float64, flags=0, session=None):
        s = session or Session.get()
        h = ct.c_void_p()
        f = K.phist_b200_Dcreate_problem if np.dtype(dtype) == np.float64 else K.phist_b200_Screate_problem
        K.chk(f, ct.byref(h), s.comm, problem.encode(), flags=flags)
        return cls(h, dtype)

    def sell_info(self):
        C = ct.c_int()
        sigma = ct.c_int64()
        nch = ct.c_int64()
        npad = ct.c_int64()
        perm = np.zeros(self.nrows, np.int32)
        K.chk(xfn(self.dtype, "sparseMat_sell_info"), self.h, ct.byref(C), ct.byref(sigma),
              ct.byref(nch), ct.byref(npad), K.ptr(perm))
        return dict(C=C.value, sigma=sigma.value, nchunks=nch.value, nnz_padded=npad.value, perm=perm)

    def delete(self):
        if self.h:
            K.chk(fn(self.dtype, "sparseMat_delete"), self.h)
            self.h = ct.c_void_p()


def sync():
    K.chk(K.phist_b200_synchronize)


def launch_count():
    c = ct.c_uint64()
    K.chk(K.phist_b200_launch_count, ct.byref(c))
    return c.value


def stream_handle():
    s = ct.c_void_p()
    K.chk(K.phist_b200_get_stream, ct.byref(s))
    return s.value or 0
