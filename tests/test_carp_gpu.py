"""CARP sweeps on the GPU (carp_setup / carp_sweep / carp_destroy).

Two layouts: the default block-coloured sweep (row blocks with their X
footprint staged in shared memory, one launch per block colour) and the
row-colour sweep (one launch per class of a distance-2 colouring; option
carp_blocks = 0).  Either must equal the oracle's sequential Kaczmarz sweep
over the row order the library reports (kacz_sub_def.h update formulae) to
rounding, the segments of that order must be distance-2 independent sets,
repeated sweeps must be bitwise reproducible (the reference's CarpTest checks
repeatability, CarpTest_def.hpp:579-611), and sweeps must drive the residual
of (A - sigma I) x = b down.  The block sweep is also checked at the
benchmarked size (honeycomb 1024 x 1024 x 2 sites, 8 shifts).
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import relerr, sort_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[1, 0], ids=["blocks", "rowcolour"])
def layout(request, session):
    from phist_b200 import kernels as K
    K.chk(K.phist_b200_set_option, b"carp_blocks", request.param)
    yield request.param
    K.chk(K.phist_b200_set_option, b"carp_blocks", 1)


def _setup(A, shifts, dtype=np.float64):
    from phist_b200 import kernels as K
    from phist_b200.objects import fn
    work = ct.c_void_p()
    sh = np.ascontiguousarray(shifts, dtype)
    K.chk(fn(dtype, "carp_setup"), A.h, len(sh), K.sptr(sh, dtype), ct.byref(work))
    return work, sh


def _with_diagonal(rp, c):
    cols = []
    prp = [0]
    for i in range(len(rp) - 1):
        row = list(c[rp[i]:rp[i + 1]])
        if i not in row:
            row.append(i)
        cols.extend(row)
        prp.append(len(cols))
    return np.array(prp, np.int64), np.array(cols, np.int32)


def _order(work, n):
    from phist_b200 import kernels as K
    rows = np.zeros(n, np.int32)
    nc = ct.c_int()
    K.chk(K.phist_b200_Dcarp_color_order, work, K.ptr(rows), ct.byref(nc), None)
    cp = np.zeros(nc.value + 1, np.int64)
    K.chk(K.phist_b200_Dcarp_color_order, work, None, None, K.ptr(cp))
    return rows, cp


@pytest.mark.parametrize("prob,nvec", [("sprandn388", 1), ("sprandn388", 4), ("symmMat20", 3),
                                       ("spshift388", 8), ("jadaTestMat512", 2),
                                       ("sprandn_nodiag388", 4), ("spshift25", 1)])
def test_carp_sweep_vs_oracle(session, layout, oracle, testmats, prob, nvec):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v, shape = testmats(prob)
    A = SparseMat.from_crs(rp, c, v, ncols=shape[1])
    n = shape[0]
    rng = np.random.default_rng(nvec)
    shifts = rng.uniform(-1, 1, nvec)
    omega = rng.uniform(0.8, 1.6, nvec)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    work, sh = _setup(A, shifts)
    rows, cp = _order(work, n)
    assert sorted(rows) == list(range(n))
    colour = np.zeros(n, np.int32)
    for k in range(len(cp) - 1):
        colour[rows[cp[k]:cp[k + 1]]] = k
    # the shift term writes x_i, so every row's own index belongs to its pattern
    prp, pcol = _with_diagonal(rp, c)
    assert oracle.check_dist2(prp, pcol, shape[1], colour) == 0
    X = Mvec(A.row_map, nvec).set(x0)
    B = Mvec(A.row_map, nvec).set(b)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    ref = oracle.carp_sweep(rp, c, v, shifts, b, x0, omega, order=rows)
    assert relerr(X.get(), ref) < 1e-13
    # rhs NULL means b = 0
    X.set(x0)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), None, X.h, work, K.sptr(omega, np.float64))
    ref0 = oracle.carp_sweep(rp, c, v, shifts, None, x0, omega, order=rows)
    assert relerr(X.get(), ref0) < 1e-13
    # repeatability
    X.set(x0)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    again = X.get()
    X.set(x0)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    assert np.array_equal(again, X.get())
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (X, B, A):
        o.delete()


def test_carp_converges_honeycomb(session, oracle):
    """many sweeps on the shifted honeycomb operator reduce the residual of
    the normal equations; real shifts inside the spectrum"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = G.honeycomb(24, 24, 4)
    n = len(rp) - 1
    A = SparseMat.from_crs(rp, c, v)
    nvec = 4
    shifts = np.array([-2.0, -0.5, 0.7, 2.2])
    omega = np.ones(nvec)
    b = G.random_block(n, nvec, 11)
    work, sh = _setup(A, shifts)
    X = Mvec(A.row_map, nvec)
    B = Mvec(A.row_map, nvec).set(b)
    for _ in range(200):
        K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    x = X.get()
    r = b - oracle.spmmv(rp, c, v, x, shifts=-shifts)
    assert np.all(np.linalg.norm(r, axis=0) < 0.3 * np.linalg.norm(b, axis=0))
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (X, B, A):
        o.delete()


def test_carp_rc_reduces_to_real(session, layout, oracle, testmats):
    """complex-shift variant with zero imaginary parts equals the real sweep"""
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v, shape = testmats("sprandn388")
    A = SparseMat.from_crs(rp, c, v)
    n, nvec = 388, 2
    sr = np.array([0.3, -0.4])
    si = np.zeros(2)
    om = np.array([1.0, 1.2])
    rng = np.random.default_rng(3)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    work = ct.c_void_p()
    K.chk(K.phist_Dcarp_setup_rc, A.h, 2, K.sptr(sr, np.float64), K.sptr(si, np.float64), ct.byref(work))
    rows, _ = _order(work, n)
    Xr = Mvec(A.row_map, nvec).set(x0)
    Xi = Mvec(A.row_map, nvec)
    B = Mvec(A.row_map, nvec).set(b)
    K.chk(K.phist_Dcarp_sweep_rc, A.h, K.sptr(sr, np.float64), K.sptr(si, np.float64), B.h, Xr.h, Xi.h,
          work, K.sptr(om, np.float64))
    ref = oracle.carp_sweep(rp, c, v, sr, b, x0, om, order=rows)
    assert relerr(Xr.get(), ref) < 1e-13
    assert np.abs(Xi.get()).max() == 0.0
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (Xr, Xi, B, A):
        o.delete()


@pytest.mark.parametrize("nvec", [8, 32])
def test_carp_block_sweep_benchmark_size(session, oracle, nvec):
    """the benchmarked matrix: honeycomb 1024 x 1024 cells, 2 sites each
    (n = 2,097,152), block layout, against the oracle's sequential sweep in
    the reported order"""
    import os

    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    oracle.set_threads(os.cpu_count() or 1)
    rp, c, v = G.honeycomb(1024, 1024, 1)
    n = len(rp) - 1
    A = SparseMat.from_crs(rp, c, v)
    rng = np.random.default_rng(nvec)
    shifts = rng.uniform(-2, 2, nvec)
    omega = np.full(nvec, 1.2)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    work, sh = _setup(A, shifts)
    rows, cp = _order(work, n)
    assert len(cp) - 1 <= 64  # block colours x steps: few segments
    X = Mvec(A.row_map, nvec).set(x0)
    B = Mvec(A.row_map, nvec).set(b)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    ref = oracle.carp_sweep(rp, c, v, shifts, b, x0, omega, order=rows)
    assert relerr(X.get(), ref) < 1e-13
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (X, B, A):
        o.delete()


def test_carp_sweep_strided_views(session, layout, oracle):
    """X and B as column views of wider mvecs (leading dimension > nvec)"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = G.honeycomb(30, 20, 2)
    n = len(rp) - 1
    A = SparseMat.from_crs(rp, c, v)
    nvec = 3
    rng = np.random.default_rng(9)
    shifts = rng.uniform(-1, 1, nvec)
    omega = np.ones(nvec)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    work, sh = _setup(A, shifts)
    rows, _ = _order(work, n)
    Xw = Mvec(A.row_map, 7).set(rng.uniform(-1, 1, (n, 7)))
    Bw = Mvec(A.row_map, 5).set(rng.uniform(-1, 1, (n, 5)))
    X = Xw.view(2, 4)
    B = Bw.view(1, 3)
    X.set(x0)
    B.set(b)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    ref = oracle.carp_sweep(rp, c, v, shifts, b, x0, omega, order=rows)
    assert relerr(X.get(), ref) < 1e-13
    full = Xw.get()
    assert relerr(full[:, 2:5], ref) < 1e-13
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (X, B, Xw, Bw, A):
        o.delete()


def test_carp_sweep_repeated_columns(session, layout, oracle):
    """rows that hold a column twice (the diagonal split into two entries and
    an off-diagonal entry repeated): every entry is its own projection term,
    as in the sequential sweep"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp0, c0, v0 = G.honeycomb(20, 16, 5)
    n = len(rp0) - 1
    rows_c, rows_v = [], []
    for i in range(n):
        cc = list(c0[rp0[i]:rp0[i + 1]])
        vv = list(v0[rp0[i]:rp0[i + 1]])
        if i % 3 == 0:
            k = cc.index(i)
            vv[k] *= 0.5
            cc.append(i)
            vv.append(vv[k])
        if i % 5 == 1:
            cc.append(cc[0])
            vv.append(0.25)
        rows_c.append(cc)
        rows_v.append(vv)
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(x) for x in rows_c])
    # the library keeps the entries of a row stably sorted by column
    rp, c, v = sort_rows(rp, np.concatenate(rows_c).astype(np.int32), np.concatenate(rows_v))
    A = SparseMat.from_crs(rp, c, v)
    nvec = 4
    rng = np.random.default_rng(17)
    shifts = rng.uniform(-1, 1, nvec)
    omega = rng.uniform(0.8, 1.4, nvec)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    work, sh = _setup(A, shifts)
    rows, _ = _order(work, n)
    X = Mvec(A.row_map, nvec).set(x0)
    B = Mvec(A.row_map, nvec).set(b)
    K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work, K.sptr(omega, np.float64))
    ref = oracle.carp_sweep(rp, c, v, shifts, b, x0, omega, order=rows)
    assert relerr(X.get(), ref) < 1e-13
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    for o in (X, B, A):
        o.delete()


def test_set_option_rejects_unknown_names(session):
    from phist_b200 import kernels as K
    assert K.iflag_of(K.phist_b200_set_option, b"no_such_option", 1) < 0
