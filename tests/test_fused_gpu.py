"""Single-pass fused SpMMV operations and the block gather/scatter.

* fused_spmv_mvTmv (phist_kernels_fused_decl.h:57-68): W = alpha A V + beta W
  with W'W and V'W formed from the new rows of W in the same pass.  W must
  equal the plain SpMMV bit for bit (same row arithmetic), the products the
  oracle's at 1e-13; W = NULL (products only) and beta != 0 are covered, on
  stencil matrices with sigma-sorted and unsorted SELL layouts and tile
  counts that leave partial tiles.
* fused_spmv_pair (:45-48): Y = alpha (s1_j A1 + s2_j A2) X + beta Y in one
  pass over two matrices whose SELL layouts differ (one row-permuted by the
  sigma sort, one not), against the composition PHIST's fallback computes
  (common/kernels_no_fused_spmv_pair.cpp), 1e-13.
* mvec_gather_mvecs / mvec_scatter_mvecs (phist_kernels_decl.h:736-737,
  mvec_module.F90:1005-1145): blocks side by side into one mvec and back,
  bit for bit.
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.fixture
def sell_default(session):
    from phist_b200 import kernels as K
    yield
    K.chk(K.phist_b200_set_sell_params, 32, 256)


@pytest.mark.parametrize("prob,sigma", [("ANDERSON3D-26-S1", 256), ("LAPLACE3D-23", 256), ("LAPLACE3D-23", 1),
                                        ("HONEYCOMB-41x23-S4", 256)])
@pytest.mark.parametrize("nvec", [1, 2, 4, 8, 16, 32])
def test_fused_spmv_mvTmv_single_pass(session, oracle, sell_default, prob, sigma, nvec):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SdMat, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, sigma)
    rp, c, v = G.problem(prob)
    A = SparseMat.from_crs(rp, c, v, flags=K.PHIST_SPARSEMAT_PERM_LOCAL if sigma > 1 else 0)
    n = len(rp) - 1
    x = G.random_block(n, nvec, 41)
    w0 = G.random_block(n, nvec, 42)
    X = Mvec(A.domain_map, nvec).set(x)
    W = Mvec(A.row_map, nvec)
    P = Mvec(A.row_map, nvec)
    Gw, Gv = SdMat(nvec, nvec), SdMat(nvec, nvec)
    for alpha, beta in ((1.0, 0.0), (-0.5, 2.0)):
        W.set(w0)
        K.chk(K.phist_Dfused_spmv_mvTmv, alpha, A.h, X.h, beta, W.h, Gw.h, Gv.h)
        P.set(w0)
        K.chk(K.phist_DsparseMat_times_mvec, alpha, A.h, X.h, beta, P.h)
        wn = W.get()
        assert np.array_equal(wn, P.get())
        ref = oracle.spmmv(rp, c, v, x, alpha=alpha, beta=beta, y=w0)
        assert relerr(wn, ref) < TOL
        assert relerr(Gw.get(), ref.T @ ref) < TOL
        assert relerr(Gv.get(), x.T @ ref) < TOL
    # W = NULL: the products of alpha A V only (fused_decl.h:67)
    Gw2 = SdMat(nvec, nvec)
    K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, None, Gw2.h, None)
    ref = oracle.spmmv(rp, c, v, x)
    assert relerr(Gw2.get(), ref.T @ ref) < TOL
    # bitwise reproducible
    K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, None, Gw.h, None)
    assert np.array_equal(Gw.get(), Gw2.get())
    for o in (X, W, P, Gw, Gv, Gw2, A):
        o.delete()


def test_fused_spmv_mvTmv_anderson_L128(session, oracle):
    """the benchmark matrix (n = 2,097,152) at block width 8"""
    import os

    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SdMat, SparseMat
    oracle.set_threads(os.cpu_count() or 1)
    rp, c, v = G.anderson3d(128, 1)
    A = SparseMat.from_problem("ANDERSON3D-128-S1", flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n = A.nrows
    x = G.random_block(n, 8, 3)
    X = Mvec(A.domain_map, 8).set(x)
    W = Mvec(A.row_map, 8)
    Gw, Gv = SdMat(8, 8), SdMat(8, 8)
    K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, W.h, Gw.h, Gv.h)
    ref = oracle.spmmv(rp, c, v, x)
    assert relerr(W.get(), ref) < TOL
    assert relerr(Gw.get(), ref.T @ ref) < TOL
    assert relerr(Gv.get(), x.T @ ref) < TOL
    for o in (X, W, Gw, Gv, A):
        o.delete()


@pytest.mark.parametrize("nvec", [1, 3, 8, 32, 40])
def test_fused_spmv_pair_single_pass(session, oracle, sell_default, nvec):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp1, c1, v1 = G.problem("LAPLACE3D-23")
    rp2, c2, v2 = G.problem("LAPDIAG3D-23-S5")
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    A1 = SparseMat.from_crs(rp1, c1, v1, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)  # rows sorted: permuted
    K.chk(K.phist_b200_set_sell_params, 32, 1)
    A2 = SparseMat.from_crs(rp2, c2, v2)
    assert not np.array_equal(A1.sell_info()["perm"], np.arange(A1.nrows))
    n = A1.nrows
    rng = np.random.default_rng(nvec)
    x = G.random_block(n, nvec, 51)
    y0 = G.random_block(n, nvec, 52)
    s1 = rng.uniform(-2, 2, nvec)
    s2 = rng.uniform(-2, 2, nvec)
    X = Mvec(A1.domain_map, nvec).set(x)
    Y = Mvec(A1.row_map, nvec)
    for alpha, beta in ((0.5, 2.0), (1.0, 0.0)):
        Y.set(y0)
        K.chk(K.phist_Dfused_spmv_pair, alpha, K.sptr(s1, np.float64), A1.h, K.sptr(s2, np.float64), A2.h,
              X.h, beta, Y.h)
        t1 = oracle.spmmv(rp1, c1, v1, x, alpha=alpha)
        t2 = oracle.spmmv(rp2, c2, v2, x, alpha=alpha)
        ref = s2 * t2 + (s1 * t1 + beta * y0)
        assert relerr(Y.get(), ref) < TOL, (alpha, beta)
    for o in (X, Y, A1, A2):
        o.delete()


def test_gather_scatter_mvecs(session):
    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec
    n = 30011
    mp = Map(n)
    widths = [2, 4, 1, 3]
    blocks = [random_block(n, w, 60 + i) for i, w in enumerate(widths)]
    Ws = [Mvec(mp.h, w).set(b) for w, b in zip(widths, blocks)]
    V = Mvec(mp.h, 12).set(np.full((n, 12), 9.0))
    arr = (ct.c_void_p * len(Ws))(*[w.h.value for w in Ws])
    K.chk(K.phist_Dmvec_gather_mvecs, V.h, arr, len(Ws))
    full = V.get()
    assert np.array_equal(full[:, :10], np.hstack(blocks))
    assert np.all(full[:, 10:] == 9.0)
    # scatter a changed V back into the blocks; a strided view as the source
    new = random_block(n, 12, 70)
    V.set(new)
    Vv = V.view(1, 10)
    K.chk(K.phist_Dmvec_scatter_mvecs, Vv.h, arr, len(Ws))
    off = 1
    for w, W in zip(widths, Ws):
        assert np.array_equal(W.get(), new[:, off:off + w])
        off += w
    # more block columns than V has: rejected
    small = Mvec(mp.h, 5)
    assert K.iflag_of(K.phist_Dmvec_gather_mvecs, small.h, arr, len(Ws)) == K.PHIST_INVALID_INPUT
    for o in Ws + [Vv, V, small, mp]:
        o.delete()
