"""Block products and BLAS1 kernels on the GPU against the oracle
(MvecSdMatTest_def.hpp / MvecSdMatFusedTest_def.hpp / MvecTest_def.hpp
cases: full vectors, views, in-place, fused, robust reductions)."""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13

SHAPES = [(1, 1), (2, 3), (4, 4), (5, 7), (8, 8), (4, 40), (40, 4), (16, 16), (32, 32), (64, 64), (13, 29),
          (24, 8), (8, 24), (64, 16), (16, 64), (40, 56)]


def _mk(n, ncol, data, dtype=np.float64):
    from phist_b200.objects import Map, Mvec
    m = Map(n)
    v = Mvec(m.h, ncol, dtype).set(data)
    return m, v


@pytest.mark.parametrize("m,k", SHAPES)
@pytest.mark.parametrize("n", [1000, 70001])
def test_mvecT_times_mvec(session, oracle, n, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    rng = np.random.default_rng(m * 100 + k)
    V = rng.uniform(-1, 1, (n, m))
    W = rng.uniform(-1, 1, (n, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W)
    C0 = rng.uniform(-1, 1, (m, k))
    C = SdMat(m, k).set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vh.h, Wh.h, 2.0, C.h)
    ref = oracle.mvTmv(V, W, alpha=0.5, beta=2.0, C=C0)
    assert relerr(C.get(), ref) < TOL
    # host copy is coherent without an explicit download
    assert relerr(C.host(), ref) < TOL
    # determinism: same launch, same bits
    C.set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vh.h, Wh.h, 2.0, C.h)
    first = C.get()
    C.set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vh.h, Wh.h, 2.0, C.h)
    assert np.array_equal(first, C.get())
    for o in (Vh, Wh, C, mp):
        o.delete()


def test_mvecT_times_mvec_views(session, oracle):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 5000
    rng = np.random.default_rng(1)
    V = rng.uniform(-1, 1, (n, 10))
    W = rng.uniform(-1, 1, (n, 9))
    mp, Vh = _mk(n, 10, V)
    _, Wh = _mk(n, 9, W)
    Vv = Vh.view(2, 6)
    Wv = Wh.view(1, 3)
    C = SdMat(8, 8)
    Cv = __import__("ctypes").c_void_p()
    K.chk(K.phist_DsdMat_view_block, C.h, __import__("ctypes").byref(Cv), 1, 5, 2, 4)
    K.chk(K.phist_DmvecT_times_mvec, 1.0, Vv.h, Wv.h, 0.0, Cv)
    full = C.get()
    ref = np.zeros((8, 8))
    ref[1:6, 2:5] = V[:, 2:7].T @ W[:, 1:4]
    assert relerr(full, ref) < TOL
    K.chk(K.phist_DsdMat_delete, Cv)
    for o in (Vv, Wv, Vh, Wh, C, mp):
        o.delete()


@pytest.mark.parametrize("m,k", SHAPES)
def test_mvec_times_sdMat(session, oracle, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 33333
    rng = np.random.default_rng(m + 31 * k)
    V = rng.uniform(-1, 1, (n, m))
    W0 = rng.uniform(-1, 1, (n, k))
    S = rng.uniform(-1, 1, (m, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W0)
    C = SdMat(m, k).set(S)
    for alpha, beta in ((1.0, 0.0), (0.5, -2.0)):
        Wh.set(W0)
        K.chk(K.phist_Dmvec_times_sdMat, alpha, Vh.h, C.h, beta, Wh.h)
        assert relerr(Wh.get(), oracle.mvsd(V, S, alpha=alpha, beta=beta, W=W0)) < TOL
    for o in (Vh, Wh, C, mp):
        o.delete()


@pytest.mark.parametrize("m,k", [(1, 1), (4, 4), (8, 5), (20, 20), (40, 20), (32, 32), (64, 64), (7, 3)])
def test_mvec_times_sdMat_inplace(session, oracle, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 20011
    rng = np.random.default_rng(2)
    V = rng.uniform(-1, 1, (n, m))
    M = rng.uniform(-1, 1, (m, k))
    mp, Vh = _mk(n, m, V)
    C = SdMat(m, k).set(M)
    K.chk(K.phist_Dmvec_times_sdMat_inplace, Vh.h, C.h)
    out = Vh.get()
    ref = oracle.mvsdi(V, M)
    assert relerr(out, ref) < TOL
    assert np.array_equal(out[:, k:], V[:, k:])
    for o in (Vh, C, mp):
        o.delete()


@pytest.mark.parametrize("m,k", [(1, 1), (4, 4), (8, 4), (40, 4), (16, 16), (32, 32)])
def test_VC_add_WD(session, oracle, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 12345
    rng = np.random.default_rng(3)
    V = rng.uniform(-1, 1, (n, m))
    W = rng.uniform(-1, 1, (n, k))
    Cm = rng.uniform(-1, 1, (m, k))
    Dm = rng.uniform(-1, 1, (k, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W)
    C = SdMat(m, k).set(Cm)
    D = SdMat(k, k).set(Dm)
    K.chk(K.phist_Dmvec_times_sdMat_add_mvec_times_sdMat, Vh.h, C.h, Wh.h, D.h)
    assert relerr(Wh.get(), oracle.mvsd_add_mvsd(V, Cm, W, Dm)) < TOL
    for o in (Vh, Wh, C, D, mp):
        o.delete()


@pytest.mark.parametrize("m,k", [(1, 1), (4, 4), (8, 8), (40, 4), (16, 16), (32, 32), (6, 9), (64, 64), (24, 40),
                                 (64, 8)])
def test_fused_mvsd_mvTmv(session, oracle, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 40009
    rng = np.random.default_rng(4)
    V = rng.uniform(-1, 1, (n, m))
    W = rng.uniform(-1, 1, (n, k))
    S = rng.uniform(-1, 1, (m, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W)
    C = SdMat(m, k).set(S)
    G = SdMat(k, k)
    K.chk(K.phist_Dfused_mvsd_mvTmv, 0.5, Vh.h, C.h, -1.0, Wh.h, G.h)
    Wr, Gr = oracle.fused_mvsd_mvTmv(V, S, W, alpha=0.5, beta=-1.0)
    assert relerr(Wh.get(), Wr) < TOL
    assert relerr(G.get(), Gr) < TOL
    for o in (Vh, Wh, C, G, mp):
        o.delete()


@pytest.mark.parametrize("mv,m,k", [(1, 1, 1), (4, 4, 4), (40, 8, 8), (8, 8, 5), (32, 32, 32), (20, 16, 16),
                                    (64, 64, 64), (12, 24, 24), (64, 16, 13)])
def test_fused_mvsdi_mvTmv(session, oracle, mv, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 30011
    rng = np.random.default_rng(5)
    V = rng.uniform(-1, 1, (n, mv))
    W = rng.uniform(-1, 1, (n, m))
    Cm = rng.uniform(-1, 1, (m, k))
    D0 = rng.uniform(-1, 1, (mv, k))
    mp, Vh = _mk(n, mv, V)
    _, Wh = _mk(n, m, W)
    C = SdMat(m, k).set(Cm)
    D = SdMat(mv, k).set(D0)
    K.chk(K.phist_Dfused_mvsdi_mvTmv, 2.0, Vh.h, Wh.h, C.h, 0.5, D.h)
    Wr, Dr = oracle.fused_mvsdi_mvTmv(V, W, Cm, alpha=2.0, beta=0.5, D=D0)
    out = Wh.get()
    assert relerr(out[:, :k], Wr) < TOL
    assert relerr(D.get(), Dr) < TOL
    for o in (Vh, Wh, C, D, mp):
        o.delete()


@pytest.mark.parametrize("nvec", [1, 2, 3, 4, 8, 13, 32, 64, 70])
def test_blas1(session, oracle, nvec):
    from phist_b200 import kernels as K
    n = 100003
    rng = np.random.default_rng(nvec)
    X = rng.uniform(-1, 1, (n, nvec))
    Y = rng.uniform(-1, 1, (n, nvec))
    mp, Xh = _mk(n, nvec, X)
    _, Yh = _mk(n, nvec, Y)
    d = np.zeros(nvec)
    K.chk(K.phist_Dmvec_dot_mvec, Xh.h, Yh.h, K.sptr(d, np.float64))
    assert relerr(d, oracle.dot(X, Y)) < TOL
    K.chk(K.phist_Dmvec_norm2, Xh.h, K.sptr(d, np.float64))
    assert relerr(d, np.sqrt((X * X).sum(0))) < TOL
    K.chk(K.phist_Dmvec_add_mvec, 0.5, Xh.h, -2.0, Yh.h)
    Y1 = 0.5 * X - 2.0 * Y
    assert relerr(Yh.get(), Y1) < TOL
    a = rng.uniform(-1, 1, nvec)
    K.chk(K.phist_Dmvec_vadd_mvec, K.sptr(a, np.float64), Xh.h, 1.0, Yh.h)
    Y2 = a * X + Y1
    assert relerr(Yh.get(), Y2) < TOL
    K.chk(K.phist_Dmvec_vscale, Yh.h, K.sptr(a, np.float64))
    Y3 = Y2 * a
    assert relerr(Yh.get(), Y3) < TOL
    K.chk(K.phist_Dmvec_scale, Yh.h, 3.0)
    assert relerr(Yh.get(), 3.0 * Y3) < TOL
    K.chk(K.phist_Dmvec_normalize, Yh.h, K.sptr(d, np.float64))
    nrm = np.sqrt(((3.0 * Y3) ** 2).sum(0))
    assert relerr(d, nrm) < TOL
    assert np.allclose(np.linalg.norm(Yh.get(), axis=0), 1.0, atol=1e-13)
    K.chk(K.phist_Dmvec_put_value, Yh.h, 1.25)
    assert np.all(Yh.get() == 1.25)
    K.chk(K.phist_Dmvec_times_mvec_elemwise, 2.0, Xh.h, Yh.h)
    assert relerr(Yh.get(), 2.5 * X) < TOL
    # compensated dots (PHIST_ROBUST_REDUCTIONS)
    K.chk(K.phist_Dmvec_dot_mvec, Xh.h, Xh.h, K.sptr(d, np.float64), flags=K.PHIST_ROBUST_REDUCTIONS)
    assert relerr(d, oracle.dot(X, X, prec=True)) < 1e-15
    for o in (Xh, Yh, mp):
        o.delete()


def test_random_and_blocks(session):
    from phist_b200 import kernels as K
    from phist_b200.objects import Map, Mvec
    n = 10000
    m = Map(n)
    V = Mvec(m.h, 6)
    K.chk(K.phist_Dmvec_random, V.h)
    v = V.get()
    assert v.min() >= -1 and v.max() < 1 and abs(v.mean()) < 0.02
    B = Mvec(m.h, 3)
    K.chk(K.phist_Dmvec_get_block, V.h, B.h, 2, 4)
    assert np.array_equal(B.get(), v[:, 2:5])
    K.chk(K.phist_Dmvec_put_value, B.h, 7.0)
    K.chk(K.phist_Dmvec_set_block, V.h, B.h, 1, 3)
    w = V.get()
    assert np.all(w[:, 1:4] == 7.0) and np.array_equal(w[:, [0, 4, 5]], v[:, [0, 4, 5]])
    # host mirror protocol: extract_view + from_device / to_device
    import ctypes as ct
    p = ct.POINTER(ct.c_double)()
    lda = K.lidx()
    K.chk(K.phist_Dmvec_extract_view, V.h, ct.byref(p), ct.byref(lda))
    K.chk(K.phist_Dmvec_from_device, V.h)
    assert lda.value == 6 and p[5 * 6 + 2] == 7.0
    p[0] = 42.0
    K.chk(K.phist_Dmvec_to_device, V.h)
    assert V.get()[0, 0] == 42.0
    for o in (V, B, m):
        o.delete()


def test_sdmat_ops(session):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    rng = np.random.default_rng(1)
    a = rng.uniform(-1, 1, (5, 4))
    b = rng.uniform(-1, 1, (4, 3))
    c0 = rng.uniform(-1, 1, (5, 3))
    A, B, C = SdMat(5, 4).set(a), SdMat(4, 3).set(b), SdMat(5, 3).set(c0)
    K.chk(K.phist_DsdMat_times_sdMat, 2.0, A.h, B.h, 0.5, C.h)
    assert relerr(C.get(), 2.0 * a @ b + 0.5 * c0) < 1e-15
    D = SdMat(4, 3).set(b)
    E = SdMat(4, 4)
    K.chk(K.phist_DsdMatT_times_sdMat, 1.0, A.h, A.h, 0.0, E.h)
    assert relerr(E.get(), a.T @ a) < 1e-15
    K.chk(K.phist_DsdMat_times_sdMatT, 1.0, B.h, D.h, 0.0, E.h)
    assert relerr(E.get(), b @ b.T) < 1e-15
    K.chk(K.phist_DsdMat_add_sdMat, -1.0, B.h, 2.0, D.h)
    assert relerr(D.get(), b) < 1e-15
    K.chk(K.phist_DsdMat_identity, E.h)
    assert np.array_equal(E.get(), np.eye(4))
    for o in (A, B, C, D, E):
        o.delete()


def test_single_precision_block_kernels(session, oracle):
    """FP32 variants (mixed form) against the FP64 oracle, tolerance 1e-5"""
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 50000
    rng = np.random.default_rng(9)
    V = rng.uniform(-1, 1, (n, 8)).astype(np.float32)
    W = rng.uniform(-1, 1, (n, 8)).astype(np.float32)
    mp, Vh = _mk(n, 8, V, np.float32)
    _, Wh = _mk(n, 8, W, np.float32)
    C = SdMat(8, 8, np.float32)
    K.chk(K.phist_SmvecT_times_mvec, 1.0, Vh.h, Wh.h, 0.0, C.h)
    assert relerr(C.get(), V.astype(float).T @ W.astype(float)) < 1e-5
    d = np.zeros(8, np.float32)
    K.chk(K.phist_Smvec_dot_mvec, Vh.h, Wh.h, K.sptr(d, np.float32))
    assert relerr(d, (V.astype(float) * W).sum(0)) < 1e-5
    for o in (Vh, Wh, C, mp):
        o.delete()


@pytest.mark.parametrize("m,k", [(1, 1), (4, 4), (8, 8), (12, 12), (32, 32), (8, 5), (40, 24)])
@pytest.mark.parametrize("n", [30011, 2097152])
def test_fused_mvsdi_mvTmv_self(session, n, m, k):
    """V and W the same block, as PHIST's orthogrrB passes them
    (phist_orthogrr_def.hpp:291): W <- W C in place, then D = alpha W'W(:,:k) +
    beta D with W read after the update -- the builtin's self variants
    (gemm_kernels_fused_sCD.F90:516-543)"""
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    rng = np.random.default_rng(m * 7 + k)
    W = rng.uniform(-1, 1, (n, m))
    Cm = rng.uniform(-1, 1, (m, k))
    D0 = rng.uniform(-1, 1, (m, k))
    mp, Wh = _mk(n, m, W)
    C = SdMat(m, k).set(Cm)
    D = SdMat(m, k).set(D0)
    K.chk(K.phist_Dfused_mvsdi_mvTmv, 0.5, Wh.h, Wh.h, C.h, -1.0, D.h)
    new = W.copy()
    new[:, :k] = W @ Cm
    out = Wh.get()
    assert relerr(out, new) < TOL
    assert relerr(D.get(), 0.5 * new.T @ new[:, :k] - D0) < TOL
    for o in (Wh, C, D, mp):
        o.delete()
