"""Parity at the benchmarked sizes: the 3D Anderson model with L=128
(n = 2,097,152, nnz = 14,680,064, on-site U[-8.25,8.25] seed 1).

* SpMMV on the full matrix in SELL-32-256 and SELL-32-1, block widths
  1..32, against the oracle at 1e-13 relative (the launch shapes, chunk
  counts and grids here are the ones bench.py times, which the small test
  matrices do not reach);
* the block products at n = 2,097,152 with m, k in {4, 8, 16, 32, 64}
  (one-wave TMA/DMMA grids and the GPU-wide second reduction pass);
* PHIST's own orthogonalisation routines (orthog, chol_QR, svqb from
  src/core, compiled unchanged against this library) on an n x 32 block of
  uniform[-1,1] entries from seed 2, with the checks of PHIST's
  test/core/OrthogTest_def.hpp and SVQB_Test_def.hpp: Q'Q = I and
  Q R1 = W - V R2 to 10 x releps (releps = largest column norm x eps,
  test/kernels/KernelTestWithVectors_def.h:447-461), plus rank-deficient
  inputs whose nullspace dimension must be reported.
"""
import ctypes as ct
import os

import numpy as np
import pytest

from conftest import ROOT, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13
L = 128
N = L ** 3
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def anderson(session, oracle):
    from phist_b200 import generators as G
    oracle.set_threads(os.cpu_count() or 1)
    return G.anderson3d(L, 1)


@pytest.mark.parametrize("sigma", [256, 1])
def test_spmmv_anderson_L128(session, oracle, anderson, sigma):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = anderson
    K.chk(K.phist_b200_set_sell_params, 32, sigma)
    try:
        A = SparseMat.from_problem("ANDERSON3D-%d-S1" % L,
                                   flags=K.PHIST_SPARSEMAT_PERM_LOCAL if sigma > 1 else 0)
    finally:
        K.chk(K.phist_b200_set_sell_params, 32, 256)
    assert A.nrows == N and A.nnz == 7 * N
    for nvec in (1, 2, 4, 8, 16, 32):
        x = G.random_block(N, nvec, 3)
        X = Mvec(A.domain_map, nvec).set(x)
        Y = Mvec(A.row_map, nvec)
        K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        ref = oracle.spmmv(rp, c, v, x)
        err = relerr(Y.get(), ref)
        assert err < TOL, (nvec, err)
        if nvec in (4, 32):
            # shifted, beta != 0 (jadaOp's apply_shifted at full size)
            y0 = G.random_block(N, nvec, 4)
            sh = np.linspace(-2.0, 2.0, nvec)
            Y.set(y0)
            K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, -0.5, A.h, K.sptr(sh, np.float64), X.h, 1.5, Y.h)
            ref = oracle.spmmv(rp, c, v, x, alpha=-0.5, beta=1.5, y=y0, shifts=sh)
            assert relerr(Y.get(), ref) < TOL, nvec
        X.delete()
        Y.delete()
    A.delete()


WIDTHS = [(4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (4, 64), (64, 4), (8, 32), (32, 16)]


@pytest.fixture(scope="module")
def blocks(session):
    """n x 64 blocks V, W (uniform[-1,1), seeds 2 and 3) resident once"""
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec
    mp = Map(N)
    V = random_block(N, 64, 2)
    W = random_block(N, 64, 3)
    Vh = Mvec(mp.h, 64).set(V)
    Wh = Mvec(mp.h, 64).set(W)
    yield mp, V, W, Vh, Wh
    Vh.delete()
    Wh.delete()
    mp.delete()


@pytest.mark.parametrize("m,k", WIDTHS)
def test_block_products_n2M(session, oracle, blocks, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SdMat
    mp, V, W, Vh, Wh = blocks
    rng = np.random.default_rng(m * 1000 + k)
    Vv = Vh.view(0, m - 1)  # strided views of the n x 64 roots (lda = 64)
    Wv = Wh.view(0, k - 1)
    Vm = np.ascontiguousarray(V[:, :m])
    Wm = np.ascontiguousarray(W[:, :k])
    # mvecT_times_mvec on the views and on contiguous copies
    C0 = rng.uniform(-1, 1, (m, k))
    C = SdMat(m, k).set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vv.h, Wv.h, 2.0, C.h)
    ref = oracle.mvTmv(Vm, Wm, alpha=0.5, beta=2.0, C=C0)
    assert relerr(C.get(), ref) < TOL
    Vc = Mvec(mp.h, m).set(Vm)
    Wc = Mvec(mp.h, k).set(Wm)
    C.set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vc.h, Wc.h, 2.0, C.h)
    assert relerr(C.get(), ref) < TOL
    # mvec_times_sdMat, W = alpha V S + beta W
    S = rng.uniform(-1, 1, (m, k))
    Sm = SdMat(m, k).set(S)
    K.chk(K.phist_Dmvec_times_sdMat, -1.0, Vc.h, Sm.h, 0.5, Wc.h)
    Wref = oracle.mvsd(Vm, S, alpha=-1.0, beta=0.5, W=Wm)
    assert relerr(Wc.get(), Wref) < TOL
    # fused W = V S (beta 0) with W'W in the same pass
    G = SdMat(k, k)
    K.chk(K.phist_Dfused_mvsd_mvTmv, 1.0, Vc.h, Sm.h, 0.0, Wc.h, G.h)
    Wr, Gr = oracle.fused_mvsd_mvTmv(Vm, S, Wm, alpha=1.0, beta=0.0)
    assert relerr(Wc.get(), Wr) < TOL
    assert relerr(G.get(), Gr) < TOL
    if k <= m:
        # in place, V(:, :k) <- V M, and the fused in-place product with V'W
        M = rng.uniform(-1, 1, (m, k))
        Mm = SdMat(m, k).set(M)
        Vc.set(Vm)
        K.chk(K.phist_Dmvec_times_sdMat_inplace, Vc.h, Mm.h)
        out = Vc.get()
        assert relerr(out[:, :k], oracle.mvsdi(Vm, M)[:, :k]) < TOL
        Xh = Mvec(mp.h, 16).set(np.ascontiguousarray(W[:, 48:64]))
        D0 = rng.uniform(-1, 1, (16, k))
        D = SdMat(16, k).set(D0)
        Vc.set(Vm)
        K.chk(K.phist_Dfused_mvsdi_mvTmv, 2.0, Xh.h, Vc.h, Mm.h, -0.5, D.h)
        Wr2, Dr = oracle.fused_mvsdi_mvTmv(np.ascontiguousarray(W[:, 48:64]), Vm, M, alpha=2.0, beta=-0.5, D=D0)
        assert relerr(Vc.get()[:, :k], Wr2) < TOL
        assert relerr(D.get(), Dr) < TOL
        for o in (Mm, Xh, D):
            o.delete()
    for o in (Vv, Wv, Vc, Wc, C, Sm, G):
        o.delete()


# ------------------------------------------------------------------ orthog
_core = None


def core():
    """PHIST's solver layers (src/core etc.), compiled unchanged against this
    library (phist_b200/solvers/Makefile)"""
    global _core
    if _core is None:
        path = os.path.join(ROOT, "phist_b200", "lib", "libphist_solvers.so")
        if not os.path.exists(path):
            pytest.skip("PHIST solver layers not built")
        lib = ct.CDLL(path)
        vp, ip = ct.c_void_p, ct.POINTER(ct.c_int)
        lib.phist_Dorthog.argtypes = [vp, vp, vp, vp, vp, ct.c_int, ip, ip]
        lib.phist_Dchol_QR.argtypes = [vp, vp, ip]
        lib.phist_Dsvqb.argtypes = [vp, vp, ct.POINTER(ct.c_double), ip]
        _core = lib
    return _core


def _orth_err(Q):
    k = Q.shape[1]
    return np.abs(Q.T @ Q - np.eye(k)).max()


def _releps(A):
    return np.linalg.norm(A, axis=0).max() * EPS


@pytest.mark.parametrize("n", [N, 10007])
def test_chol_qr_svqb_n_by_32(session, n):
    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec, SdMat
    lib = core()
    mp = Map(n)
    W0 = random_block(n, 32, 2)
    tol = 10 * _releps(W0)
    # CholQR: Q R = W, Q'Q = I
    Wh = Mvec(mp.h, 32).set(W0)
    R = SdMat(32, 32)
    K.chk(lib.phist_Dchol_QR, Wh.h, R.h)
    Q = Wh.get()
    assert _orth_err(Q) < tol
    assert np.abs(Q @ R.get() - W0).max() < tol
    # SVQB: Q = W B, Q'Q = I, e = column norms of W
    Wh.set(W0)
    B = SdMat(32, 32)
    e = np.zeros(32)
    K.chk(lib.phist_Dsvqb, Wh.h, B.h, K.sptr(e, np.float64))
    Q = Wh.get()
    assert _orth_err(Q) < tol
    assert np.abs(Q - W0 @ B.get()).max() < tol * np.abs(B.get()).max() * 32
    assert np.allclose(e, np.linalg.norm(W0, axis=0), rtol=100 * EPS)
    for o in (Wh, R, B, mp):
        o.delete()


@pytest.mark.parametrize("n", [N, 10007])
def test_orthog_against_basis(session, n):
    """orthog(V, W): Q R1 = W - V R2, Q'Q = I, V'Q = 0 (OrthogTest_def.hpp),
    V an orthonormal n x 8 basis, W the n x 32 seed-2 block"""
    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec, SdMat
    lib = core()
    mp = Map(n)
    V0, _ = np.linalg.qr(random_block(n, 8, 7))
    W0 = random_block(n, 32, 2)
    Vh = Mvec(mp.h, 8).set(V0)
    Wh = Mvec(mp.h, 32).set(W0)
    R1, R2 = SdMat(32, 32), SdMat(8, 32)
    rank = ct.c_int(0)
    flag = K.iflag_of(lib.phist_Dorthog, Vh.h, Wh.h, None, R1.h, R2.h, 3, ct.byref(rank))
    assert flag == 0, flag
    assert rank.value == 40
    Q = Wh.get()
    tol = 10 * _releps(W0)
    assert _orth_err(Q) < tol
    assert np.abs(V0.T @ Q).max() < 10 * _releps(V0)
    assert np.abs(Q @ R1.get() + V0 @ R2.get() - W0).max() < tol
    for o in (Vh, Wh, R1, R2, mp):
        o.delete()


def test_rank_deficient_blocks(session):
    """a block with two copies of one column: chol_QR reports a nullspace of
    dimension 1 (iflag = m - r = 1) and fills it with a random column
    orthogonalised against the rest (phist_chol_QR_def.hpp:70-115), so Q is
    orthonormal and Q R = W still holds; svqb reports m - r = 1, zeroes one
    column and leaves the others orthonormal (phist_svqb_decl.h:18-29; which
    column is zeroed follows the eigenvalue order of PHIST's qb step)"""
    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec, SdMat
    lib = core()
    n = 20011
    mp = Map(n)
    W0 = random_block(n, 8, 9)
    W0[:, 5] = W0[:, 2]
    Wh = Mvec(mp.h, 8).set(W0)
    R = SdMat(8, 8)
    assert K.iflag_of(lib.phist_Dchol_QR, Wh.h, R.h) == 1
    Q = Wh.get()
    assert _orth_err(Q) < 10 * _releps(W0)
    assert np.abs(Q @ R.get() - W0).max() < 10 * _releps(W0)
    Wh.set(W0)
    B = SdMat(8, 8)
    e = np.zeros(8)
    assert K.iflag_of(lib.phist_Dsvqb, Wh.h, B.h, K.sptr(e, np.float64)) == 1
    Q = Wh.get()
    nrm = np.linalg.norm(Q, axis=0)
    null = nrm < 1e-8
    assert null.sum() == 1, nrm          # one column spans the nullspace: zero
    assert _orth_err(Q[:, ~null]) < 10 * _releps(W0)
    for o in (Wh, R, B, mp):
        o.delete()
