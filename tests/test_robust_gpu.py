"""Compensated Gram products for PHIST_ROBUST_REDUCTIONS on the GPU.

mvecT_times_mvec, fused_mvsd_mvTmv and fused_mvsdi_mvTmv with the flag set
form their sums in double-double (Dot2), as PHIST's builtin does through
gemm_kernels_sC_prec.c when orthogrrB passes the flag
(phist_orthogrr_def.hpp:89,152,167).  The results are compared with the
oracle's compensated restatement (itself pinned against PHIST's
dgemm_sc_prec_<m>_k in tests/test_oracle.py) within the Dot2 error bound of
two differently ordered compensated sums: 8 eps |C| + 4 n eps^2 sum|v||w|.
On ill-conditioned columns (large cancelling terms) plain FP64 is far off
and the compensated products are not.
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def _bound(V, W, ref, C0=None, beta=0.0):
    n = V.shape[0]
    b = 8 * EPS * np.abs(ref) + 4 * n * EPS ** 2 * (np.abs(V).T @ np.abs(W))
    if C0 is not None:
        b += 4 * EPS * np.abs(beta * C0)
    return b


def _mk(n, ncol, data):
    from phist_b200.objects import Map, Mvec
    m = Map(n)
    return m, Mvec(m.h, ncol).set(data)


def _illcond(rng, n, m):
    return rng.uniform(-1, 1, (n, m)) * np.exp(rng.uniform(-18, 18, (n, m)))


@pytest.mark.parametrize("m,k", [(1, 1), (2, 3), (4, 4), (5, 7), (8, 8), (16, 16), (32, 32), (64, 64),
                                 (13, 29), (40, 56), (70, 3), (3, 130)])
@pytest.mark.parametrize("n", [1000, 100003])
def test_robust_mvecT_times_mvec(session, oracle, n, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    rng = np.random.default_rng(m * 131 + k)
    V = _illcond(rng, n, m)
    W = rng.uniform(-1, 1, (n, k))
    C0 = rng.uniform(-1, 1, (m, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W)
    C = SdMat(m, k).set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vh.h, Wh.h, 2.0, C.h, flags=K.PHIST_ROBUST_REDUCTIONS)
    got = C.get()
    ref = oracle.mvTmv(V, W, alpha=0.5, beta=2.0, C=C0, prec=True)
    assert np.all(np.abs(got - ref) <= _bound(0.5 * V, W, ref, C0, 2.0))
    # bitwise reproducible
    C.set(C0)
    K.chk(K.phist_DmvecT_times_mvec, 0.5, Vh.h, Wh.h, 2.0, C.h, flags=K.PHIST_ROBUST_REDUCTIONS)
    assert np.array_equal(C.get(), got)
    for o in (Vh, Wh, C, mp):
        o.delete()


def test_robust_beats_plain_on_cancellation(session, oracle):
    """columns built to cancel: u.v - u.v + 1e-9 u.w; the exact dot of the
    stored values comes from Python integers (every double is an integer
    multiple of 2^-1074)"""
    from fractions import Fraction

    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    rng = np.random.default_rng(11)
    h = 2000
    u = rng.uniform(-1, 1, h) * 1e6
    v = rng.uniform(-1, 1, h)
    w = rng.uniform(-1, 1, h)
    x = np.concatenate([u, u])[:, None]
    y = np.concatenate([v, -v + 1e-9 * w])[:, None]
    exact = float(sum(Fraction(a) * Fraction(b) for a, b in zip(x[:, 0], y[:, 0])))
    mp, Xh = _mk(2 * h, 1, x)
    _, Yh = _mk(2 * h, 1, y)
    C = SdMat(1, 1)
    K.chk(K.phist_DmvecT_times_mvec, 1.0, Xh.h, Yh.h, 0.0, C.h, flags=K.PHIST_ROBUST_REDUCTIONS)
    robust = C.get()[0, 0]
    K.chk(K.phist_DmvecT_times_mvec, 1.0, Xh.h, Yh.h, 0.0, C.h)
    plain = C.get()[0, 0]
    assert abs(robust - exact) <= 4 * EPS * abs(exact)
    assert abs(plain - exact) > 1e3 * abs(robust - exact) + 1e-30
    for o in (Xh, Yh, C, mp):
        o.delete()


@pytest.mark.parametrize("m,k", [(4, 4), (8, 8), (16, 5), (32, 32), (64, 64)])
def test_robust_fused_mvsd_mvTmv(session, oracle, m, k):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 50021
    rng = np.random.default_rng(7 * m + k)
    V = rng.uniform(-1, 1, (n, m))
    W0 = rng.uniform(-1, 1, (n, k))
    S = rng.uniform(-1, 1, (m, k))
    mp, Vh = _mk(n, m, V)
    _, Wh = _mk(n, k, W0)
    C = SdMat(m, k).set(S)
    G = SdMat(k, k)
    K.chk(K.phist_Dfused_mvsd_mvTmv, 0.5, Vh.h, C.h, -1.0, Wh.h, G.h, flags=K.PHIST_ROBUST_REDUCTIONS)
    Wn = Wh.get()
    assert relerr(Wn, oracle.mvsd(V, S, alpha=0.5, beta=-1.0, W=W0)) < 1e-13
    ref = oracle.mvTmv(Wn, Wn, prec=True)
    assert np.all(np.abs(G.get() - ref) <= _bound(Wn, Wn, ref))
    for o in (Vh, Wh, C, G, mp):
        o.delete()


@pytest.mark.parametrize("mv,m,k", [(4, 4, 4), (8, 8, 5), (16, 32, 32), (64, 64, 64), (3, 12, 12)])
@pytest.mark.parametrize("alias", [False, True])
def test_robust_fused_mvsdi_mvTmv(session, oracle, mv, m, k, alias):
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    n = 40009
    rng = np.random.default_rng(mv + 3 * m + 5 * k)
    W0 = rng.uniform(-1, 1, (n, m))
    Cm = rng.uniform(-1, 1, (m, k))
    mp, Wh = _mk(n, m, W0)
    if alias:
        Vh, V, mv = Wh, None, m
    else:
        V = rng.uniform(-1, 1, (n, mv))
        _, Vh = _mk(n, mv, V)
    D0 = rng.uniform(-1, 1, (mv, k))
    C = SdMat(m, k).set(Cm)
    D = SdMat(mv, k).set(D0)
    K.chk(K.phist_Dfused_mvsdi_mvTmv, 2.0, Vh.h, Wh.h, C.h, 0.5, D.h, flags=K.PHIST_ROBUST_REDUCTIONS)
    Wn = Wh.get()
    assert relerr(Wn[:, :k], W0 @ Cm) < 1e-13
    Vn = Wn if alias else V
    ref = oracle.mvTmv(Vn, np.ascontiguousarray(Wn[:, :k]), alpha=2.0, beta=0.5, C=D0, prec=True)
    assert np.all(np.abs(D.get() - ref) <= _bound(2.0 * Vn, Wn[:, :k], ref, D0, 0.5))
    objs = (Wh, C, D, mp) if alias else (Wh, Vh, C, D, mp)
    for o in objs:
        o.delete()


def test_robust_orthog_n2M(session):
    """PHIST's orthog with PHIST_ROBUST_REDUCTIONS on the n x 32 seed-2 block
    against an orthonormal n x 8 basis (n = 2,097,152): every Gram product
    of orthogrrB runs compensated; the decomposition must hold as in
    test/core/OrthogTest_def.hpp"""
    import os

    from conftest import ROOT
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec
    from phist_b200 import kernels as K
    from phist_b200.objects import SdMat
    path = os.path.join(ROOT, "phist_b200", "lib", "libphist_solvers.so")
    if not os.path.exists(path):
        pytest.skip("PHIST solver layers not built")
    lib = ct.CDLL(path)
    vp, ip = ct.c_void_p, ct.POINTER(ct.c_int)
    lib.phist_Dorthog.argtypes = [vp, vp, vp, vp, vp, ct.c_int, ip, ip]
    n = 1 << 21
    mp = Map(n)
    V0, _ = np.linalg.qr(random_block(n, 8, 7))
    W0 = random_block(n, 32, 2)
    Vh = Mvec(mp.h, 8).set(V0)
    Wh = Mvec(mp.h, 32).set(W0)
    R1, R2 = SdMat(32, 32), SdMat(8, 32)
    rank = ct.c_int(0)
    flag = K.iflag_of(lib.phist_Dorthog, Vh.h, Wh.h, None, R1.h, R2.h, 4, ct.byref(rank),
                      flags=K.PHIST_ROBUST_REDUCTIONS)
    assert flag == 0, flag
    assert rank.value == 40
    Q = Wh.get()
    tol = 10 * np.linalg.norm(W0, axis=0).max() * EPS
    assert np.abs(Q.T @ Q - np.eye(32)).max() < tol
    assert np.abs(V0.T @ Q).max() < 10 * EPS * np.sqrt(n)
    assert np.abs(Q @ R1.get() + V0 @ R2.get() - W0).max() < tol
    for o in (Vh, Wh, R1, R2, mp):
        o.delete()
