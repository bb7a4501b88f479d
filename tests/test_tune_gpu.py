"""SpMMV autotuner (phist_b200_{D,S}sparseMat_autotune, pb_tune.cu): it picks
the SELL chunk height C, the sorting window sigma and the kernel variant per
block width by timing the matrix itself.  Whatever it picks, Y = A X must not
change by a single bit (rows sum their entries in column order in every
layout; the permutation is internal), the fused SpMMV+dot must still match,
and the reported configuration must be one of the candidates."""
import ctypes as ct

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

WIDTHS = [1, 2, 3, 4, 8, 16, 32]
TPRS = {0: (1,), 1: (1,), 2: (1, 2), 3: (1, 2, 4), 4: (2, 4, 8), 5: (4, 8, 16)}


def _products(A, dtype):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, fn
    out = {}
    for w in WIDTHS:
        X = Mvec(A.domain_map, w, dtype=dtype)
        Y = Mvec(A.row_map, w, dtype=dtype)
        x = np.random.default_rng(w).uniform(-1, 1, (A.ncols, w))
        X.set(x)
        K.chk(fn(dtype, "sparseMat_times_mvec"), 1.0, A.h, X.h, 0.0, Y.h)
        out[w] = Y.get()
        X.delete()
        Y.delete()
    return out


def _tuning(A, dtype):
    from phist_b200 import kernels as K
    C, sig = ct.c_int(), ct.c_int64()
    tpr, unr, stg = (np.zeros(6, np.int32) for _ in range(3))
    f = K.phist_b200_DsparseMat_get_tuning if dtype == np.float64 else K.phist_b200_SsparseMat_get_tuning
    K.chk(f, A.h, ct.byref(C), ct.byref(sig), K.ptr(tpr), K.ptr(unr), K.ptr(stg))
    return C.value, sig.value, tpr, unr, stg


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("source", ["sprandn388", "LAPLACE3D-12", "ANDERSON3D-16-S1", "HONEYCOMB-16-S2-W1"])
def test_autotune_keeps_every_bit(session, testmats, source, dtype):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import SparseMat
    if source.startswith("sprandn"):
        rp, c, v, shape = testmats(source)
        A = SparseMat.from_crs(rp, c, v, ncols=shape[1], dtype=dtype)
    else:
        rp, c, v = G.problem(source)
        A = SparseMat.from_crs(rp, c, v, dtype=dtype)
    before = _products(A, dtype)
    widths = np.array([1, 4, 8, 32], np.int32)
    best = np.zeros(len(widths))
    f = K.phist_b200_DsparseMat_autotune if dtype == np.float64 else K.phist_b200_SsparseMat_autotune
    K.chk(f, A.h, len(widths), K.ptr(widths), 2, K.ptr(best))
    assert (best > 0).all() and np.isfinite(best).all()
    C, sig, tpr, unr, stg = _tuning(A, dtype)
    assert C in (8, 16, 32)
    assert sig in (1, 4 * C, 1024)
    lens = np.diff(rp)
    if (lens == lens[0]).all():
        assert sig == 1
    for lg in range(6):
        assert tpr[lg] in TPRS[lg], (lg, tpr)
        assert unr[lg] in (0, 1) and stg[lg] in (0, 1)
    after = _products(A, dtype)
    for w in WIDTHS:
        np.testing.assert_array_equal(before[w], after[w])
    A.delete()


def test_autotune_fused_dot_and_shift_paths(session, oracle):
    """the fused SpMMV + column dots and the shifted product on a retuned
    matrix against the oracle"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = G.problem("LAPDIAG3D-10-S2")
    A = SparseMat.from_crs(rp, c, v)
    widths = np.array([2, 8], np.int32)
    K.chk(K.phist_b200_DsparseMat_autotune, A.h, 2, K.ptr(widths), 2, None)
    n, w = A.nrows, 8
    x = np.random.default_rng(3).uniform(-1, 1, (n, w))
    X = Mvec(A.domain_map, w).set(x)
    Y = Mvec(A.row_map, w)
    sh = np.linspace(-1, 1, w)
    K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, 1.0, A.h, K.sptr(sh, np.float64), X.h, 0.0, Y.h)
    ref = oracle.spmmv(rp, c, v, x, shifts=sh)
    assert relerr(Y.get(), ref) < 1e-14
    wdw = np.zeros(w)
    K.chk(K.phist_Dfused_spmv_mvdot, 1.0, A.h, X.h, 0.0, Y.h, K.sptr(wdw, np.float64), None)
    y = oracle.spmmv(rp, c, v, x)
    assert relerr(Y.get(), y) < 1e-14
    assert relerr(wdw, (y * y).sum(axis=0)) < 1e-13
    for o in (X, Y, A):
        o.delete()


def test_autotune_rejects_bad_widths(session):
    from phist_b200 import kernels as K
    from phist_b200.objects import SparseMat
    A = SparseMat.from_problem("LAPLACE3D-6")
    for bad in ([0], [33], []):
        wd = np.array(bad or [1], np.int32)
        assert K.iflag_of(K.phist_b200_DsparseMat_autotune, A.h, len(bad), K.ptr(wd), 1, None) < 0
    A.delete()
