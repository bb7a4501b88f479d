"""The numpy problem generators agree bit for bit with the library's row
functions (pure host code of the library, no GPU)."""
import ctypes as ct

import numpy as np
import pytest


@pytest.mark.parametrize("prob", ["LAPLACE3D-6", "LAPDIAG3D-7-S5", "ANDERSON3D-5-S1",
                                  "ANDERSON3D-3-S1-W4", "HONEYCOMB-4x3-S4", "HONEYCOMB-2-S4-W2",
                                  "ANDERSON3D-1-S0", "HONEYCOMB-1x1-S1"])
def test_rowfunc_matches_numpy(lib_built, prob):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    n = K.gidx()
    m = K.lidx()
    pr = K.phist_b200_problem_create(prob.encode(), 0, ct.byref(n), ct.byref(m))
    assert pr
    rp, c, v = G.problem(prob)
    assert len(rp) - 1 == n.value
    cols = np.zeros(16, np.int64)
    vals = np.zeros(16)
    ln = K.lidx()
    for i in range(n.value):
        assert K.phist_b200_problem_rowfunc(i, ct.byref(ln), K.ptr(cols), K.ptr(vals), pr) == 0
        L = ln.value
        assert L <= m.value
        assert np.array_equal(cols[:L], c[rp[i]:rp[i + 1]])
        assert np.array_equal(vals[:L], v[rp[i]:rp[i + 1]])
    ct.CDLL(None).free(ct.c_void_p(pr))


def test_unknown_problem_rejected(lib_built):
    from phist_b200 import kernels as K
    n = K.gidx()
    m = K.lidx()
    assert not K.phist_b200_problem_create(b"NOSUCH-5", 0, ct.byref(n), ct.byref(m))


def test_problem_sizes():
    from phist_b200 import generators as G
    rp, c, v = G.laplace3d(8)
    n = 8 ** 3
    assert len(rp) == n + 1 and rp[-1] == 7 * n - 6 * 8 * 8
    assert np.allclose(np.bincount(np.repeat(np.arange(n), np.diff(rp)), v), 0.0 + 6 - np.diff(rp) + 1)
    rp, c, v = G.anderson3d(6, 1)
    assert rp[-1] == 7 * 6 ** 3
    d = v[np.repeat(np.arange(6 ** 3), np.diff(rp)) == c]
    assert d.min() >= -8.25 and d.max() < 8.25
    rp, c, v = G.honeycomb(8, 8, 4)
    assert rp[-1] == 4 * 128
    # symmetric pattern
    A = np.zeros((128, 128))
    A[np.repeat(np.arange(128), np.diff(rp)), c] = v
    assert np.array_equal(A, A.T)


def test_unif_range():
    from phist_b200 import generators as G
    u = G.unif(3, np.arange(100000))
    assert u.min() >= -1 and u.max() < 1 and abs(u.mean()) < 0.01
