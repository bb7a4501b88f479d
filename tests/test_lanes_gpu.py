"""Per-thread lanes: host threads that drive the library concurrently get
their own CUDA streams and device scratch.  The same computation gives
bitwise identical results run alone and run in the mix with others, and the
lanes are really distinct (the library reports more than one)."""
import ctypes as ct
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _work(seed, out, problem="ANDERSON3D-16-S1", nvec=4, steps=40):
    """power-iteration-like chain of library calls; returns the final block,
    the column norms of every step and the last Gram matrix"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SdMat, SparseMat
    A = SparseMat.from_problem(problem)
    n = A.nrows
    X = Mvec(A.domain_map, nvec).set(G.random_block(n, nvec, seed))
    Y = Mvec(A.row_map, nvec)
    C = SdMat(nvec, nvec)
    norms = []
    for _ in range(steps):
        K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        nrm = np.zeros(nvec)
        K.chk(K.phist_Dmvec_normalize, Y.h, K.sptr(nrm, np.float64))
        norms.append(nrm.copy())
        K.chk(K.phist_DmvecT_times_mvec, 1.0, Y.h, Y.h, 0.0, C.h)
        X, Y = Y, X
    out[seed] = (X.get(), np.array(norms), C.get())
    for o in (X, Y, C, A):
        o.delete()


def test_results_identical_alone_and_concurrent(session):
    from phist_b200 import kernels as K
    seeds = [3, 4, 5, 6]
    alone = {}
    for sd in seeds:
        _work(sd, alone)
    mixed = {}
    ts = [threading.Thread(target=_work, args=(sd, mixed)) for sd in seeds]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for sd in seeds:
        for a, b in zip(alone[sd], mixed[sd]):
            assert np.array_equal(a, b), sd
    nl = ct.c_int()
    K.chk(K.phist_b200_lane_count, ct.byref(nl))
    assert nl.value >= 2
