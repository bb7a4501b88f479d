"""Failure path of the bounded device waits.

The TMA-fed kernels wait on mbarriers with a limit of about one second of
wall time (pb_tma.cuh mbar_wait); when a copy never lands they store an
error code in the device error word and return instead of hanging, and the
next synchronisation reports it.  phist_b200_selftest_bounded_wait runs a
kernel whose wait cannot complete (an mbarrier that nothing arrives on), so
the limit really runs out here: the call must come back after about a
second with PHIST_FUNCTIONAL_ERROR, the word must be cleared, and the
context must stay usable for ordinary work.  No GPU fault is involved.
"""
import time

import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_is_reported(session, oracle):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    t0 = time.perf_counter()
    f = K.iflag_of(K.phist_b200_selftest_bounded_wait)
    dt = time.perf_counter() - t0
    assert f == K.PHIST_FUNCTIONAL_ERROR
    assert 0.9 < dt < 60.0, dt
    # the error word was cleared: the next synchronisation is clean
    assert K.iflag_of(K.phist_b200_synchronize) == 0
    # the context still computes correctly
    rp, c, v = G.problem("LAPLACE3D-12")
    A = SparseMat.from_crs(rp, c, v)
    x = G.random_block(A.nrows, 4, 7)
    X = Mvec(A.domain_map, 4).set(x)
    Y = Mvec(A.row_map, 4)
    K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
    assert relerr(Y.get(), oracle.spmmv(rp, c, v, x)) < 1e-13
    # and a second run reports again (the path is repeatable)
    assert K.iflag_of(K.phist_b200_selftest_bounded_wait) == K.PHIST_FUNCTIONAL_ERROR
    assert K.iflag_of(K.phist_b200_synchronize) == 0
    for o in (X, Y, A):
        o.delete()
