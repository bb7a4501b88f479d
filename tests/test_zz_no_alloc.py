"""phist_b200_DmvecT_times_mvec_noalloc: the allocation-free variant of
mvecT_times_mvec, for callers that cannot allocate device memory (a host that
owns the whole device-memory budget after start-up).  Called through the C
ABI on raw device pointers; its result must equal that of the regular entry
point phist_DmvecT_times_mvec within the FP64 tolerance of the other
block-product tests (1e-13 relative), on two calls in a row (the second call
reuses the shared scratch array the first one left behind).

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as ct

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _dev(mv):
    from phist_b200 import kernels as K
    p = ct.POINTER(ct.c_double)()
    lda = K.lidx()
    K.chk(K.phist_b200_Dmvec_device_view, mv.h, ct.byref(p), ct.byref(lda))
    return ct.cast(p, ct.c_void_p), lda.value


def test_noalloc_matches_regular_entry_point(session):
    import torch

    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, Mvec, SdMat
    n = 300007
    mp = Map(n)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row, different shapes and alpha/beta
    for (m, k, alpha, beta, seed) in ((8, 5, 1.0, 0.0, 1), (64, 64, 0.5, 2.0, 2)):
        V = Mvec(mp.h, m).set(random_block(n, m, seed))
        W = Mvec(mp.h, k).set(random_block(n, k, seed + 10))
        C0 = random_block(m, k, seed + 20)
        Cref = SdMat(m, k).set(C0)
        K.chk(K.phist_DmvecT_times_mvec, alpha, V.h, W.h, beta, Cref.h)
        ref = Cref.get()
        # column-major m x k output in caller-owned device memory
        Cd = torch.from_numpy(np.asfortranarray(C0).T.copy()).to("cuda")  # (k, m) == col-major (m, k)
        vp, ldv = _dev(V)
        wp, ldw = _dev(W)
        K.chk(K.phist_b200_DmvecT_times_mvec_noalloc, n, m, k, alpha, vp, ldv, wp, ldw, beta,
              ct.c_void_p(Cd.data_ptr()), m, stream)
        torch.cuda.synchronize()
        got = Cd.cpu().numpy().T
        assert relerr(got, ref) < TOL, (m, k)
        for o in (V, W, Cref):
            o.delete()
    mp.delete()


def test_noalloc_rejects_oversize(session):
    import os

    from phist_b200 import kernels as K
    os.environ["PHIST_B200_QUIET"] = "1"
    dummy = ct.c_void_p(1)
    assert K.iflag_of(K.phist_b200_DmvecT_times_mvec_noalloc, 10, 65, 4, 1.0, dummy, 65, dummy, 4,
                      0.0, dummy, 65, None) == K.PHIST_INVALID_INPUT
    assert K.iflag_of(K.phist_b200_DmvecT_times_mvec_noalloc, 10, 4, 4, 1.0, dummy, 3, dummy, 4,
                      0.0, dummy, 4, None) == K.PHIST_INVALID_INPUT
    del os.environ["PHIST_B200_QUIET"]
