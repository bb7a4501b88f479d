"""phist_b200_DmvecT_times_mvec_noalloc: the allocation-free variant of
mvecT_times_mvec, for callers that cannot allocate device memory (a host that
owns the whole device-memory budget after start-up).  Called through the C
ABI on raw device pointers; its result must equal that of the regular entry
point phist_DmvecT_times_mvec within the FP64 tolerance of the other
block-product tests (1e-13 relative), on two calls in a row (the second call
reuses the shared scratch array the first one left behind).

The cases cover contiguous and strided operands (V and W as column views of
wider blocks, C with a leading dimension above m whose extra rows must stay
untouched), n = 0 (C = beta*C), and widths on both sides of the m*k = 256
switch between the two micro-tile shapes.

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


def _block(mp, n, w, pad, seed):
    """an n x w block, as a view of columns 1..w of an n x (w + pad) block
    when pad > 0 (leading dimension above w); returns (root, block)"""
    from phist_b200.generators import random_block
    from phist_b200.objects import Mvec
    root = Mvec(mp.h, w + pad).set(random_block(n, w + pad, seed))
    if pad == 0:
        return root, root
    return root, root.view(1, w)


def _noalloc(n, m, k, alpha, V, W, beta, C0, ldc):
    """runs the allocation-free entry point with C (m x k, column-major,
    leading dimension ldc) in caller-owned device memory; returns the full
    ldc x k array afterwards"""
    import torch

    from phist_b200 import kernels as K
    buf = np.full((ldc, k), 7.25)  # rows m..ldc-1 are guards
    buf[:m, :] = C0
    Cd = torch.from_numpy(np.asfortranarray(buf).T.copy()).to("cuda")  # (k, ldc) == col-major (ldc, k)
    vp, ldv = _dev(V) if V is not None else (ct.c_void_p(0), m)
    wp, ldw = _dev(W) if W is not None else (ct.c_void_p(0), k)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    K.chk(K.phist_b200_DmvecT_times_mvec_noalloc, n, m, k, alpha, vp, ldv, wp, ldw, beta,
          ct.c_void_p(Cd.data_ptr()), ldc, stream)
    torch.cuda.synchronize()
    return Cd.cpu().numpy().T


CASES = [
    # n, m, k, alpha, beta, pad_v, pad_w, ldc_extra
    (300007, 8, 5, 1.0, 0.0, 0, 0, 0),
    (300007, 64, 64, 0.5, 2.0, 0, 0, 0),
    (100003, 1, 64, 1.0, 0.0, 0, 0, 0),     # m*k = 64: small micro-tiles
    (100003, 64, 3, -1.0, 1.0, 3, 0, 2),    # 192, strided V, ldc > m
    (100003, 15, 17, 1.0, 0.5, 0, 2, 3),    # 255: small tiles, strided W
    (100003, 16, 16, 2.0, 0.0, 1, 1, 1),    # 256: large tiles, both strided
    (100003, 17, 16, 1.0, -1.0, 2, 3, 4),   # 272
]


@pytest.mark.parametrize("n,m,k,alpha,beta,pv,pw,lx", CASES)
def test_noalloc_matches_regular_entry_point(session, n, m, k, alpha, beta, pv, pw, lx):
    from phist_b200 import kernels as K
    from phist_b200.generators import random_block
    from phist_b200.objects import Map, SdMat
    mp = Map(n)
    Vr, V = _block(mp, n, m, pv, 1 + m)
    Wr, W = _block(mp, n, k, pw, 11 + k)
    C0 = random_block(m, k, 21)
    Cref = SdMat(m, k).set(C0)
    K.chk(K.phist_DmvecT_times_mvec, alpha, V.h, W.h, beta, Cref.h)
    ref = Cref.get()
    # two calls in a row on the same inputs: the second starts from the
    # scratch contents the first one left
    for _ in range(2):
        out = _noalloc(n, m, k, alpha, V, W, beta, C0, m + lx)
        assert relerr(out[:m, :], ref) < TOL, (m, k)
        assert np.all(out[m:, :] == 7.25), "rows past m of C were written"
    for o in {id(x): x for x in (V, Vr, W, Wr, Cref)}.values():
        o.delete()
    mp.delete()


def test_noalloc_empty_rows(session):
    """n = 0: no rows to sum, C = beta*C exactly (PHIST's mvecT_times_mvec on
    an empty local block)"""
    from phist_b200.generators import random_block
    C0 = random_block(4, 6, 5)
    for beta in (0.0, -0.5):
        out = _noalloc(0, 4, 6, 1.0, None, None, beta, C0, 5)
        assert np.array_equal(out[:4, :], beta * C0)
        assert np.all(out[4:, :] == 7.25)


def test_noalloc_rejects_oversize(session, monkeypatch):
    from phist_b200 import kernels as K
    monkeypatch.setenv("PHIST_B200_QUIET", "1")
    dummy = ct.c_void_p(1)
    assert K.iflag_of(K.phist_b200_DmvecT_times_mvec_noalloc, 10, 65, 4, 1.0, dummy, 65, dummy, 4,
                      0.0, dummy, 65, None) == K.PHIST_INVALID_INPUT
    assert K.iflag_of(K.phist_b200_DmvecT_times_mvec_noalloc, 10, 4, 4, 1.0, dummy, 3, dummy, 4,
                      0.0, dummy, 4, None) == K.PHIST_INVALID_INPUT
