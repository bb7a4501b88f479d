"""The resident-grid SpMMV kernel that prefetches the next tile's matrix
entries into shared memory (phist_b200_set_spmv_prefetch) against the
oracle and against the one-tile-per-block kernel.

Both run PHIST's row loop term for term (spmvm_kernels.F90:494-523), so the
results must be bitwise equal, and equal to the oracle at 1e-13.  Covered:
every block width class 1..32 with every threads-per-row choice, alpha/beta
and shift variants, sigma-sorted and unsorted layouts (rows of 4..7 entries
in the Dirichlet Laplacian), matrices whose chunk count is not a multiple of
the tile, and the 2D honeycomb lattice.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.fixture
def restore(session):
    from phist_b200 import kernels as K
    yield
    K.chk(K.phist_b200_set_spmv_prefetch, 1)
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    for nv, tpr in ((4, 1), (8, 2), (16, 4), (32, 8)):
        K.chk(K.phist_b200_set_spmv_config, nv, tpr, 1)


TPRS = {1: (1,), 2: (1,), 4: (1, 2), 8: (1, 2, 4), 16: (2, 4, 8), 32: (4, 8, 16)}


@pytest.mark.parametrize("prob,sigma", [("ANDERSON3D-26-S1", 256), ("LAPLACE3D-23", 256), ("LAPLACE3D-23", 1),
                                        ("HONEYCOMB-41x23-S4", 256)])
@pytest.mark.parametrize("nvec", [1, 2, 4, 8, 16, 32])
def test_prefetch_kernel_matches_oracle_and_one_tile_kernel(session, oracle, restore, prob, sigma, nvec):
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, sigma)
    rp, c, v = G.problem(prob)
    A = SparseMat.from_crs(rp, c, v, flags=K.PHIST_SPARSEMAT_PERM_LOCAL if sigma > 1 else 0)
    n = len(rp) - 1
    x = G.random_block(n, nvec, 31)
    y0 = G.random_block(n, nvec, 32)
    sh = np.linspace(-1.25, 1.25, nvec)
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec)
    for alpha, beta, s in ((1.0, 0.0, None), (-0.5, 2.0, None), (0.75, -0.5, sh)):
        ref = oracle.spmmv(rp, c, v, x, alpha=alpha, beta=beta, y=y0, shifts=s)
        for tpr in TPRS[nvec]:
            if nvec >= 4:
                K.chk(K.phist_b200_set_spmv_config, nvec, tpr, 1)
            outs = []
            for pf in (0, 1):
                K.chk(K.phist_b200_set_spmv_prefetch, pf)
                Y.set(y0)
                if s is None:
                    K.chk(K.phist_DsparseMat_times_mvec, alpha, A.h, X.h, beta, Y.h)
                else:
                    K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, alpha, A.h, K.sptr(s, np.float64), X.h, beta, Y.h)
                outs.append(Y.get())
            assert relerr(outs[1], ref) < TOL, (alpha, beta, tpr)
            assert np.array_equal(outs[0], outs[1]), (alpha, beta, tpr)
    X.delete()
    Y.delete()
    A.delete()


@pytest.mark.parametrize("nvec", [4, 32])
def test_prefetch_kernel_single_precision(session, oracle, restore, nvec):
    """FP32 (the mixed form's correction equations) against the FP64 oracle
    at 1e-5 and bitwise against the one-tile kernel"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = G.problem("ANDERSON3D-20-S1")
    A = SparseMat.from_crs(rp, c, v, dtype=np.float32, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n = len(rp) - 1
    x = G.random_block(n, nvec, 3).astype(np.float32)
    X = Mvec(A.domain_map, nvec, np.float32).set(x)
    Y = Mvec(A.row_map, nvec, np.float32)
    outs = []
    for pf in (0, 1):
        K.chk(K.phist_b200_set_spmv_prefetch, pf)
        K.chk(K.phist_SsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        outs.append(Y.get())
    assert np.array_equal(outs[0], outs[1])
    assert relerr(outs[1], oracle.spmmv(rp, c, v, x.astype(np.float64))) < 1e-5
    X.delete()
    Y.delete()
    A.delete()
