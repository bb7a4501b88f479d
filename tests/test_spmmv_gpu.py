"""SpMMV on the GPU (through the C ABI) against the CPU oracle.

Covers the reference's SparseMatTest cases (speye, spzero, sprandn,
sprandn_nodiag, spshift at n=25/388, nvec 1/4/7/12; test/kernels/
SparseMatTest.cpp:28-263), the A2_precalc_result golden vectors, shifts,
alpha/beta variants, strided views, the SELL-C-sigma variants and the fused
dot/axpby epilogues.  FP64 tolerance: 1e-13 relative (norm-wise).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _dense(rp, c, v, shape):
    A = np.zeros(shape)
    for i in range(shape[0]):
        for p in range(rp[i], rp[i + 1]):
            A[i, c[p]] += v[p]
    return A


@pytest.fixture(params=[(32, 1), (32, 256), (8, 16), (1, 1)], ids=lambda p: "C%d-s%d" % p)
def sell(request, session):
    from phist_b200 import kernels as K
    C, sigma = request.param
    K.chk(K.phist_b200_set_sell_params, C, sigma)
    yield request.param
    K.chk(K.phist_b200_set_sell_params, 32, 256)


def _mat(testmats, name, sigma, dtype=np.float64):
    from phist_b200 import kernels as K
    from phist_b200.objects import SparseMat
    rp, c, v, shape = testmats(name)
    flags = K.PHIST_SPARSEMAT_PERM_LOCAL if sigma > 1 else 0
    return SparseMat.from_crs(rp, c, v, ncols=shape[1], dtype=dtype, flags=flags), (rp, c, v, shape)


def test_a2_precalc_result_gpu(session, testmats, sell):
    from phist_b200 import kernels as K
    from phist_b200.objects import Map, Mvec
    g = np.load(os.path.join(GOLDEN, "a2_precalc.npz"))
    A, (rp, c, v, shape) = _mat(testmats, "sprandn25", sell[1])
    for nv in (1, 4):
        x = np.arange(25)[:, None] + np.arange(nv)[None, :] * 25.0
        X = Mvec(A.domain_map, nv).set(x)
        Y = Mvec(A.row_map, nv)
        K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        y = Y.get()
        assert np.abs(y - g["y_nv%d" % nv]).max() <= np.sqrt(np.finfo(float).eps)
        assert relerr(y, g["y_nv%d" % nv]) < TOL
        X.delete(); Y.delete()
    A.delete()


MATS = ["speye25", "spzero25", "sprandn25", "sprandn_nodiag25", "spshift25",
        "speye388", "sprandn388", "sprandn_nodiag388", "spshift388", "sprandsym163", "jadaTestMat512"]


@pytest.mark.parametrize("name", MATS)
@pytest.mark.parametrize("nvec", [1, 2, 4, 7, 8, 12, 16, 32, 40])
def test_spmmv_vs_oracle(session, testmats, oracle, sell, name, nvec):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec
    A, (rp, c, v, shape) = _mat(testmats, name, sell[1])
    rng = np.random.default_rng(nvec * 7 + len(name))
    x = rng.uniform(-1, 1, (shape[1], nvec))
    y0 = rng.uniform(-1, 1, (shape[0], nvec))
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec)
    for alpha, beta in ((1.0, 0.0), (-0.5, 2.0), (0.0, 0.7), (2.0, 1.0)):
        Y.set(y0)
        K.chk(K.phist_DsparseMat_times_mvec, alpha, A.h, X.h, beta, Y.h)
        ref = oracle.spmmv(rp, c, v, x, alpha=alpha, beta=beta, y=y0)
        assert relerr(Y.get(), ref) < TOL, (alpha, beta)
    # per-column shifts (apply_shifted of jadaOp, phist_operator_def.hpp:102)
    sh = rng.uniform(-3, 3, nvec)
    Y.set(y0)
    K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, 1.5, A.h, K.sptr(sh, np.float64), X.h, -1.0, Y.h)
    ref = oracle.spmmv(rp, c, v, x, alpha=1.5, beta=-1.0, y=y0, shifts=sh)
    assert relerr(Y.get(), ref) < TOL
    # scalar shift
    Y.set(y0)
    K.chk(K.phist_DsparseMat_times_mvec_add_mvec, 0.5, A.h, 0.25, X.h, 1.0, Y.h)
    ref = oracle.spmmv(rp, c, v, x, alpha=0.5, beta=1.0, y=y0, shifts=np.full(nvec, 0.25))
    assert relerr(Y.get(), ref) < TOL
    X.delete(); Y.delete(); A.delete()


@pytest.mark.parametrize("nvec,j0,j1", [(8, 2, 5), (12, 0, 3), (16, 1, 1), (33, 5, 36 - 4), (10, 4, 7)])
def test_spmmv_views(session, testmats, oracle, nvec, j0, j1):
    """strided column views of X and Y (mvec_view_block, SparseMatTest views)"""
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec
    A, (rp, c, v, shape) = _mat(testmats, "sprandn388", 256)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (shape[1], nvec))
    y = rng.uniform(-1, 1, (shape[0], nvec + 3))
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec + 3).set(y)
    Xv = X.view(j0, j1)
    Yv = Y.view(j0 + 2, j1 + 2)
    K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, Xv.h, 0.5, Yv.h)
    ref = y.copy()
    ref[:, j0 + 2:j1 + 3] = oracle.spmmv(rp, c, v, x[:, j0:j1 + 1], alpha=1.0, beta=0.5, y=y[:, j0 + 2:j1 + 3])
    out = Y.get()
    assert relerr(out, ref) < TOL
    assert np.array_equal(out[:, :j0 + 2], y[:, :j0 + 2])   # untouched columns
    Xv.delete(); Yv.delete(); X.delete(); Y.delete(); A.delete()


@pytest.mark.parametrize("nvec", [1, 3, 4, 8, 16, 32])
def test_fused_spmv_mvdot(session, testmats, oracle, nvec):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec
    A, (rp, c, v, shape) = _mat(testmats, "sprandn388", 1)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (shape[1], nvec))
    y0 = rng.uniform(-1, 1, (shape[0], nvec))
    u0 = rng.uniform(-1, 1, (shape[0], nvec))
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec).set(y0)
    wdw = np.zeros(nvec)
    vdw = np.zeros(nvec)
    K.chk(K.phist_Dfused_spmv_mvdot, 2.0, A.h, X.h, 0.5, Y.h, K.sptr(wdw, np.float64), K.sptr(vdw, np.float64))
    y = oracle.spmmv(rp, c, v, x, alpha=2.0, beta=0.5, y=y0)
    assert relerr(Y.get(), y) < TOL
    assert relerr(wdw, (y * y).sum(0)) < TOL
    assert relerr(vdw, (x * y).sum(0)) < TOL
    # with the axpby epilogue U = gamma W + delta U
    U = Mvec(A.row_map, nvec).set(u0)
    Y.set(y0)
    K.chk(K.phist_Dfused_spmv_mvdot_mvadd, 2.0, A.h, X.h, 0.5, Y.h, -1.0, 3.0, U.h,
          K.sptr(wdw, np.float64), K.sptr(vdw, np.float64))
    assert relerr(U.get(), -1.0 * y + 3.0 * u0) < TOL
    assert relerr(wdw, (y * y).sum(0)) < TOL
    # only one of the dots requested (NULL arrays allowed)
    Y.set(y0)
    K.chk(K.phist_Dfused_spmv_mvdot, 2.0, A.h, X.h, 0.5, Y.h, None, K.sptr(vdw, np.float64))
    assert relerr(vdw, (x * y).sum(0)) < TOL
    for o in (X, Y, U):
        o.delete()
    A.delete()


@pytest.mark.parametrize("nvec", [1, 4, 8])
def test_fused_spmv_mvTmv(session, testmats, oracle, nvec):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SdMat
    A, (rp, c, v, shape) = _mat(testmats, "sprandn388", 1)
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, (shape[1], nvec))
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec)
    WtW = SdMat(nvec, nvec)
    VtW = SdMat(nvec, nvec)
    K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, Y.h, WtW.h, VtW.h)
    y = oracle.spmmv(rp, c, v, x)
    assert relerr(Y.get(), y) < TOL
    assert relerr(WtW.get(), y.T @ y) < TOL
    assert relerr(VtW.get(), x.T @ y) < TOL
    # W == NULL is allowed (fused_decl.h:67)
    K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, None, WtW.h, None)
    assert relerr(WtW.get(), y.T @ y) < TOL
    for o in (X, Y, WtW, VtW):
        o.delete()
    A.delete()


def test_fused_spmv_pair(session, testmats, oracle):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec
    A1, (rp1, c1, v1, sh1) = _mat(testmats, "sprandn388", 1)
    A2, (rp2, c2, v2, sh2) = _mat(testmats, "spshift388", 1)
    rng = np.random.default_rng(8)
    nvec = 3
    x = rng.uniform(-1, 1, (388, nvec))
    y0 = rng.uniform(-1, 1, (388, nvec))
    s1 = np.array([1.0, -0.5, 2.0])
    s2 = np.array([0.0, 1.5, -1.0])
    X = Mvec(A1.domain_map, nvec).set(x)
    Y = Mvec(A1.row_map, nvec).set(y0)
    K.chk(K.phist_Dfused_spmv_pair, 0.5, K.sptr(s1, np.float64), A1.h, K.sptr(s2, np.float64), A2.h, X.h, 2.0, Y.h)
    ref = 0.5 * (oracle.spmmv(rp1, c1, v1, x) * s1 + oracle.spmmv(rp2, c2, v2, x) * s2) + 2.0 * y0
    assert relerr(Y.get(), ref) < TOL
    for o in (X, Y, A1, A2):
        o.delete()


@pytest.mark.parametrize("sigma", [1, 256])
def test_sell_permutation_bitexact(session, testmats, oracle, sigma):
    """the sigma sort of the library equals the oracle's, bit for bit"""
    from phist_b200 import kernels as K
    K.chk(K.phist_b200_set_sell_params, 32, sigma)
    A, (rp, c, v, shape) = _mat(testmats, "sprandn388", sigma)
    info = A.sell_info()
    assert np.array_equal(info["perm"], oracle.sell_perm(rp, sigma))
    lens = np.diff(rp)[info["perm"]]
    nch = info["nchunks"]
    padded = sum(int(lens[ch * 32:(ch + 1) * 32].max()) * 32 for ch in range(nch))
    assert info["nnz_padded"] == padded
    A.delete()
    K.chk(K.phist_b200_set_sell_params, 32, 256)


def test_spmmv_single_precision(session, testmats, oracle):
    """FP32 matrix and vectors with FP32 accumulation (mixed-precision form);
    error against the FP64 oracle is stated as a tolerance of 1e-5"""
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec
    A, (rp, c, v, shape) = _mat(testmats, "sprandn388", 256, dtype=np.float32)
    rng = np.random.default_rng(9)
    for nvec in (1, 2, 4, 8, 16, 32):
        x = rng.uniform(-1, 1, (388, nvec)).astype(np.float32)
        X = Mvec(A.domain_map, nvec, np.float32).set(x)
        Y = Mvec(A.row_map, nvec, np.float32)
        K.chk(K.phist_SsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        ref64 = oracle.spmmv(rp, c, v, x.astype(np.float64))
        ref32 = oracle.spmmv(rp, c, v.astype(np.float32), x)
        assert relerr(Y.get(), ref64) < 1e-5
        assert relerr(Y.get(), ref32) < 1e-5
        X.delete(); Y.delete()
    A.delete()


def test_rowfunc_matrix_equals_crs(session, oracle):
    """sparseMat_create_fromRowFunc (the builtin generators' path) and the
    CRS constructor build the same operator"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    for prob in ("ANDERSON3D-16-S1", "HONEYCOMB-16x12-S4", "LAPLACE3D-12"):
        A = SparseMat.from_problem(prob)
        rp, c, v = G.problem(prob)
        n = len(rp) - 1
        assert A.nrows == n and A.nnz == rp[-1]
        x = G.random_block(n, 4, 1)
        X = Mvec(A.domain_map, 4).set(x)
        Y = Mvec(A.row_map, 4)
        K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
        assert relerr(Y.get(), oracle.spmmv(rp, c, v, x)) < TOL
        X.delete(); Y.delete(); A.delete()


@pytest.mark.parametrize("prob", ["ANDERSON3D-24-S1", "HONEYCOMB-40x24-S4", "LAPLACE3D-20"])
@pytest.mark.parametrize("nvec", [8, 16, 32])
def test_staged_kernel_matches_oracle_and_register_path(session, oracle, prob, nvec):
    """short-row matrices at block widths 8..32 take the shared-memory staged
    kernel; it must agree with the oracle and with the register kernel"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    rp, c, v = G.problem(prob)
    A = SparseMat.from_crs(rp, c, v, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n = len(rp) - 1
    x = G.random_block(n, nvec, 7)
    y0 = G.random_block(n, nvec, 8)
    sh = np.linspace(-1, 1, nvec)
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec)
    outs = []
    for staged_min in (8, 99):
        K.chk(K.phist_b200_set_spmv_staged, staged_min)
        Y.set(y0)
        K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, 0.75, A.h, K.sptr(sh, np.float64), X.h, -0.5, Y.h)
        outs.append(Y.get())
    K.chk(K.phist_b200_set_spmv_staged, 99)  # the library default
    ref = oracle.spmmv(rp, c, v, x, alpha=0.75, beta=-0.5, y=y0, shifts=sh)
    assert relerr(outs[0], ref) < TOL
    assert relerr(outs[1], ref) < TOL
    assert relerr(outs[0], outs[1]) < 1e-15
    X.delete(); Y.delete(); A.delete()


@pytest.mark.parametrize("nvec,tprs", [(4, (1, 2)), (8, (1, 2, 4)), (16, (2, 4, 8)), (32, (4, 8, 16))])
@pytest.mark.parametrize("prob", ["LAPDIAG3D-12-S5", "HONEYCOMB-20-S4-W1"])
def test_every_launch_shape_matches_oracle(session, oracle, prob, nvec, tprs):
    """every threads-per-row choice of phist_b200_set_spmv_config, unrolled
    (rows of at most 8 entries) and runtime-loop kernels, against the oracle"""
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    rp, c, v = G.problem(prob)
    A = SparseMat.from_crs(rp, c, v, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n = len(rp) - 1
    x = G.random_block(n, nvec, 11)
    y0 = G.random_block(n, nvec, 12)
    sh = np.linspace(-1, 1, nvec)
    X = Mvec(A.domain_map, nvec).set(x)
    Y = Mvec(A.row_map, nvec)
    ref = oracle.spmmv(rp, c, v, x, alpha=0.75, beta=-0.5, y=y0, shifts=sh)
    defaults = {4: 1, 8: 2, 16: 4, 32: 8}
    try:
        for tpr in tprs:
            for unroll in (1, 0):
                K.chk(K.phist_b200_set_spmv_config, nvec, tpr, unroll)
                Y.set(y0)
                K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, 0.75, A.h, K.sptr(sh, np.float64), X.h, -0.5, Y.h)
                assert relerr(Y.get(), ref) < TOL, (tpr, unroll)
    finally:
        K.chk(K.phist_b200_set_spmv_config, nvec, defaults[nvec], 1)
    X.delete(); Y.delete(); A.delete()


def test_read_mm(session, oracle, testmats, tmp_path):
    """sparseMat_read_mm (phist_kernels_decl.h:98) on a MatrixMarket file"""
    import ctypes as ct
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat, Session
    rp, c, v, shape = testmats("sprandn25")
    path = tmp_path / "a.mm"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n%d %d %d\n" % (shape[0], shape[1], rp[-1]))
        for i in range(shape[0]):
            for p in range(rp[i], rp[i + 1]):
                f.write("%d %d %.17g\n" % (i + 1, c[p] + 1, v[p]))
    h = ct.c_void_p()
    K.chk(K.phist_DsparseMat_read_mm, ct.byref(h), Session.get().comm, str(path).encode())
    A = SparseMat(h, np.float64)
    x = np.random.default_rng(1).uniform(-1, 1, (25, 2))
    X = Mvec(A.domain_map, 2).set(x)
    Y = Mvec(A.row_map, 2)
    K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h)
    assert relerr(Y.get(), oracle.spmmv(rp, c, v, x)) < TOL
    X.delete(); Y.delete(); A.delete()


def test_shape_errors(session, testmats):
    """invalid input gives -55 and leaves no device fault"""
    from phist_b200 import kernels as K
    from phist_b200.objects import Map, Mvec
    os.environ["PHIST_B200_QUIET"] = "1"
    A, _ = _mat(testmats, "sprandn25", 1)
    X = Mvec(A.domain_map, 2)
    Y = Mvec(A.row_map, 3)
    assert K.iflag_of(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h) == K.PHIST_INVALID_INPUT
    m = Map(24)
    Z = Mvec(m.h, 2)
    assert K.iflag_of(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Z.h) == K.PHIST_INVALID_INPUT
    assert K.iflag_of(K.phist_DsparseMat_times_mvec, 1.0, None, X.h, 0.0, Z.h) == K.PHIST_BAD_CAST
    assert K.iflag_of(K.phist_DsparseMatT_times_mvec, 1.0, A.h, X.h, 0.0, Z.h) == K.PHIST_NOT_IMPLEMENTED
    for o in (X, Y, Z, A, m):
        o.delete()
    del os.environ["PHIST_B200_QUIET"]
