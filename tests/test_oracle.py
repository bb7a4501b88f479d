"""CPU oracle pinned against PHIST's own golden vectors and C kernels (no GPU).

* A2_precalc_result (test/kernels/SparseMatTest_def.hpp:751-950): hard-coded
  results of Y = A X for A = Dsprandn25, X(i,j) = i + j*n, checked there with
  max-abs error <= sqrt(eps) (:946); fixtures in tests/golden/a2_precalc.npz.
* PHIST's builtin C SpMMV kernels (spmvm_kernels_nt.c) and compensated dot
  (dot_kernels_prec.c), compiled from the PHIST sources into oracle/_ref/.
* Small pure-Python transcriptions of the builtin loops for the rest.
"""
import numpy as np
import pytest

from conftest import relerr

EPS = np.finfo(np.float64).eps


def test_a2_precalc_golden(oracle, testmats):
    import os
    from conftest import GOLDEN
    g = np.load(os.path.join(GOLDEN, "a2_precalc.npz"))
    rp, c, v, shape = testmats("sprandn25")
    n = shape[0]
    for nv in (1, 4):
        x = np.arange(n)[:, None] + np.arange(nv)[None, :] * float(n)
        y = oracle.spmmv(rp, c, v, x)
        err = np.abs(y - g["y_nv%d" % nv]).max()
        assert err <= np.sqrt(EPS), err   # the reference test's bound
        assert err <= 1e-12 * np.abs(g["y_nv%d" % nv]).max()


def _need_ref(oracle):
    if not oracle.ref_available():
        pytest.skip("PHIST C kernels not built into oracle/_ref")


@pytest.mark.parametrize("mat", ["sprandn388", "sprandn_nodiag388", "spshift388", "speye388", "sprandsym163"])
@pytest.mark.parametrize("nvec", [1, 2, 4, 8])
def test_spmmv_bitexact_vs_phist_c_kernels(oracle, testmats, mat, nvec):
    """the oracle and PHIST's builtin NT kernels (beta=0, both compiled
    without FMA contraction) agree bit for bit, shifts included"""
    _need_ref(oracle)
    rp, c, v, shape = testmats(mat)
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (shape[1], nvec))
    sh = rng.uniform(-2, 2, nvec)
    for alpha in (1.0, -0.7):
        yr = oracle.ref_spmmv_nt(rp, c, v, x, alpha=alpha, shifts=sh)
        yo = oracle.spmmv(rp, c, v, x, alpha=alpha, beta=0.0, shifts=sh)
        assert np.array_equal(yr, yo), np.abs(yr - yo).max()


@pytest.mark.parametrize("nvec", [1, 2, 4, 8])
def test_spmmv_close_to_phist_prec_kernels(oracle, nvec):
    """PHIST's compensated (double-double) SpMMV kernels agree with the plain
    oracle to rounding on a synthetic Anderson matrix"""
    _need_ref(oracle)
    from phist_b200 import generators as G
    rp, c, v = G.anderson3d(12, 1)
    x = G.random_block(len(rp) - 1, nvec, 5)
    yr = oracle.ref_spmmv_nt(rp, c, v, x, prec=True)
    yo = oracle.spmmv(rp, c, v, x)
    assert relerr(yo, yr) < 1e-15


@pytest.mark.parametrize("nvec", [1, 2, 4])
def test_dot_prec_vs_phist(oracle, nvec):
    """compensated column dots: oracle Dot2 vs PHIST ddot_prec_<nvec>"""
    _need_ref(oracle)
    rng = np.random.default_rng(3)
    n = 4096
    # ill-conditioned: large cancelling terms
    x = rng.uniform(-1, 1, (n, nvec)) * np.exp(rng.uniform(-20, 20, (n, nvec)))
    y = rng.uniform(-1, 1, (n, nvec))
    s, cc = oracle.ref_ddot_prec(x, y)
    d = oracle.dot(x, y, prec=True)
    exact = np.array([float(sum(np.longdouble(a) * np.longdouble(b) for a, b in zip(x[:, j], y[:, j]))) for j in range(nvec)])
    for j in range(nvec):
        ref = s[j] + cc[j]
        assert abs(d[j] - ref) <= 4 * EPS * abs(ref) + 1e-300, (d[j], ref)
        assert abs(d[j] - exact[j]) <= 1e-12 * np.abs(x[:, j] * y[:, j]).sum()


def test_spmmv_beta_alpha_semantics(oracle, testmats):
    """alpha=0 only scales y (crsmat_module.F90:1508-1511); beta mixes"""
    rp, c, v, shape = testmats("sprandn25")
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (25, 3))
    y0 = rng.uniform(-1, 1, (25, 3))
    y = oracle.spmmv(rp, c, v, x, alpha=0.0, beta=0.5, y=y0)
    assert np.array_equal(y, 0.5 * y0)
    A = np.zeros((25, 25))
    for i in range(25):
        for p in range(rp[i], rp[i + 1]):
            A[i, c[p]] += v[p]
    sh = np.array([0.5, -1.0, 2.0])
    y = oracle.spmmv(rp, c, v, x, alpha=2.0, beta=-0.5, y=y0, shifts=sh)
    ref = 2.0 * (A @ x + x * sh[None, :]) - 0.5 * y0
    assert relerr(y, ref) < 1e-14


def test_block_products_vs_numpy(oracle):
    rng = np.random.default_rng(7)
    n = 10007
    for m, k in ((1, 1), (4, 4), (5, 3), (8, 16), (32, 32)):
        V = rng.uniform(-1, 1, (n, m))
        W = rng.uniform(-1, 1, (n, k))
        C0 = rng.uniform(-1, 1, (m, k))
        C = oracle.mvTmv(V, W, alpha=0.5, beta=2.0, C=C0)
        assert relerr(C, 0.5 * V.T @ W + 2.0 * C0) < 1e-13
        Cp = oracle.mvTmv(V, W, alpha=0.5, beta=2.0, C=C0, prec=True)
        assert relerr(Cp, 0.5 * V.T @ W + 2.0 * C0) < 1e-14
        S = rng.uniform(-1, 1, (m, k))
        W2 = oracle.mvsd(V, S, alpha=1.5, beta=-1.0, W=W)
        assert relerr(W2, 1.5 * V @ S - W) < 1e-14
        if k <= m:
            M = rng.uniform(-1, 1, (m, k))
            Vi = oracle.mvsdi(V, M)
            assert relerr(Vi[:, :k], V @ M) < 1e-14
            assert np.array_equal(Vi[:, k:], V[:, k:])
        D = rng.uniform(-1, 1, (k, k))
        W3 = oracle.mvsd_add_mvsd(V, S, W, D)
        assert relerr(W3, V @ S + W @ D) < 1e-14
        W4, G = oracle.fused_mvsd_mvTmv(V, S, W, alpha=1.5, beta=-1.0)
        assert relerr(G, W4.T @ W4) < 1e-13
        if k <= m:
            Wi, Dd = oracle.fused_mvsdi_mvTmv(W[:, :min(k, m)] if False else V, V, rng.uniform(-1, 1, (m, k)), alpha=1.0, beta=0.0)
            assert Dd.shape == (m, k)


def _kacz_python(rp, col, val, shifts, b, x, omega, order):
    """direct transcription of kacz_sub_def.h:50-150 (one row at a time)"""
    x = x.copy()
    nvec = x.shape[1]
    for i in order:
        tmp = -shifts * x[i]
        nrm = 0.0
        d = 0.0
        for p in range(rp[i], rp[i + 1]):
            tmp = tmp + val[p] * x[col[p]]
            nrm += val[p] * val[p]
            if col[p] == i:
                d = val[p]
        if b is not None:
            tmp = tmp - b[i]
        rn = nrm - 2 * d * shifts + shifts * shifts
        rn = np.where(rn == 0.0, 1.0, rn)
        tmp = tmp * omega / rn
        x[i] = x[i] + tmp * shifts
        for p in range(rp[i], rp[i + 1]):
            x[col[p]] = x[col[p]] - tmp * val[p]
    return x


@pytest.mark.parametrize("mat", ["sprandn25", "spshift25", "symmMat20"])
def test_kaczmarz_vs_transcription(oracle, testmats, mat):
    rp, c, v, shape = testmats(mat)
    n = shape[0]
    rng = np.random.default_rng(2)
    nvec = 3
    x = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec))
    sh = np.array([0.0, 0.3, -1.2])
    om = np.array([1.0, 1.5, 0.8])
    order = np.arange(n)
    xo = oracle.carp_sweep(rp, c, v, sh, b, x, om)
    xp = _kacz_python(rp, c, v, sh, b, x, om, order)
    xp = _kacz_python(rp, c, v, sh, b, xp, om, order[::-1])
    assert relerr(xo, xp) < 1e-14


def test_kaczmarz_converges_on_spd(oracle):
    """CARP sweeps (SSOR on the normal equations) reduce the residual"""
    from phist_b200 import generators as G
    rp, c, v = G.laplace3d(6)
    n = len(rp) - 1
    b = G.random_block(n, 2, 9)
    x = np.zeros((n, 2))
    sh = np.array([0.0, 0.5])
    om = np.ones(2)
    r0 = np.linalg.norm(b)
    for _ in range(30):
        x = oracle.carp_sweep(rp, c, v, sh, b, x, om)
    r = b - (oracle.spmmv(rp, c, v, x, shifts=-sh))
    assert np.linalg.norm(r) < 0.05 * r0


def test_sell_perm(oracle, testmats):
    rp, c, v, shape = testmats("sprandn388")
    lens = np.diff(rp)
    for sigma in (1, 4, 32, 256, 10000):
        perm = oracle.sell_perm(rp, sigma)
        ref = np.arange(len(lens))
        if sigma > 1:
            for w0 in range(0, len(lens), sigma):
                w = np.arange(w0, min(w0 + sigma, len(lens)))
                ref[w0:w0 + len(w)] = w[np.argsort(-lens[w], kind="stable")]
        assert np.array_equal(perm, ref)


def test_dist2_checker(oracle):
    from phist_b200 import generators as G
    rp, c, v = G.laplace3d(4)
    n = len(rp) - 1
    assert oracle.check_dist2(rp, c, n, np.arange(n)) == 0       # all distinct
    assert oracle.check_dist2(rp, c, n, np.zeros(n)) != 0        # all equal


def test_oracle_jada_gmres_is_the_krylov_minimiser():
    """the numpy restatement of PHIST's correction-equation GMRES: after j
    steps its iterate minimises ||b - P(A - sigma I) x|| over the Krylov
    space of b (checked by dense least squares); with a large enough basis it
    converges; the result has unit norm"""
    from oracle import oracle as O
    rng = np.random.default_rng(0)
    n = 60
    A = rng.standard_normal((n, n))
    A = A + A.T + 10 * np.eye(n)
    Q = np.linalg.qr(rng.standard_normal((n, 3)))[0]
    R = rng.standard_normal((n, 2))
    R -= Q @ (Q.T @ R)
    P = np.eye(n) - Q @ Q.T
    for j in (1, 3, 7):
        t, conv = O.jada_gmres(A, Q, R[:, :1], [0.5], [1e-30], j, 20)
        op = P @ (A - 0.5 * np.eye(n))
        # an orthonormal basis of the Krylov space (the power basis is too
        # ill-conditioned for a tight comparison)
        K = np.zeros((n, j))
        v = R[:, 0] / np.linalg.norm(R[:, 0])
        for i in range(j):
            K[:, i] = v
            v = op @ v
            v -= K[:, :i + 1] @ (K[:, :i + 1].T @ v)
            v -= K[:, :i + 1] @ (K[:, :i + 1].T @ v)
            v /= np.linalg.norm(v)
        c, *_ = np.linalg.lstsq(op @ K, R[:, 0], rcond=None)
        x = K @ c
        assert not conv[0]
        assert np.linalg.norm(t[:, 0] - x / np.linalg.norm(x)) < 1e-10
    t, conv = O.jada_gmres(A, Q, R, [0.5, 1.0], [1e-10, 1e-10], 200, 60)
    assert conv.all()
    assert np.allclose(np.linalg.norm(t, axis=0), 1.0)
    for s, sg in enumerate((0.5, 1.0)):
        y = P @ (A - sg * np.eye(n)) @ t[:, s]
        a = (y @ R[:, s]) / (y @ y)
        assert np.linalg.norm(a * y - R[:, s]) < 1e-9 * np.linalg.norm(R[:, s])


def test_oracle_jada_gmres_restart_semantics():
    """restarted GMRES(m) in the restatement: two cycles of m steps equal
    x1 = argmin over K_m(b), then x2 = x1 + argmin over K_m(b - op x1)
    (dense least squares on orthonormal Krylov bases), scaled to unit norm"""
    from oracle import oracle as O
    rng = np.random.default_rng(1)
    n, m = 50, 4
    A = rng.standard_normal((n, n))
    A = A + A.T + 8 * np.eye(n)
    Q = np.linalg.qr(rng.standard_normal((n, 2)))[0]
    b = rng.standard_normal(n)
    b -= Q @ (Q.T @ b)
    sigma = 0.7
    P = np.eye(n) - Q @ Q.T
    op = P @ (A - sigma * np.eye(n))

    def krylov_min(r):
        K = np.zeros((n, m))
        v = r / np.linalg.norm(r)
        for i in range(m):
            K[:, i] = v
            v = op @ v
            for _ in range(2):
                v -= K[:, :i + 1] @ (K[:, :i + 1].T @ v)
            v /= np.linalg.norm(v)
        c, *_ = np.linalg.lstsq(op @ K, r, rcond=None)
        return K @ c

    x1 = krylov_min(b)
    x2 = x1 + krylov_min(b - op @ x1)
    t, conv = O.jada_gmres(A, Q, b[:, None], [sigma], [1e-30], 2 * m, m)
    assert not conv[0]
    assert np.linalg.norm(t[:, 0] - x2 / np.linalg.norm(x2)) < 1e-10


def test_oracle_jada_minres_equals_gmres_on_symmetric_operators():
    """the numpy restatement of PHIST's MINRES: for a symmetric A the
    projected operator is symmetric on the complement of Q, so MINRES and
    GMRES minimise the residual over the same Krylov space and their iterates
    after j steps coincide (restarted too); converged runs solve the
    systems"""
    from oracle import oracle as O
    rng = np.random.default_rng(2)
    n = 60
    A = rng.standard_normal((n, n))
    A = A + A.T + 10 * np.eye(n)
    Q = np.linalg.qr(rng.standard_normal((n, 3)))[0]
    R = rng.standard_normal((n, 2))
    R -= Q @ (Q.T @ R)
    P = np.eye(n) - Q @ Q.T
    for j, m in ((1, 20), (3, 20), (8, 20), (10, 4)):
        tm, cm = O.jada_minres(A, Q, R, [0.5, -0.3], [1e-30, 1e-30], j, m)
        tg, cg = O.jada_gmres(A, Q, R, [0.5, -0.3], [1e-30, 1e-30], j, m)
        assert not cm.any() and not cg.any()
        assert np.linalg.norm(tm - tg) < 1e-9, (j, m, np.linalg.norm(tm - tg))
    # restarted MINRES needs the basis of its cap here: Lanczos without
    # reorthogonalisation converges late on this indefinite operator (about
    # 80 steps unrestarted for n = 60), and a restart after 60 steps keeps
    # only a 1e-4 residual
    t, conv = O.jada_minres(A, Q, R, [0.5, 1.0], [1e-10, 1e-10], 400, 63)
    assert conv.all()
    for s, sg in enumerate((0.5, 1.0)):
        y = P @ (A - sg * np.eye(n)) @ t[:, s]
        a = (y @ R[:, s]) / (y @ y)
        assert np.linalg.norm(a * y - R[:, s]) < 1e-9 * np.linalg.norm(R[:, s])


def test_oracle_carp_cgmn_solves_shifted_systems():
    """the CGMN restatement converges to the dense solutions of
    (A - sigma_j I) x_j = b_j (small honeycomb, shifts outside the spectrum)"""
    from oracle import oracle as O
    from phist_b200 import generators as G
    rp, c, v = G.honeycomb(6, 6, 2)
    n = len(rp) - 1
    A = np.zeros((n, n))
    np.add.at(A, (np.repeat(np.arange(n), np.diff(rp)), c), v)
    sig = np.array([-4.0, 4.5])
    b = np.random.default_rng(0).uniform(-1, 1, (n, 2))
    x = O.carp_cgmn(rp, c, v, sig, b, 60)
    for j in range(2):
        xs = np.linalg.solve(A - sig[j] * np.eye(n), b[:, j])
        assert np.linalg.norm(x[:, j] - xs) / np.linalg.norm(xs) < 1e-10


@pytest.mark.parametrize("m,k", [(1, 3), (2, 5), (4, 4), (4, 9)])
def test_mvTmv_prec_vs_phist(oracle, m, k):
    """compensated Gram products: the oracle's Dot2 restatement against
    PHIST's own dgemm_sc_prec_<m>_k (gemm_kernels_sC_prec.c) on
    ill-conditioned columns (large cancelling terms), to a few ulp"""
    _need_ref(oracle)
    rng = np.random.default_rng(m * 10 + k)
    n = 4096
    V = rng.uniform(-1, 1, (n, m)) * np.exp(rng.uniform(-20, 20, (n, m)))
    W = rng.uniform(-1, 1, (n, k))
    hi, lo = oracle.ref_gemm_sc_prec(V, W)
    C = oracle.mvTmv(V, W, prec=True)
    ref = hi + lo
    # Dot2 bound (Ogita-Rump-Oishi 2005, Prop. 5.3) for two differently
    # ordered compensated sums: a few ulp of the result plus n eps^2 sum|v w|
    bound = 8 * EPS * np.abs(ref) + 4 * n * EPS ** 2 * (np.abs(V).T @ np.abs(W))
    assert np.all(np.abs(C - ref) <= bound)
    # plain FP64 loses digits on these columns; the compensated sums do not
    plain = oracle.mvTmv(V, W)
    assert np.abs(plain - ref).max() > np.abs(C - ref).max()
