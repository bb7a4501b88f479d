"""Device-resident GMRES and MINRES for the Jacobi-Davidson correction
equations (phist_b200_{D,S}jadaCorrection_{gmres,minres}, csrc/pb_gmres.cu)
against the numpy restatements of PHIST's GMRES and MINRES in the oracle: the
iterate after a given number of steps is unique (the residual minimiser over
the Krylov space), so cut-off runs, restarted runs and converged runs must
agree with it.  For the symmetric test operators MINRES and GMRES minimise
over the same space, so the MINRES iterate also equals GMRES's."""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu


def _dense(rp, c, v):
    n = len(rp) - 1
    A = np.zeros((n, n))
    np.add.at(A, (np.repeat(np.arange(n), np.diff(rp)), c), v)
    return A


def _setup(problem, nq, k, seed, extra=0):
    from phist_b200 import generators as G
    rp, c, v = G.problem(problem)
    n = len(rp) - 1
    rng = np.random.default_rng(seed)
    Q = np.linalg.qr(rng.standard_normal((n, nq)))[0] if nq else np.zeros((n, 0))
    R = rng.standard_normal((n, k + extra))
    R -= Q @ (Q.T @ R)
    sigma = rng.uniform(0.5, 1.5, k)
    return rp, c, v, Q, R, sigma


def _run(rp, c, v, Q, R, sigma, tol, max_iter, max_bas, res_index=None, dtype=np.float64, solver="gmres"):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    A = SparseMat.from_crs(rp, c, v, dtype=dtype)
    k = len(sigma)
    Qm = Mvec(A.row_map, Q.shape[1], dtype=dtype).set(Q) if Q.shape[1] else None
    Rm = Mvec(A.row_map, R.shape[1], dtype=dtype).set(R)
    Tm = Mvec(A.row_map, k, dtype=dtype)
    sg = np.ascontiguousarray(sigma, np.float64)
    tl = np.full(k, tol, np.float64)
    idx = np.ascontiguousarray(res_index, np.int32) if res_index is not None else None
    f = getattr(K, "phist_b200_%sjadaCorrection_%s" % ("D" if dtype == np.float64 else "S", solver))
    iflag = K.iflag_of(f, A.h, Qm.h if Qm else None, Rm.h, K.ptr(idx) if idx is not None else None, k, K.ptr(sg),
                       K.ptr(tl), max_iter, max_bas, Tm.h)
    t = Tm.get()
    for o in (Qm, Rm, Tm, A):
        if o is not None:
            o.delete()
    return t, iflag


@pytest.mark.parametrize("problem,nq,k,max_iter,max_bas", [("LAPDIAG3D-8-S1", 6, 4, 7, 20),
                                                           ("LAPDIAG3D-8-S1", 6, 4, 12, 4),
                                                           ("HONEYCOMB-12-S3-W1", 3, 2, 9, 5),
                                                           ("LAPLACE3D-7", 0, 3, 10, 20),
                                                           ("LAPDIAG3D-9-S4", 4, 4, 30, 30),
                                                           ("LAPDIAG3D-8-S1", 2, 8, 22, 22)])
def test_gmres_cut_off_matches_oracle(session, oracle, problem, nq, k, max_iter, max_bas):
    """no convergence within max_iter (tolerance unreachable): the iterate of
    exactly max_iter steps, with restarts every max_bas steps"""
    rp, c, v, Q, R, sigma = _setup(problem, nq, k, 3)
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-30, max_iter, max_bas)
    ref, conv = oracle.jada_gmres(_dense(rp, c, v), Q, R, sigma, np.full(k, 1e-30), max_iter, max_bas)
    assert iflag == k and not conv.any()
    assert np.abs(np.linalg.norm(t, axis=0) - 1).max() < 1e-12
    assert relerr(t, ref) < 1e-9, relerr(t, ref)


def test_gmres_converges_and_res_index(session, oracle):
    """converged systems (tolerance 1e-9), right-hand sides picked by resIndex
    from a wider block, solution orthogonal to Q up to the tolerance"""
    rp, c, v, Q, R, sigma = _setup("LAPDIAG3D-9-S2", 5, 3, 4, extra=2)
    idx = [4, 0, 2]
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-9, 300, 40, res_index=idx)
    A = _dense(rp, c, v)
    ref, conv = oracle.jada_gmres(A, Q, R, sigma, np.full(3, 1e-9), 300, 40, res_index=idx)
    assert iflag == 0 and conv.all()
    assert relerr(t, ref) < 1e-7
    P = np.eye(len(A)) - Q @ Q.T
    for s in range(3):
        b = R[:, idx[s]]
        y = P @ (A - sigma[s] * np.eye(len(A))) @ t[:, s]
        # t is the solution scaled to unit norm: the best multiple of y fits b
        a = (y @ b) / (y @ y)
        assert np.linalg.norm(a * y - b) / np.linalg.norm(b) < 1e-8


def test_gmres_fp32(session, oracle):
    """the FP32 form (FP32 SpMMV and block products, FP64 small dense part)
    against the FP64 oracle: agreement to FP32 rounding"""
    rp, c, v, Q, R, sigma = _setup("LAPDIAG3D-8-S1", 6, 4, 5)
    R *= 1024.0 / np.linalg.norm(R, axis=0)
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-5, 200, 40, dtype=np.float32)
    A = _dense(rp, c, v)
    ref, conv = oracle.jada_gmres(A, Q, R, sigma, np.full(4, 1e-5), 200, 40)
    assert iflag == 0 and conv.all()
    # both stop near the tolerance, possibly a step apart
    assert relerr(t, ref) < 1e-3
    P = np.eye(len(A)) - Q @ Q.T
    for s in range(4):
        y = P @ (A - sigma[s] * np.eye(len(A))) @ t[:, s].astype(np.float64)
        a = (y @ R[:, s]) / (y @ y)
        assert np.linalg.norm(a * y - R[:, s]) / np.linalg.norm(R[:, s]) < 1e-4


def test_gmres_bad_arguments(session):
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    A = SparseMat.from_problem("LAPLACE3D-4")
    R = Mvec(A.row_map, 2)
    T = Mvec(A.row_map, 3)
    sg = np.zeros(3)
    tl = np.full(3, 1e-8)
    # t has 3 columns, 3 systems, but R has only 2 columns for the default resIndex
    assert K.iflag_of(K.phist_b200_DjadaCorrection_gmres, A.h, None, R.h, None, 3, K.ptr(sg), K.ptr(tl), 10, 10,
                      T.h) < 0
    for o in (R, T, A):
        o.delete()


# symmetric problems only (PHIST's MINRES needs a symmetric operator)
@pytest.mark.parametrize("problem,nq,k,max_iter,max_bas", [("LAPDIAG3D-8-S1", 6, 4, 7, 20),
                                                           ("LAPDIAG3D-8-S1", 6, 4, 12, 4),
                                                           ("LAPLACE3D-7", 0, 3, 10, 20),
                                                           ("LAPDIAG3D-9-S4", 4, 4, 16, 16),
                                                           ("LAPDIAG3D-8-S1", 2, 8, 10, 10)])
def test_minres_cut_off_matches_oracle(session, oracle, problem, nq, k, max_iter, max_bas):
    """no convergence within max_iter: the MINRES iterate of exactly max_iter
    steps (restarts every max_bas), against the oracle's MINRES and GMRES"""
    rp, c, v, Q, R, sigma = _setup(problem, nq, k, 3)
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-30, max_iter, max_bas, solver="minres")
    A = _dense(rp, c, v)
    ref, conv = oracle.jada_minres(A, Q, R, sigma, np.full(k, 1e-30), max_iter, max_bas)
    gm, _ = oracle.jada_gmres(A, Q, R, sigma, np.full(k, 1e-30), max_iter, max_bas)
    assert iflag == k and not conv.any()
    assert np.abs(np.linalg.norm(t, axis=0) - 1).max() < 1e-12
    assert relerr(t, ref) < 1e-9, relerr(t, ref)
    assert relerr(t, gm) < 1e-7, relerr(t, gm)


def test_minres_converges_and_res_index(session, oracle):
    """converged systems (tolerance 1e-9), right-hand sides picked by resIndex
    from a wider block; each t solves its system up to its scale"""
    rp, c, v, Q, R, sigma = _setup("LAPDIAG3D-9-S2", 5, 3, 4, extra=2)
    idx = [4, 0, 2]
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-9, 400, 40, res_index=idx, solver="minres")
    A = _dense(rp, c, v)
    ref, conv = oracle.jada_minres(A, Q, R, sigma, np.full(3, 1e-9), 400, 40, res_index=idx)
    assert iflag == 0 and conv.all()
    assert relerr(t, ref) < 1e-6
    P = np.eye(len(A)) - Q @ Q.T
    for s in range(3):
        b = R[:, idx[s]]
        y = P @ (A - sigma[s] * np.eye(len(A))) @ t[:, s]
        a = (y @ b) / (y @ y)
        assert np.linalg.norm(a * y - b) / np.linalg.norm(b) < 1e-8


def test_minres_fp32(session, oracle):
    """the FP32 form against the FP64 oracle: agreement to FP32 rounding.
    FP32 Lanczos loses orthogonality sooner: with restarts after 40 steps one
    of these systems stalls above 1e-5 (so does the restatement run in FP32),
    with the largest basis (63) all converge"""
    rp, c, v, Q, R, sigma = _setup("LAPDIAG3D-8-S1", 6, 4, 5)
    R *= 1024.0 / np.linalg.norm(R, axis=0)
    t, iflag = _run(rp, c, v, Q, R, sigma, 1e-5, 400, 63, dtype=np.float32, solver="minres")
    A = _dense(rp, c, v)
    ref, conv = oracle.jada_minres(A, Q, R, sigma, np.full(4, 1e-5), 400, 63)
    assert iflag == 0 and conv.all()
    assert relerr(t, ref) < 1e-3
    P = np.eye(len(A)) - Q @ Q.T
    for s in range(4):
        y = P @ (A - sigma[s] * np.eye(len(A))) @ t[:, s].astype(np.float64)
        a = (y @ R[:, s]) / (y @ y)
        assert np.linalg.norm(a * y - R[:, s]) / np.linalg.norm(R[:, s]) < 1e-4
