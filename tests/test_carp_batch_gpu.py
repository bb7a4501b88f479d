"""Batched multi-shift CARP-CG on the GPU (phist_b200_DcarpCG_batch): the
CGMN recurrence of PHIST's carp_cg (phist_carp_cg_def.hpp:440-690) for a
queue of shifted systems (A - sigma_j I) x_j = b_j through a few slots, with
converged systems handing their slot to the next one; FP64 and FP32-inner
with FP64 refinement.

Checked independently of the library: residuals recomputed with numpy on the
generator's CRS arrays, and the solutions compared with dense solves (error
bounded by cond(A - sigma I) times the residual)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense(rp, c, v):
    n = len(rp) - 1
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    np.add.at(A, (rows, c), v)
    return A


def _run(problem, nsys, block, mixed, tol=1e-10, max_iter=60000, check=10, seed=7):
    import ctypes as ct

    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    rp, c, v = G.problem(problem)
    n = len(rp) - 1
    A = SparseMat.from_crs(rp, c, v)
    sig = 2.5 * G.unif(seed, np.arange(nsys, dtype=np.uint64))
    b = G.random_block(n, nsys, seed + 1) if nsys else np.zeros((n, 0))
    B = Mvec(A.row_map, max(nsys, 1)).set(b if nsys else np.zeros((n, 1)))
    X = Mvec(A.row_map, max(nsys, 1))
    iters = np.zeros(max(nsys, 1), np.int32)
    rel = np.zeros(max(nsys, 1))
    iflag = K.iflag_of(K.phist_b200_DcarpCG_batch, A.h, nsys, K.ptr(sig), B.h, X.h, block, tol, max_iter, check,
                       mixed, 1e-5, K.ptr(iters), K.ptr(rel))
    x = X.get()
    for o in (B, X, A):
        o.delete()
    return rp, c, v, sig, b, x[:, :nsys], iters[:nsys], rel[:nsys], iflag


@pytest.mark.parametrize("mixed", [0, 1])
@pytest.mark.parametrize("problem,nsys,block", [("HONEYCOMB-24-S4-W1", 10, 4), ("LAPDIAG3D-10-S5", 7, 8),
                                                ("HONEYCOMB-16x12-S2-W1", 5, 1)])
def test_batch_converges_to_fp64_residual(session, problem, nsys, block, mixed):
    tol = 1e-10
    rp, c, v, sig, b, x, iters, rel, iflag = _run(problem, nsys, block, mixed, tol)
    assert iflag == 0, (iflag, rel)
    assert (iters > 0).all()
    A = _dense(rp, c, v)
    lam = np.linalg.eigvalsh(A) if np.allclose(A, A.T) else None
    for j in range(nsys):
        r = b[:, j] - (A @ x[:, j] - sig[j] * x[:, j])
        relj = np.linalg.norm(r) / np.linalg.norm(b[:, j])
        assert relj <= 2 * tol, (j, relj)
        assert abs(relj - rel[j]) <= 1e-3 * relj + 1e-14
        xs = np.linalg.solve(A - sig[j] * np.eye(len(b)), b[:, j])
        if lam is not None:
            cond = np.abs(lam - sig[j]).max() / np.abs(lam - sig[j]).min()
            err = np.linalg.norm(x[:, j] - xs) / np.linalg.norm(xs)
            assert err <= cond * 4 * tol, (j, err, cond)


def test_batch_unconverged_is_reported(session):
    """an iteration cap far below what the systems need: every system is
    reported unconverged with its (finite) residual"""
    rp, c, v, sig, b, x, iters, rel, iflag = _run("HONEYCOMB-24-S4-W1", 6, 4, 0, max_iter=20, check=10)
    assert iflag == 6
    assert np.isfinite(rel).all() and (rel > 1e-10).all()
    assert (iters <= 30).all()


def test_batch_no_systems(session):
    *_, iflag = _run("HONEYCOMB-8-S4-W1", 0, 4, 0)
    assert iflag == 0


@pytest.mark.parametrize("mixed", [0, 1])
def test_batch_graph_replay_is_bitwise_identical(session, mixed):
    """the iteration replayed as a CUDA graph and launched kernel by kernel
    give the same iterates bit for bit (refills re-record the graph: 9
    systems through 4 slots)"""
    from phist_b200 import kernels as K
    K.chk(K.phist_b200_set_graphs, 0)
    try:
        *_, x0, it0, rel0, f0 = _run("HONEYCOMB-16x12-S2-W1", 9, 4, mixed)
    finally:
        K.chk(K.phist_b200_set_graphs, 1)
    *_, x1, it1, rel1, f1 = _run("HONEYCOMB-16x12-S2-W1", 9, 4, mixed)
    assert f0 == f1 == 0
    np.testing.assert_array_equal(it0, it1)
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_array_equal(rel0, rel1)


@pytest.mark.parametrize("mixed", [0, 1])
def test_block_tuner_and_auto_block(session, mixed):
    """the slot-count tuner times widths 1..min(32, nsys) and picks one of
    them; block <= 0 solves with that count and gives the same bits as
    passing the count explicitly"""
    import ctypes as ct

    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import SparseMat
    rp, c, v = G.problem("HONEYCOMB-16x12-S2-W1")
    A = SparseMat.from_crs(rp, c, v)
    nsys = 6
    blk = ct.c_int()
    us = np.zeros(6)
    K.chk(K.phist_b200_DcarpCG_tune_block, A.h, nsys, mixed, 2, ct.byref(blk), K.ptr(us))
    A.delete()
    assert blk.value in (1, 2, 4)
    assert (us[:3] > 0).all() and (us[3:] == 0).all()
    *_, x0, it0, rel0, f0 = _run("HONEYCOMB-16x12-S2-W1", nsys, 0, mixed)
    *_, x1, it1, rel1, f1 = _run("HONEYCOMB-16x12-S2-W1", nsys, blk.value, mixed)
    assert f0 == f1 == 0
    np.testing.assert_array_equal(it0, it1)
    np.testing.assert_array_equal(x0, x1)


def test_batch_iterates_match_oracle_cgmn(session, oracle):
    """iterate-level parity: after exactly 25 CGMN iterations (all systems in
    slots at once, cap reached, nothing refilled) the batched solver's
    iterates equal the numpy restatement of PHIST's recurrence
    (oracle.carp_cgmn) over the same colour order"""
    import ctypes as ct

    from conftest import relerr
    from phist_b200 import generators as G
    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat
    from test_carp_gpu import _order
    rp, c, v = G.problem("HONEYCOMB-10-S3-W1")
    n = len(rp) - 1
    A = SparseMat.from_crs(rp, c, v)
    sig = np.array([-4.0, 4.2, -3.8, 4.6])
    nsys, iters = len(sig), 25
    b = G.random_block(n, nsys, 9)
    work = ct.c_void_p()
    one = np.zeros(1)
    K.chk(K.phist_Dcarp_setup, A.h, 1, K.sptr(one, np.float64), ct.byref(work))
    rows, _ = _order(work, n)
    K.chk(K.phist_Dcarp_destroy, A.h, work)
    B = Mvec(A.row_map, nsys).set(b)
    X = Mvec(A.row_map, nsys)
    it = np.zeros(nsys, np.int32)
    rel = np.zeros(nsys)
    iflag = K.iflag_of(K.phist_b200_DcarpCG_batch, A.h, nsys, K.ptr(sig), B.h, X.h, nsys, 1e-30, iters, iters, 0,
                       1e-5, K.ptr(it), K.ptr(rel))
    x = X.get()
    for o in (B, X, A):
        o.delete()
    assert iflag == nsys and (it == iters).all()
    ref = oracle.carp_cgmn(rp, c, v, sig, b, iters, order=rows)
    assert relerr(x, ref) < 1e-10, relerr(x, ref)
