"""PHIST's own CARP-CG solver (carp_cgState_create/reset/iterate,
src/krylov/phist_carp_cg_def.hpp), compiled unchanged from the PHIST sources
into phist_b200/lib/ and driven by phist_b200/solvers/carp_run.cpp, on the
b200 kernel library: shifted indefinite systems (A - sigma_j I) x_j = b_j of
the honeycomb tight-binding matrix, one shift and right-hand side per column.

Checked independently of the library: the solutions written by the driver
are put into the shifted systems with numpy (CRS arrays of the generator
mirror) and compared with dense solves.  PHIST's CARP-CG stops when the
explicit residual ||b - (A - sigma I) x|| falls below tol*||b||
(phist_carp_cg_def.hpp:548-566)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
RUNNER = os.path.join(ROOT, "phist_b200", "lib", "carp_run")


def run(problem, *kv, timeout=600):
    if not os.path.exists(RUNNER):
        pytest.skip("PHIST solver layers not built (phist_b200/solvers/Makefile)")
    out = subprocess.run([RUNNER, problem] + list(kv), capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def crs_matvec(rp, c, v, x):
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    y = np.zeros_like(x)
    np.add.at(y, rows, v[:, None] * x[c])
    return y


# One system per CARP-CG state.  With several columns per state PHIST keeps
# iterating converged columns with alpha = (1-conv)*(r'r/p'q)
# (phist_carp_cg_def.hpp:525); their search direction can cancel to exactly
# zero, and 0*(x/0) turns the column into NaN.  That is PHIST's own
# arithmetic, reproduced here in a host replay of its loop over this library.
@pytest.mark.parametrize("nshifts,block", [(4, 1), (3, 1)])
def test_carp_cg_honeycomb_shifts(session, tmp_path, nshifts, block):
    from phist_b200.generators import honeycomb, unif
    L, seed, tol = 24, 4, 1e-10
    out = str(tmp_path / "x.bin")
    r = run("HONEYCOMB-%d-S%d-W1" % (L, seed), "nshifts=%d" % nshifts, "block=%d" % block,
            "tol=%g" % tol, "maxIter=40000", "seed=%d" % seed, "out=" + out)
    rp, c, v = honeycomb(L, L, seed)
    n = len(rp) - 1
    assert r["n"] == n and r["nconv"] == nshifts
    shifts = 2.5 * unif(seed, np.arange(nshifts, dtype=np.uint64))
    np.testing.assert_array_equal(np.asarray(r["shifts"]), shifts)
    b = np.stack([unif(seed + 1 + j, np.arange(n, dtype=np.uint64)) for j in range(nshifts)], 1)
    x = np.fromfile(out, dtype=np.float64).reshape(n, nshifts)
    res = b - (crs_matvec(rp, c, v, x) - shifts[None, :] * x)
    rel = np.linalg.norm(res, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 2 * tol, rel
    np.testing.assert_allclose(np.asarray(r["relres"]), rel, rtol=1e-3, atol=1e-14)
    # dense solves: the error is bounded by cond(A - sigma I) times the residual
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    np.add.at(A, (rows, c), v)
    lam = np.linalg.eigvalsh(A)
    for j in range(nshifts):
        xs = np.linalg.solve(A - shifts[j] * np.eye(n), b[:, j])
        cond = np.abs(lam - shifts[j]).max() / np.abs(lam - shifts[j]).min()
        err = np.linalg.norm(x[:, j] - xs) / np.linalg.norm(xs)
        assert err <= cond * 4 * tol, (j, err, cond)


def test_carp_cg_mixed_refinement(session, tmp_path):
    """FP32 CARP-CG sweeps inside FP64 iterative refinement reach the same
    FP64 relative residual as the all-FP64 solver"""
    from phist_b200.generators import honeycomb, unif
    L, seed, tol, ns = 24, 4, 1e-10, 4
    out = str(tmp_path / "x.bin")
    r = run("HONEYCOMB-%d-S%d-W1" % (L, seed), "nshifts=%d" % ns, "block=1", "tol=%g" % tol,
            "maxIter=40000", "seed=%d" % seed, "mixed=1", "innerTol=1e-5", "out=" + out)
    assert r["mixed"] == 1 and r["nconv"] == ns
    assert all(k >= 2 for k in r["refinements"])
    # corrections solved in FP64 once FP32 stopped paying: never more than all
    assert all(0 <= f <= k for f, k in zip(r["fp64_refinements"], r["refinements"]))
    rp, c, v = honeycomb(L, L, seed)
    n = len(rp) - 1
    shifts = 2.5 * unif(seed, np.arange(ns, dtype=np.uint64))
    b = np.stack([unif(seed + 1 + j, np.arange(n, dtype=np.uint64)) for j in range(ns)], 1)
    x = np.fromfile(out, dtype=np.float64).reshape(n, ns)
    res = b - (crs_matvec(rp, c, v, x) - shifts[None, :] * x)
    rel = np.linalg.norm(res, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 2 * tol, rel
