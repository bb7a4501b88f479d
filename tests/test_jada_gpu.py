"""PHIST's own block Jacobi-Davidson (subspacejada), compiled unchanged from
the PHIST sources into phist_b200/lib/ (phist_b200/solvers/Makefile), running
on the b200 kernel library: the drop-in boundary exercised by the reference's
own caller, in FP64 and in the mixed form (FP32 correction equations through
PHIST's user-defined inner-solver hook, pb_mixed_jada.h).  Checked against the closed-form spectrum of the Dirichlet 7-point
Laplacian on L^3: lambda = sum_d (2 - 2 cos(k_d pi / (L+1))), k_d = 1..L.
The reference's JaDa test accepts residuals below 20*tol
(test/jada/TestSubspaceJaDa_def.hpp:167); eigenvalues must match to 1e-10
relative to the spectral radius (12)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
RUNNER = os.path.join(ROOT, "phist_b200", "lib", "jada_run")


def laplace_eigs(L, k):
    t = 2.0 - 2.0 * np.cos(np.arange(1, L + 1) * np.pi / (L + 1))
    ev = (t[:, None, None] + t[None, :, None] + t[None, None, :]).ravel()
    return np.sort(ev)[:k]


def run(problem, *kv, timeout=600):
    if not os.path.exists(RUNNER):
        pytest.skip("PHIST solver layers not built (phist_b200/solvers/Makefile)")
    out = subprocess.run([RUNNER, problem] + list(kv), capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def check_spectrum(ev, L, nwant, tol=1e-10):
    """Every converged Ritz value is an exact eigenvalue (to tol relative to
    the spectral radius 12) and lies at the low end of the spectrum.  Block
    JaDa with locking may skip one copy of a multiple eigenvalue (the 7-point
    Laplacian has many threefold ones), so the smallest eigenvalue must be
    found and no converged value may lie above the (nwant+3)-th exact one."""
    exact = laplace_eigs(L, nwant + 6)
    ev = np.sort(np.asarray(ev))
    for lam in ev:
        assert np.abs(exact - lam).min() <= tol * 12.0, (lam, exact)
    assert abs(ev[0] - exact[0]) <= tol * 12.0
    assert ev[-1] <= exact[nwant + 2] + tol * 12.0


@pytest.mark.parametrize("L,sigma", [(12, 1), (16, 256)])
def test_subspacejada_laplace_small(session, L, sigma):
    tol = 1e-10
    r = run("LAPLACE3D-%d" % L, "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR", "sigma=%d" % sigma)
    assert r["nConv"] >= 10
    check_spectrum(r["ev"][:10], L, 10, tol)
    assert max(r["resExplicit"][:10]) < 20 * tol
    assert r["launches"] > 0


def test_subspacejada_config1_laplace64(session):
    """the FP64 drop-in configuration: 7-point Laplacian 64^3, 10 smallest
    eigenpairs, block size 4, minBase 20, maxBase 40, tol 1e-10, start vector
    uniform[-1,1] seed 0"""
    tol = 1e-10
    r = run("LAPLACE3D-64", "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR", "seed=0", timeout=1200)
    assert r["nConv"] >= 10
    check_spectrum(r["ev"][:10], 64, 10, tol)
    assert max(r["resExplicit"][:10]) < 20 * tol


@pytest.mark.parametrize("L", [12, 16])
def test_subspacejada_mixed_laplace_small(session, L):
    """FP32 correction equations, FP64 outer iteration on the Laplacian: every
    converged value is an exact eigenvalue at the low end of the spectrum, to
    the FP64 tolerance (which copies of the threefold eigenvalues are found
    may differ from the FP64 run, see check_spectrum)"""
    tol = 1e-10
    args = ["LAPLACE3D-%d" % L, "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR"]
    r32 = run(*(args + ["mixed=1"]))
    assert r32["mixed"] == 1 and r32["inner_calls"] > 0
    assert r32["nConv"] >= 10
    check_spectrum(r32["ev"][:10], L, 10, tol)
    assert max(r32["resExplicit"][:10]) < 20 * tol


def lapdiag_eigs(L, seed, k):
    """the k smallest eigenvalues and the spectral radius of the Laplacian
    plus random diagonal (dense eigvalsh of the generator's CRS arrays)"""
    from phist_b200.generators import lapdiag3d
    rp, c, v = lapdiag3d(L, seed)
    n = len(rp) - 1
    A = np.zeros((n, n))
    np.add.at(A, (np.repeat(np.arange(n), np.diff(rp)), c), v)
    lam = np.linalg.eigvalsh(A)
    return lam[:k], np.abs(lam).max()


@pytest.mark.parametrize("L", [12, 16])
def test_subspacejada_mixed_matches_fp64(session, L):
    """FP32 correction equations, FP64 outer iteration: the same eigenpairs
    to the same tolerance as the all-FP64 run, within a few more outer
    iterations.  The random diagonal separates the eigenvalues, so both runs
    must find exactly the 10 smallest."""
    tol, seed = 1e-10, 3
    args = ["LAPDIAG3D-%d-S%d" % (L, seed), "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR"]
    r64 = run(*args)
    r32 = run(*(args + ["mixed=1"]))
    assert r32["mixed"] == 1 and r32["inner_calls"] > 0
    assert r64["nConv"] >= 10 and r32["nConv"] >= 10
    exact, rho = lapdiag_eigs(L, seed, 10)
    for r in (r64, r32):
        assert np.abs(np.sort(r["ev"][:10]) - exact).max() <= tol * rho, (r["mixed"], r["ev"][:10], exact)
        assert max(r["resExplicit"][:10]) < 20 * tol
    assert np.abs(np.sort(r32["ev"][:10]) - np.sort(r64["ev"][:10])).max() <= tol * rho
    assert r32["nIter"] <= 1.5 * r64["nIter"] + 5


def anderson_spectrum(L, seed):
    """all eigenvalues of the periodic Anderson matrix (dense eigvalsh of the
    generator's CRS arrays)"""
    from phist_b200.generators import anderson3d
    rp, c, v = anderson3d(L, seed)
    n = len(rp) - 1
    A = np.zeros((n, n))
    for i in range(n):
        A[i, c[rp[i]:rp[i + 1]]] += v[rp[i]:rp[i + 1]]
    return np.linalg.eigvalsh(A)


@pytest.mark.parametrize("mixed", [0, 1])
def test_subspacejada_anderson(session, mixed):
    """8 smallest eigenpairs of a 3D Anderson matrix (L=10, disorder 16.5,
    simple spectrum) in FP64 and with FP32 correction equations: the
    converged values are the 8 smallest of the dense spectrum to tol
    relative to the spectral radius"""
    tol = 1e-10
    nev = 8
    r = run("ANDERSON3D-10-S3", "numEigs=%d" % nev, "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR", "seed=3", "maxIters=400", "mixed=%d" % mixed)
    assert r["nConv"] >= nev
    lam = anderson_spectrum(10, 3)
    rho = np.abs(lam).max()
    ev = np.sort(np.asarray(r["ev"][:nev]))
    assert np.abs(ev - lam[:nev]).max() <= tol * rho, (ev, lam[:nev])
    assert max(r["resExplicit"][:nev]) < 20 * tol


@pytest.mark.parametrize("L", [12, 16])
def test_subspacejada_device_gmres(session, L):
    """correction equations on the library's device-resident GMRES (FP64, and
    FP32 with mixed=1): the same 10 smallest eigenpairs to the same
    tolerance; FP64 within 10 % (+2) of the outer iterations of PHIST's own
    GMRES, FP32 within the mixed form's bound"""
    tol, seed = 1e-10, 3
    args = ["LAPDIAG3D-%d-S%d" % (L, seed), "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR"]
    r64 = run(*args)
    rd = run(*(args + ["devgmres=1"]))
    rm = run(*(args + ["devgmres=1", "mixed=1"]))
    exact, rho = lapdiag_eigs(L, seed, 10)
    for r in (rd, rm):
        assert r["devgmres"] == 1 and r["inner_calls"] > 0
        assert r["nConv"] >= 10
        assert np.abs(np.sort(r["ev"][:10]) - exact).max() <= tol * rho, (r["mixed"], r["ev"][:10], exact)
        assert max(r["resExplicit"][:10]) < 20 * tol
    assert rd["nIter"] <= 1.1 * r64["nIter"] + 2, (rd["nIter"], r64["nIter"])
    assert rm["nIter"] <= 1.5 * r64["nIter"] + 5, (rm["nIter"], r64["nIter"])


@pytest.mark.parametrize("L", [12, 16])
def test_subspacejada_device_minres(session, L):
    """innerSolvType=MINRES with the device solver: the correction equations
    on the library's device MINRES (FP64, and FP32 with mixed=1); the same 10
    smallest eigenpairs of the symmetric problem to the same tolerance, FP64
    within 10 % (+2) of the outer iterations of PHIST's own MINRES (host
    Lanczos on this library's kernels)"""
    tol, seed = 1e-10, 3
    args = ["LAPDIAG3D-%d-S%d" % (L, seed), "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40",
            "convTol=%g" % tol, "which=SR", "innerSolvType=MINRES"]
    rp = run(*args)
    rd = run(*(args + ["devgmres=1"]))
    rm = run(*(args + ["devgmres=1", "mixed=1"]))
    exact, rho = lapdiag_eigs(L, seed, 10)
    for r in (rp, rd, rm):
        assert r["nConv"] >= 10
        assert np.abs(np.sort(r["ev"][:10]) - exact).max() <= tol * rho, (r["mixed"], r["ev"][:10], exact)
        assert max(r["resExplicit"][:10]) < 20 * tol
    for r in (rd, rm):
        assert r["devgmres"] == 1 and r["inner_calls"] > 0
    assert rd["nIter"] <= 1.1 * rp["nIter"] + 2, (rd["nIter"], rp["nIter"])
    assert rm["nIter"] <= 1.5 * rp["nIter"] + 5, (rm["nIter"], rp["nIter"])
