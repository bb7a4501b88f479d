"""PHIST's own block Jacobi-Davidson (subspacejada), compiled unchanged from
the PHIST sources into oracle/_ref/ (oracle/solvers/Makefile), running on the
b200 kernel library: the drop-in boundary exercised by the reference's own
caller.  Checked against the closed-form spectrum of the Dirichlet 7-point
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
RUNNER = os.path.join(ROOT, "oracle", "_ref", "jada_run")


def laplace_eigs(L, k):
    t = 2.0 - 2.0 * np.cos(np.arange(1, L + 1) * np.pi / (L + 1))
    ev = (t[:, None, None] + t[None, :, None] + t[None, None, :]).ravel()
    return np.sort(ev)[:k]


def run(problem, *kv, timeout=600):
    if not os.path.exists(RUNNER):
        pytest.skip("PHIST solver layers not built (oracle/solvers/Makefile)")
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
