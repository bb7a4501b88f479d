"""The served form (phist_b200/solvers/serve_run.cpp): a Poisson stream of
eigen-solves (PHIST's unchanged subspacejada per request) served by a pool of
host threads, each driving its own lane of the library, so that several
solves are on the GPU at once.  Checked: every request converges (explicit
residual below 20*tol, the bar of PHIST's TestSubspaceJaDa), its eigenvalues
match the dense spectrum, solves really overlap, and each result is the same
served alone as in the mix."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
RUNNER = os.path.join(ROOT, "phist_b200", "lib", "serve_run")


def run(*kv, timeout=900):
    if not os.path.exists(RUNNER):
        pytest.skip("PHIST solver layers not built (phist_b200/solvers/Makefile)")
    out = subprocess.run([RUNNER] + list(kv), capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def lapdiag_eigs(L, seed, k):
    from phist_b200.generators import lapdiag3d
    rp, c, v = lapdiag3d(L, seed)
    n = len(rp) - 1
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    np.add.at(A, (rows, c), v)
    return np.linalg.eigvalsh(A)[:k], np.abs(np.linalg.eigvalsh(A)).max()


@pytest.mark.parametrize("mixed,devgmres", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_served_stream_matches_alone_and_spectrum(session, mixed, devgmres):
    tol = 1e-10
    common = ["nreq=6", "rate=500", "lmin=8", "lmax=12", "seed=5", "numEigs=6", "blockSize=2", "minBas=12",
              "maxBas=24", "tol=%g" % tol, "mixed=%d" % mixed, "devgmres=%d" % devgmres]
    mix = run(*(common + ["workers=3"]))
    assert mix["failed"] == 0 and mix["unconverged"] == 0
    assert mix["max_resExplicit"] < 20 * tol
    assert mix["max_concurrent"] >= 2 and mix["lanes"] >= 2
    reqs = {r["id"]: r for r in mix["requests"]}
    seed = 5
    for i, r in reqs.items():
        ev_exact, rho = lapdiag_eigs(r["L"], seed * 1000003 + i, 6)
        assert np.abs(np.asarray(r["ev"]) - ev_exact).max() <= tol * rho * 10, (i, r["ev"], ev_exact)
    for i in (0, 3):
        alone = run(*(common + ["workers=1", "only=%d" % i]))
        assert alone["requests"][0]["id"] == i
        np.testing.assert_array_equal(np.asarray(alone["requests"][0]["ev"]), np.asarray(reqs[i]["ev"]))
        assert alone["requests"][0]["nIter"] == reqs[i]["nIter"]
