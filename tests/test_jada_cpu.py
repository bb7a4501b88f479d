"""PHIST's unchanged subspacejada on the CPU backend (oracle/cpu_backend.cpp,
a restatement of the builtin kernel library on the host cores): the CPU
reference of the eigen-solves.

* CPU only: on the 7-point Laplacian the converged eigenvalues equal the
  closed form sum_d (2 - 2 cos(k_d pi / (L + 1))) to 1e-10, and every
  explicit residual is below 1e-10.
* GPU: the same driver arguments on the GPU library (phist_b200/lib/jada_run)
  find the same eigenvalues to 1e-10 (times the spectral radius) with outer
  iteration counts within 10 % -- the solver-level parity of the drop-in.
"""
import itertools
import os

import numpy as np
import pytest

from conftest import ROOT

JADA_GPU = os.path.join(ROOT, "phist_b200", "lib", "jada_run")


def _need_cpu(oracle):
    if not os.path.exists(oracle.JADA_CPU):
        pytest.skip("CPU solver build (oracle/_ref/jada_run_cpu) not present")


def _exact_laplace(L, k):
    t = 2 - 2 * np.cos(np.arange(1, L + 1) * np.pi / (L + 1))
    ev = sorted(a + b + c for a, b, c in itertools.product(t[:6], t[:6], t[:6]))
    return np.array(ev[:k])


ARGS = ["numEigs=10", "blockSize=4", "minBas=20", "maxBas=40", "convTol=1e-10", "which=SR", "seed=0"]


def test_cpu_backend_laplace(oracle):
    _need_cpu(oracle)
    L = 16
    d = oracle.jada_cpu(["LAPLACE3D-%d" % L] + ARGS, threads=4)
    assert d["nConv"] == 10
    ev = np.sort(np.array(d["ev"][:10]))
    assert np.abs(ev - _exact_laplace(L, 10)).max() < 1e-10 * 12
    assert max(d["resExplicit"][:10]) < 1e-10


@pytest.mark.gpu
# the random diagonal separates the Laplacian's multiple eigenvalues: with
# threefold ones (LAPLACE3D at small L) which copy converges first depends on
# rounding and the outer iteration counts spread more; the benchmark problem
# LAPLACE3D-64 is held to the 10 % bound as well
@pytest.mark.parametrize("prob", ["LAPDIAG3D-24-S1", "LAPDIAG3D-20-S5", "LAPLACE3D-64"])
def test_gpu_and_cpu_solves_agree(oracle, prob):
    import json
    import subprocess
    _need_cpu(oracle)
    if not os.path.exists(JADA_GPU):
        pytest.skip("GPU drivers not built")
    cpu = oracle.jada_cpu([prob] + ARGS)
    r = subprocess.run([JADA_GPU, prob] + ARGS, capture_output=True, text=True, timeout=600)
    gpu = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert cpu["nConv"] == gpu["nConv"] == 10
    ec = np.sort(np.array(cpu["ev"][:10]))
    eg = np.sort(np.array(gpu["ev"][:10]))
    assert np.abs(ec - eg).max() < 1e-10 * 12
    assert max(gpu["resExplicit"][:10]) < 1e-10 and max(cpu["resExplicit"][:10]) < 1e-10
    assert abs(gpu["nIter"] - cpu["nIter"]) <= max(1, 0.1 * cpu["nIter"])
