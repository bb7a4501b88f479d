"""pytest configuration: the `gpu` marker, shared fixtures and paths.

Tests marked `gpu` need a CUDA device (a B200); everything else runs on the
CPU: the oracle against PHIST's golden vectors and PHIST's own C kernels, the
generators, and the C ABI symbol table of the built library.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib_built():
    from phist_b200 import build
    build.build()
    return True


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def session(lib_built):
    if not have_gpu():
        pytest.skip("no CUDA device")
    from phist_b200.objects import Session
    return Session.get()


@pytest.fixture(scope="session")
def testmats():
    g = np.load(os.path.join(GOLDEN, "phist_testmats.npz"))
    names = sorted({k.rsplit("_", 1)[0] for k in g.files})

    def get(name):
        rp, c, v = g[name + "_rowptr"], g[name + "_col"], g[name + "_val"]
        shape = tuple(g[name + "_shape"])
        return sort_rows(rp, c, v) + (shape,)
    get.names = names
    return get


def sort_rows(rp, col, val):
    """stable sort of the column indices inside each row (the order PHIST's
    builtin library stores, crsmat_module.F90:484-516)"""
    col = col.copy()
    val = val.copy()
    for i in range(len(rp) - 1):
        a, b = rp[i], rp[i + 1]
        o = np.argsort(col[a:b], kind="stable")
        col[a:b] = col[a:b][o]
        val[a:b] = val[a:b][o]
    return rp, col, val


def relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
