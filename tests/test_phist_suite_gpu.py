"""PHIST's own test suites, run unchanged against this library.

tests/phist_suite/Makefile compiles the kernel conformance tests of the
PHIST sources (test/kernels/*.cpp with PHIST's vendored googletest) and
links them against libphist_kernels_b200.so; a second executable holds
PHIST's tests of the layers above the kernels (test/core, krylov, jada,
precon), run on PHIST's solver code compiled against this library.  The
executables are built by the package build when the PHIST sources are
present and travel with the built libraries.  The suite reads its test matrices from the working
directory by name (test/tools/MatrixIO_def.hpp: D<name>.mm, S<name>.mm);
they are written here from the golden fixture tests/golden/phist_testmats.npz
(PHIST's test/matrices converted by tests/golden/make_golden.py), single
precision as the shortest decimal of the float32 value.

Every test the suite runs must pass, except the cases listed in KNOWN with
the reason each cannot.  A test that ends the process (a crash) counts as a
failure; the runner records it and starts the tests not yet run again.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tests", "phist_suite", "_build")
EXE = os.path.join(BUILD, "phist_kernels_suite")
SOLVER_EXE = os.path.join(BUILD, "phist_solver_suite")

# test (a regular expression over "Case.test") -> why it cannot pass against
# this library
KNOWN = {
    r"[DS]SparseMatTest\w*_spshift_\d+_\d+\.shift_mvec":
        "fills the host view of an mvec and reads one back with no mvec_to_device / "
        "mvec_from_device between them (test/kernels/SparseMatTest_def.hpp:694-731); "
        "an mvec kept in device memory sees neither write, as with GHOST's CUDA build",
    r"DSparseMatTest_BENCH3D_8_A1_\d+_\d+\.(compare_with_rowFunc|fromRowFuncAndContext)":
        "calls PHIST's Fortran row function MATPDE3D_rowFunc "
        "(drivers/matfuncs/matpde3d.F90); no Fortran compiler is installed, so "
        "suite_shim.cpp's stand-in returns an error",
}


# the same for PHIST's tests of the layers above the kernels
KNOWN_SOLVER = {}


def _known(t, known=KNOWN):
    return any(re.fullmatch(k, t) for k in known)


def _write_matrices(d):
    g = np.load(os.path.join(GOLDEN, "phist_testmats.npz"))
    names = sorted({k.rsplit("_", 1)[0] for k in g.files})
    for nm in names:
        rp, c, v = g[nm + "_rowptr"], g[nm + "_col"], g[nm + "_val"]
        n, m = (int(x) for x in g[nm + "_shape"])
        rows = np.repeat(np.arange(n), np.diff(rp))
        for pre, fmt in (("D", lambda x: repr(float(x))), ("S", lambda x: repr(float(np.float32(x))))):
            with open(os.path.join(d, "%s%s.mm" % (pre, nm)), "w") as f:
                f.write("%%%%MatrixMarket matrix coordinate real general\n%d %d %d\n" % (n, m, len(c)))
                for i, j, x in zip(rows, c, v):
                    f.write("%d %d %s\n" % (i + 1, j + 1, fmt(x)))


def _list_tests(exe):
    out = subprocess.run([exe, "--gtest_list_tests"], capture_output=True, text=True, timeout=300).stdout
    tests, case = [], None
    for line in out.splitlines():
        if not line.strip() or line.startswith("["):
            continue
        if not line.startswith(" "):
            case = line.split("#")[0].strip()
        elif case:
            tests.append(case + line.split("#")[0].strip())
    return tests


def run_suite(d, log=None, exe=EXE):
    """runs the suite exe in directory d; a test that ends the process is
    recorded and the tests not yet run are started again.  Returns
    ({test: "ok" | "failed" | "crashed" | "not run"}, number of runs)"""
    _write_matrices(d)
    tests = [t for t in _list_tests(exe) if ".DISABLED_" not in t and not t.startswith("DISABLED_")]
    cases = {}
    for t in tests:
        cases.setdefault(t.split(".", 1)[0], []).append(t)
    result, runs = {}, 0
    while runs < 40:
        # test cases not finished yet, without the tests that ended a run
        todo = [c for c, ts in cases.items() if any(t not in result for t in ts)]
        if not todo:
            break
        crashed = [t for t, v in result.items() if v == "crashed"]
        filt = ":".join(c + ".*" for c in todo) + ("-" + ":".join(crashed) if crashed else "")
        runs += 1
        out = os.path.join(d, "run%d.txt" % runs)
        with open(out, "w") as f:
            r = subprocess.run(["stdbuf", "-oL", "-eL", exe, "--gtest_filter=" + filt], cwd=d, stdout=f,
                               stderr=subprocess.STDOUT, timeout=2400)
        last = None
        for line in open(out, errors="replace"):
            if line.startswith("[ RUN      ] "):
                last = line[13:].strip()
            elif line.startswith("[       OK ] ") and line.rstrip().endswith("ms)"):
                result[line[13:].rsplit(" (", 1)[0].strip()] = "ok"
            elif line.startswith("[  FAILED  ] ") and line.rstrip().endswith("ms)"):
                result[line[13:].rsplit(" (", 1)[0].strip()] = "failed"
        if log:
            log("run %d: rc %d, %d results" % (runs, r.returncode, len(result)))
        if r.returncode in (0, 1) or last is None or last in result:
            break  # ended normally (1: some tests failed), or outside a test
        result[last] = "crashed"
    for t in tests:
        result.setdefault(t, "not run")
    return result, runs


def _check(tmp_path, exe, known, min_ran):
    if not os.path.exists(exe):
        pytest.skip("PHIST's test suites are not built (they need the PHIST sources at build time)")
    result, runs = run_suite(str(tmp_path), exe=exe)
    ran = sum(v != "not run" for v in result.values())
    bad = sorted(t for t, v in result.items() if v != "ok" and not _known(t, known))
    assert ran > min_ran, "only %d tests ran" % ran
    assert not bad, "%d of %d PHIST tests failed or crashed: %s" % (
        len(bad), ran, ", ".join("%s (%s)" % (t, result[t]) for t in bad[:40]))


def test_phist_kernel_suite(tmp_path):
    _check(tmp_path, EXE, KNOWN, 1000)


def test_phist_solver_suite(tmp_path):
    _check(tmp_path, SOLVER_EXE, KNOWN_SOLVER, 300)
