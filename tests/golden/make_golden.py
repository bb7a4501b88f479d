"""Generate the golden fixtures in tests/golden/ from the PHIST source tree.

Run once, in a checkout that has the PHIST sources (the default location is
the PHIST_SRC environment variable, else /root/reference):

    python tests/golden/make_golden.py

What it writes (all small, committed):

* ``phist_testmats.npz`` -- the real-valued MatrixMarket test matrices of
  PHIST's kernel test suite (test/matrices/D*.mm), converted to 0-based CRS
  arrays in file order, named ``<name>_rowptr``, ``<name>_col``,
  ``<name>_val``, ``<name>_shape``.
* ``a2_precalc.npz`` -- the hard-coded result vectors of the known-answer
  test ``A2_precalc_result`` in test/kernels/SparseMatTest_def.hpp (real
  branch, n=25 with nvec 1 and 4): y = A x for A = Dsprandn25 and the input
  x(i,j) = i + j*n (0-based i), stored row-major as ``y_nv1`` / ``y_nv4``.

The fixtures are read by the tests; nothing at test time reads the PHIST
source tree.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MATS = ["speye25", "speye388", "spzero25", "spzero388", "sprandn25",
        "sprandn388", "sprandn_nodiag25", "sprandn_nodiag388", "spshift25",
        "spshift388", "symmMat20", "sprandsym163", "jadaTestMat512"]


def read_mm(path):
    """Read a real 'coordinate general|symmetric' MatrixMarket file into CRS.

    Entries keep their file order inside each row (a stable sort by row)."""
    with open(path) as f:
        header = f.readline().lower()
        symmetric = "symmetric" in header
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nz = (int(t) for t in line.split())
        rows, cols, vals = [], [], []
        for line in f:
            t = line.split()
            if not t:
                continue
            i, j, v = int(t[0]) - 1, int(t[1]) - 1, float(t[2])
            rows.append(i); cols.append(j); vals.append(v)
            if symmetric and i != j:
                rows.append(j); cols.append(i); vals.append(v)
    rows = np.asarray(rows, np.int64)
    order = np.argsort(rows, kind="stable")
    rowptr = np.zeros(nr + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    return (rowptr, np.asarray(cols, np.int32)[order],
            np.asarray(vals, np.float64)[order], (nr, nc))


def parse_precalc(src):
    """Pull the two real-valued precalc_result arrays out of the test source."""
    lines = open(src).read().splitlines()
    out = {}
    for nv in (1, 4):
        cond = "#if _N_ == 25 && _NV_ == %d" % nv if nv == 1 else \
               "#elif _N_ == 25 && _NV_ == %d" % nv
        start = next(i for i, l in enumerate(lines) if l.strip() == cond)
        # the real branch follows the '#else' after the complex block
        k = start
        while lines[k].strip() != "#else":
            k += 1
        body = []
        k += 1
        assert "precalc_result" in lines[k]
        k += 1
        while "};" not in lines[k]:
            body.append(lines[k])
            k += 1
        body.append(lines[k].split("}")[0])
        nums = re.findall(r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?", " ".join(body))
        y = np.array([float(s) for s in nums])
        assert y.size == 25 * nv, (nv, y.size)
        out["y_nv%d" % nv] = y.reshape(25, nv)
    return out


def main():
    src = os.environ.get("PHIST_SRC", "/root/reference")
    if not os.path.isdir(src):
        sys.exit("PHIST sources not found at %s" % src)
    arrs = {}
    for m in MATS:
        rp, ci, va, shape = read_mm(os.path.join(src, "test", "matrices", "D%s.mm" % m))
        arrs[m + "_rowptr"] = rp
        arrs[m + "_col"] = ci
        arrs[m + "_val"] = va
        arrs[m + "_shape"] = np.asarray(shape, np.int64)
    np.savez_compressed(os.path.join(HERE, "phist_testmats.npz"), **arrs)
    pre = parse_precalc(os.path.join(src, "test", "kernels", "SparseMatTest_def.hpp"))
    np.savez_compressed(os.path.join(HERE, "a2_precalc.npz"), **pre)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
