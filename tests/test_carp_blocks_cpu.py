"""Block-coloured CARP sweep: the host-side layout and the kernel's schedule,
on the CPU.

tests/carp_blocks_emu.cpp builds the row blocks, their colouring, steps and
device arrays with the library's own host code (phist_b200/csrc/
pb_carp_blocks.hpp) and runs the sweep kernel's schedule (X copied in
16-byte pieces or element by element) on the host with every copy and
index checked against the array or shared-memory region it addresses
(blocks of one launch with disjoint footprints, rows of one step touching
disjoint slots).  The result must equal the oracle's sequential
Kaczmarz sweep (kacz_sub_def.h formulae) over the reported row order to
1e-13 (the oracle forms row norms and sums in its own order), and every
segment of that order must be a distance-2 independent set -- the facts the
GPU sweep relies on (tests/test_carp_gpu.py checks the GPU result against
the same oracle).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, relerr

SRC = os.path.join(ROOT, "tests", "carp_blocks_emu.cpp")


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    d = tmp_path_factory.mktemp("carp_emu")
    exe = str(d / "carp_blocks_emu")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-o", exe, SRC], check=True)
    k = [0]

    def run(rp, col, val, shifts, omega, b, x0, max_rows=128, max_fp=256, max_nnz=2048, wide=1):
        k[0] += 1
        fin, fout = str(d / f"in{k[0]}"), str(d / f"out{k[0]}")
        n, nv = x0.shape
        with open(fin, "wb") as f:
            np.array([n, len(col), nv, b is not None], np.int64).tofile(f)
            np.asarray(rp, np.int64).tofile(f)
            np.asarray(col, np.int32).tofile(f)
            np.asarray(val, np.float64).tofile(f)
            np.asarray(shifts, np.float64).tofile(f)
            np.asarray(omega, np.float64).tofile(f)
            if b is not None:
                np.ascontiguousarray(b, np.float64).tofile(f)
            np.ascontiguousarray(x0, np.float64).tofile(f)
        r = subprocess.run([exe, fin, fout, str(max_rows), str(max_fp), str(max_nnz), str(wide)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        raw = open(fout, "rb").read()
        ok, nseg = np.frombuffer(raw[:16], np.int64)
        if not ok:
            return None
        o = 16
        rows = np.frombuffer(raw[o:o + 4 * n], np.int32)
        o += 4 * n
        seg = np.frombuffer(raw[o:o + 8 * (nseg + 1)], np.int64)
        o += 8 * (nseg + 1)
        x = np.frombuffer(raw[o:o + 8 * n * nv], np.float64).reshape(n, nv)
        o += 8 * n * nv
        st = np.frombuffer(raw[o:o + 64], np.int64)
        stats = dict(zip(["nblocks", "ncolors", "max_fp", "max_rows", "seg_stride", "max_steps", "smem", "fp_total"],
                         st.tolist()))
        return rows, seg, x, stats
    return run


def _with_diagonal(rp, c):
    cols, prp = [], [0]
    for i in range(len(rp) - 1):
        row = list(c[rp[i]:rp[i + 1]])
        if i not in row:
            row.append(i)
        cols.extend(row)
        prp.append(len(cols))
    return np.array(prp, np.int64), np.array(cols, np.int32)


def _check(emu, oracle, rp, c, v, nvec, with_b=True, seed=0, **kw):
    n = len(rp) - 1
    rng = np.random.default_rng(seed)
    shifts = rng.uniform(-1, 1, nvec)
    omega = rng.uniform(0.8, 1.6, nvec)
    x0 = rng.uniform(-1, 1, (n, nvec))
    b = rng.uniform(-1, 1, (n, nvec)) if with_b else None
    out = emu(rp, c, v, shifts, omega, b, x0, **kw)
    assert out is not None
    rows, seg, x, stats = out
    assert np.array_equal(np.sort(rows), np.arange(n))
    colour = np.zeros(n, np.int32)
    for k in range(len(seg) - 1):
        colour[rows[seg[k]:seg[k + 1]]] = k
    prp, pcol = _with_diagonal(rp, c)
    assert oracle.check_dist2(prp, pcol, n, colour) == 0
    ref = oracle.carp_sweep(rp, c, v, shifts, b, x0, omega, order=rows)
    assert relerr(x, ref) < 1e-13
    return stats


@pytest.mark.parametrize("prob", ["sprandn388", "sprandn_nodiag388", "symmMat20", "spshift388", "jadaTestMat512",
                                  "spshift25", "speye25", "sprandsym163"])
@pytest.mark.parametrize("nvec", [1, 3, 8])
@pytest.mark.parametrize("wide", [1, 0])
def test_phist_testmats(emu, oracle, testmats, prob, nvec, wide):
    rp, c, v, shape = testmats(prob)
    _check(emu, oracle, rp, c, v, nvec, seed=nvec, wide=wide)


@pytest.mark.parametrize("nvec", [1, 8, 16, 32])
def test_honeycomb(emu, oracle, nvec):
    from phist_b200 import generators as G
    rp, c, v = G.honeycomb(48, 40, 3)
    st = _check(emu, oracle, rp, c, v, nvec, seed=nvec)
    # compact blocks: footprint within 1.5x the rows, few colours and steps
    assert st["fp_total"] < 1.5 * (len(rp) - 1)
    assert st["ncolors"] <= 8 and st["max_steps"] <= 8


def test_laplace3d_and_anderson(emu, oracle):
    from phist_b200 import generators as G
    for name in ("LAPLACE3D-14", "ANDERSON3D-12-S2"):
        rp, c, v = G.problem(name)
        _check(emu, oracle, rp, c, v, 4, seed=1)


def test_rhs_null_and_small_blocks(emu, oracle):
    """b = 0, and tiny block limits (many blocks, single-row blocks)"""
    from phist_b200 import generators as G
    rp, c, v = G.honeycomb(12, 10, 1)
    _check(emu, oracle, rp, c, v, 2, with_b=False)
    _check(emu, oracle, rp, c, v, 2, with_b=False, wide=0)
    _check(emu, oracle, rp, c, v, 2, max_rows=1, max_fp=4, max_nnz=4)
    _check(emu, oracle, rp, c, v, 5, max_rows=7, max_fp=12, max_nnz=40)


def test_long_rows_fall_back(emu):
    """a row with more pattern entries than a footprint may hold: no block
    layout (the library then uses the row colouring)"""
    n = 300
    rp = np.arange(n + 1, dtype=np.int64) * 1
    rp[1:] += n - 1   # row 0 dense
    col = np.concatenate([np.arange(n), np.arange(1, n)]).astype(np.int32)
    val = np.ones(len(col))
    x0 = np.zeros((n, 1))
    assert emu(rp, col, val, [0.5], [1.0], None, x0, max_rows=128, max_fp=256, max_nnz=2048) is None
