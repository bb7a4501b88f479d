"""Seeded synthetic problems as CRS arrays (numpy), identical to the row
functions of csrc/pb_matfuncs.cu (same counter-based random numbers, same
lexicographic ordering, columns ascending inside each row).

These build the test and benchmark inputs quickly on the host; the tests check
that they agree bit for bit with the library's own row functions.
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z):
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def unif(seed, idx):
    """uniform [-1,1) numbers of pb_unif(seed, idx) in pb_blas.cuh"""
    idx = np.asarray(idx, np.uint64)
    with np.errstate(over="ignore"):
        h = _mix64(np.uint64(seed) * np.uint64(0x632BE59BD9B4E019) + _mix64(idx))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0


def _site_rand(seed, lo, hi, n):
    if hi == lo:
        return np.full(n, lo)
    u = (unif(seed, np.arange(n, dtype=np.uint64)) + 1.0) * 0.5
    return lo + (hi - lo) * u


def _assemble(n, cols, vals):
    """cols/vals: (n, k) arrays with -1 marking absent entries; sort + merge."""
    order = np.argsort(np.where(cols < 0, np.iinfo(np.int64).max, cols), axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, 1)
    vals = np.take_along_axis(vals, order, 1)
    # merge duplicate columns (tiny periodic lattices)
    dup = np.zeros_like(cols, dtype=bool)
    dup[:, 1:] = (cols[:, 1:] == cols[:, :-1]) & (cols[:, 1:] >= 0)
    if dup.any():
        for i, j in zip(*np.nonzero(dup)):
            k = j - 1
            while dup[i, k]:
                k -= 1
            vals[i, k] += vals[i, j]
        cols = np.where(dup, -1, cols)
        order = np.argsort(np.where(cols < 0, np.iinfo(np.int64).max, cols), axis=1, kind="stable")
        cols = np.take_along_axis(cols, order, 1)
        vals = np.take_along_axis(vals, order, 1)
    mask = cols >= 0
    rowptr = np.zeros(n + 1, np.int64)
    rowptr[1:] = np.cumsum(mask.sum(1))
    return rowptr, cols[mask].astype(np.int32), vals[mask]


def stencil3d(L, periodic, diag0, lo, hi, seed):
    n = L ** 3
    i = np.arange(n, dtype=np.int64)
    x, y, z = i % L, (i // L) % L, i // (L * L)
    cols, vals = [], []
    for coord, stride in ((x, 1), (y, L), (z, L * L)):
        for s in (-1, 1):
            xn = coord + s
            if periodic:
                xn = (xn + L) % L
                ok = xn != coord
            else:
                ok = (xn >= 0) & (xn < L)
            c = np.where(ok, i + (xn - coord) * stride, -1)
            cols.append(c)
            vals.append(np.where(ok, -1.0, 0.0))
    cols.append(i)
    vals.append(diag0 + _site_rand(seed, lo, hi, n))
    return _assemble(n, np.stack(cols, 1), np.stack(vals, 1))


def laplace3d(L):
    """7-point Laplacian on L^3, Dirichlet: diag 6, off-diagonals -1"""
    return stencil3d(L, False, 6.0, 0.0, 0.0, 0)


def lapdiag3d(L, seed):
    """Laplacian + uniform[0,1] random diagonal"""
    return stencil3d(L, False, 6.0, 0.0, 1.0, seed)


def anderson3d(L, seed, W=16.5):
    """periodic 3D Anderson model: hopping -1, on-site uniform[-W/2, W/2]"""
    return stencil3d(L, True, 0.0, -W / 2, W / 2, seed)


def honeycomb(Lx, Ly, seed, W=1.0):
    """honeycomb lattice, 2 sites per cell, periodic, hopping -1,
    on-site uniform[-W/2, W/2]"""
    n = 2 * Lx * Ly
    i = np.arange(n, dtype=np.int64)
    cell, s = i // 2, i % 2
    x, y = cell % Lx, cell // Lx

    def site(xx, yy, ss):
        return 2 * ((xx % Lx) + Lx * (yy % Ly)) + ss

    c1 = np.where(s == 0, site(x, y, 1), site(x, y, 0))
    c2 = np.where(s == 0, site(x - 1, y, 1), site(x + 1, y, 0))
    c3 = np.where(s == 0, site(x, y - 1, 1), site(x, y + 1, 0))
    cols = np.stack([c1, c2, c3, i], 1)
    vals = np.stack([-np.ones(n), -np.ones(n), -np.ones(n), _site_rand(seed, -W / 2, W / 2, n)], 1)
    return _assemble(n, cols, vals)


def problem(name):
    """CRS arrays for a problem string of phist_b200_Dcreate_problem"""
    parts = name.split("-")
    kind = parts[0]
    opts = {p[0]: p[1:] for p in parts[2:]}
    seed = int(opts.get("S", 0))
    if kind == "LAPLACE3D":
        return laplace3d(int(parts[1]))
    if kind == "LAPDIAG3D":
        return lapdiag3d(int(parts[1]), seed)
    if kind == "ANDERSON3D":
        return anderson3d(int(parts[1]), seed, float(opts.get("W", 16.5)))
    if kind == "HONEYCOMB":
        dims = parts[1].split("x")
        lx = int(dims[0])
        ly = int(dims[1]) if len(dims) > 1 else lx
        return honeycomb(lx, ly, seed, float(opts.get("W", 1.0)))
    raise ValueError(name)


def random_block(n, m, seed, dtype=np.float64):
    """n x m block with entries uniform[-1,1) from the counter-based generator"""
    idx = np.arange(n * m, dtype=np.uint64)
    return unif(seed, idx).reshape(n, m).astype(dtype)
