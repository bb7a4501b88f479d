"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (this project's C restatement of PHIST's builtin
kernels, phist_oracle.c) and, when present, oracle/_ref/libref_builtin*.so
(PHIST's own C kernels compiled from the PHIST sources by oracle/Makefile).
Only the tests, the smoke check and bench.py's CPU-baseline leg use it; the
library under test never does.

All arrays are numpy; row-major block vectors (n x m, C order) and
column-major small matrices (Fortran order) as in PHIST.
"""
import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF = os.path.join(HERE, "_ref", "libref_builtin.so")
REF_PREC = os.path.join(HERE, "_ref", "libref_builtin_prec.so")


def build(with_ref=None):
    """make -C oracle [ref]; ref only when the PHIST source tree named by
    the PHIST_SRC environment variable is reachable"""
    targets = ["all"]
    src = os.environ.get("PHIST_SRC", "")
    if with_ref is None:
        with_ref = bool(src) and os.path.isdir(os.path.join(src, "src", "kernels", "builtin"))
    if with_ref:
        targets.append("ref")
    env = dict(os.environ, PHIST_SRC=src)
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)


JADA_CPU = os.path.join(HERE, "_ref", "jada_run_cpu")


def build_cpu():
    """make -C oracle cpu: PHIST's FP64 solver layers on the CPU backend
    (cpu_backend.cpp) and the jada_run driver, when the PHIST sources
    (PHIST_SRC) and the solver objects are present"""
    src = os.environ.get("PHIST_SRC", "")
    if not src or not os.path.isdir(os.path.join(src, "src", "jada")):
        return False
    from phist_b200.build import openblas_path
    env = dict(os.environ, PHIST_SRC=src, OPENBLAS=openblas_path() or "")
    subprocess.run(["make", "-s", "-C", HERE, "cpu"], check=True, env=env)
    return True


def jada_cpu(args, threads=None, timeout=600):
    """runs PHIST's subspacejada on the CPU backend (oracle/_ref/jada_run_cpu)
    with the driver arguments of phist_b200/lib/jada_run; returns its JSON"""
    import json
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([JADA_CPU] + list(args), capture_output=True, text=True, timeout=timeout, env=env)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        raise RuntimeError("jada_run_cpu failed (%d): %s" % (r.returncode, r.stderr[-500:]))
    return json.loads(lines[-1])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build(with_ref=False)
        _lib = ct.CDLL(LIB)
        i64, i32, d, vp = ct.c_int64, ct.c_int, ct.c_double, ct.c_void_p
        f = ct.c_float
        _lib.orc_spmmv.argtypes = [i64, vp, vp, vp, i32, d, vp, vp, i64, d, vp, i64]
        _lib.orc_sspmmv.argtypes = [i64, vp, vp, vp, i32, f, vp, vp, i64, f, vp, i64]
        _lib.orc_mvTmv.argtypes = [i64, i32, i32, d, vp, i64, vp, i64, d, vp, i64]
        _lib.orc_mvTmv_prec.argtypes = _lib.orc_mvTmv.argtypes
        _lib.orc_mvsd.argtypes = [i64, i32, i32, d, vp, i64, vp, i64, d, vp, i64]
        _lib.orc_mvsdi.argtypes = [i64, i32, i32, vp, i64, vp, i64]
        _lib.orc_mvsd_add_mvsd.argtypes = [i64, i32, i32, vp, i64, vp, i64, vp, i64, vp, i64]
        _lib.orc_fused_mvsd_mvTmv.argtypes = [i64, i32, i32, d, vp, i64, vp, i64, d, vp, i64, vp, i64]
        _lib.orc_fused_mvsdi_mvTmv.argtypes = [i64, i32, i32, i32, d, vp, i64, vp, i64, vp, i64, d, vp, i64]
        _lib.orc_dot.argtypes = [i64, i32, vp, i64, vp, i64, vp]
        _lib.orc_dot_prec.argtypes = _lib.orc_dot.argtypes
        _lib.orc_norm2.argtypes = [i64, i32, vp, i64, vp]
        _lib.orc_vadd.argtypes = [i64, i32, d, vp, vp, i64, d, vp, i64]
        _lib.orc_kacz_sweep.argtypes = [i64, vp, vp, vp, i32, vp, vp, i64, vp, i64, vp, vp, i64]
        _lib.orc_carp_sweep.argtypes = [i64, vp, vp, vp, i32, vp, vp, i64, vp, i64, vp]
        _lib.orc_sell_perm.argtypes = [i64, vp, i64, vp]
        _lib.orc_check_dist2.argtypes = [i64, vp, vp, i64, vp]
        _lib.orc_check_dist2.restype = i64
        _lib.orc_set_num_threads.argtypes = [i32]
        _lib.orc_num_threads.restype = i32
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def _rows(a):
    return a.shape[0]


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


def spmmv(rowptr, col, val, x, alpha=1.0, beta=0.0, y=None, shifts=None):
    """Y = alpha (A + diag(shifts)) X + beta Y (row-major X, Y)"""
    x = np.ascontiguousarray(x)
    n = len(rowptr) - 1
    nvec = x.shape[1]
    if y is None:
        y = np.zeros((n, nvec), x.dtype)
    else:
        y = np.array(y, dtype=x.dtype, order="C", copy=True)
    sh = None if shifts is None else np.ascontiguousarray(shifts, x.dtype)
    if x.dtype == np.float32:
        lib().orc_sspmmv(n, _p(rowptr), _p(col), _p(np.ascontiguousarray(val, np.float32)), nvec,
                         alpha, _p(sh), _p(x), nvec, beta, _p(y), nvec)
    else:
        lib().orc_spmmv(n, _p(rowptr), _p(col), _p(np.ascontiguousarray(val, np.float64)), nvec,
                        alpha, _p(sh), _p(x), nvec, beta, _p(y), nvec)
    return y


def mvTmv(V, W, alpha=1.0, beta=0.0, C=None, prec=False):
    V = np.ascontiguousarray(V, np.float64)
    W = np.ascontiguousarray(W, np.float64)
    m, k = V.shape[1], W.shape[1]
    C = np.zeros((m, k), order="F") if C is None else np.array(C, order="F", dtype=np.float64)
    f = lib().orc_mvTmv_prec if prec else lib().orc_mvTmv
    f(V.shape[0], m, k, alpha, _p(V), m, _p(W), k, beta, _p(C), m)
    return C


def mvsd(V, C, alpha=1.0, beta=0.0, W=None):
    V = np.ascontiguousarray(V, np.float64)
    C = np.asfortranarray(C, np.float64)
    n, m = V.shape
    k = C.shape[1]
    W = np.zeros((n, k)) if W is None else np.array(W, dtype=np.float64, order="C", copy=True)
    lib().orc_mvsd(n, m, k, alpha, _p(V), m, _p(C), m, beta, _p(W), k)
    return W


def mvsdi(V, M):
    V = np.array(V, dtype=np.float64, order="C", copy=True)
    M = np.asfortranarray(M, np.float64)
    n, m = V.shape
    lib().orc_mvsdi(n, m, M.shape[1], _p(V), m, _p(M), m)
    return V


def mvsd_add_mvsd(V, C, W, D):
    V = np.ascontiguousarray(V, np.float64)
    W = np.array(W, dtype=np.float64, order="C", copy=True)
    C = np.asfortranarray(C, np.float64)
    D = np.asfortranarray(D, np.float64)
    n, m = V.shape
    k = W.shape[1]
    lib().orc_mvsd_add_mvsd(n, m, k, _p(V), m, _p(C), m, _p(W), k, _p(D), k)
    return W


def fused_mvsd_mvTmv(V, C, W, alpha=1.0, beta=0.0):
    V = np.ascontiguousarray(V, np.float64)
    W = np.array(W, dtype=np.float64, order="C", copy=True)
    C = np.asfortranarray(C, np.float64)
    n, m = V.shape
    k = W.shape[1]
    G = np.zeros((k, k), order="F")
    lib().orc_fused_mvsd_mvTmv(n, m, k, alpha, _p(V), m, _p(C), m, beta, _p(W), k, _p(G), k)
    return W, G


def fused_mvsdi_mvTmv(V, W, C, alpha=1.0, beta=0.0, D=None):
    V = np.ascontiguousarray(V, np.float64)
    W = np.array(W, dtype=np.float64, order="C", copy=True)
    C = np.asfortranarray(C, np.float64)
    n, mv = V.shape
    m = W.shape[1]
    k = C.shape[1]
    D = np.zeros((mv, k), order="F") if D is None else np.array(D, order="F", dtype=np.float64)
    lib().orc_fused_mvsdi_mvTmv(n, mv, m, k, alpha, _p(V), mv, _p(W), m, _p(C), m, beta, _p(D), mv)
    return W[:, :k], D


def dot(V, W, prec=False):
    V = np.ascontiguousarray(V, np.float64)
    W = np.ascontiguousarray(W, np.float64)
    out = np.zeros(V.shape[1])
    f = lib().orc_dot_prec if prec else lib().orc_dot
    f(V.shape[0], V.shape[1], _p(V), V.shape[1], _p(W), W.shape[1], _p(out))
    return out


def kacz_sweep(rowptr, col, val, shifts, b, x, omega, order):
    x = np.array(x, dtype=np.float64, order="C", copy=True)
    nvec = x.shape[1]
    bb = None if b is None else np.ascontiguousarray(b, np.float64)
    order = np.ascontiguousarray(order, np.int32)
    lib().orc_kacz_sweep(len(rowptr) - 1, _p(rowptr), _p(col), _p(np.ascontiguousarray(val, np.float64)),
                         nvec, _p(np.ascontiguousarray(shifts, np.float64)), _p(bb), nvec, _p(x), nvec,
                         _p(np.ascontiguousarray(omega, np.float64)), _p(order), len(order))
    return x


def carp_sweep(rowptr, col, val, shifts, b, x, omega, order=None):
    """forward sweep over `order` (default 0..n-1), then backward over its reverse"""
    n = len(rowptr) - 1
    order = np.arange(n, dtype=np.int32) if order is None else np.asarray(order, np.int32)
    x = kacz_sweep(rowptr, col, val, shifts, b, x, omega, order)
    return kacz_sweep(rowptr, col, val, shifts, b, x, omega, order[::-1].copy())


def sell_perm(rowptr, sigma):
    n = len(rowptr) - 1
    perm = np.zeros(n, np.int32)
    lib().orc_sell_perm(n, _p(rowptr), sigma, _p(perm))
    return perm


def check_dist2(rowptr, col, ncols, color):
    color = np.ascontiguousarray(color, np.int32)
    return lib().orc_check_dist2(len(rowptr) - 1, _p(rowptr), _p(col), ncols, _p(color))


# ------------------------------------------------ PHIST's own C kernels
_ref = None
_refp = None


def ref_available():
    return os.path.exists(REF) and os.path.exists(REF_PREC)


def ref_libs():
    """(plain, prec) handles of PHIST's builtin C kernels compiled from source"""
    global _ref, _refp
    if _ref is None:
        _ref = ct.CDLL(REF)
        _refp = ct.CDLL(REF_PREC)
    return _ref, _refp


def ref_spmmv_nt(rowptr, col, val, x, alpha=1.0, shifts=None, prec=False):
    """PHIST's dspmvm_nt_<nvec>_c / dspmvm_nt_strided_<nvec>_c (beta = 0).

    The kernels take Fortran (1-based) row offsets and column indices, a
    separate halo offset (= row end with one process) and 16-byte aligned
    output."""
    plain, precl = ref_libs()
    L = precl if prec else plain
    n = len(rowptr) - 1
    nvec = x.shape[1]
    rp1 = np.ascontiguousarray(rowptr + 1, np.int64)
    halo = np.ascontiguousarray(rowptr[1:] + 1, np.int64)
    col1 = np.ascontiguousarray(col + 1, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    sh = np.zeros(nvec) if shifts is None else np.ascontiguousarray(shifts, np.float64)
    # 64-byte aligned buffers
    def aligned(shape):
        nb = int(np.prod(shape)) * 8
        raw = np.zeros(nb + 64, np.uint8)
        off = (-raw.ctypes.data) % 64
        return raw[off:off + nb].view(np.float64).reshape(shape)
    xa = aligned(x.shape)
    xa[...] = x
    ya = aligned((n, nvec))
    hal = np.zeros(8)
    d, i32 = ct.c_double, ct.c_int
    if nvec == 1:
        f = L.dspmvm_nt_1_c
        f.argtypes = [i32, d] + [ct.c_void_p] * 8
        f(n, alpha, _p(rp1), _p(halo), _p(col1), _p(val), _p(sh), _p(xa), _p(hal), _p(ya))
    else:
        f = getattr(L, "dspmvm_nt_strided_%d_c" % nvec)
        f.argtypes = [i32, d] + [ct.c_void_p] * 6 + [i32, ct.c_void_p, ct.c_void_p, i32]
        f(n, alpha, _p(rp1), _p(halo), _p(col1), _p(val), _p(sh), _p(xa), nvec, _p(hal), _p(ya), nvec)
    return np.array(ya)


def ref_spmmv_nt_runner(rowptr, col, val, x, alpha=1.0):
    """PHIST's dspmvm_nt_<nvec>_c / dspmvm_nt_strided_<nvec>_c (nvec 1, 2, 4,
    8; beta = 0) on buffers prepared once (1-based indices, 64-byte aligned
    vectors): returns (run, y), run() computing y = alpha A x again.  For
    timing the reference kernels without the set-up in the timed region."""
    plain, _ = ref_libs()
    n = len(rowptr) - 1
    nvec = x.shape[1]
    keep = {}
    keep["rp1"] = np.ascontiguousarray(rowptr + 1, np.int64)
    keep["halo"] = np.ascontiguousarray(rowptr[1:] + 1, np.int64)
    keep["col1"] = np.ascontiguousarray(col + 1, np.int32)
    keep["val"] = np.ascontiguousarray(val, np.float64)
    keep["sh"] = np.zeros(nvec)
    keep["hal"] = np.zeros(8)

    def aligned(shape):
        nb = int(np.prod(shape)) * 8
        raw = np.zeros(nb + 64, np.uint8)
        off = (-raw.ctypes.data) % 64
        keep.setdefault("raw", []).append(raw)
        return raw[off:off + nb].view(np.float64).reshape(shape)
    xa = aligned(x.shape)
    xa[...] = x
    ya = aligned((n, nvec))
    d, i32 = ct.c_double, ct.c_int
    if nvec == 1:
        f = plain.dspmvm_nt_1_c
        f.argtypes = [i32, d] + [ct.c_void_p] * 8
        args = (n, alpha, _p(keep["rp1"]), _p(keep["halo"]), _p(keep["col1"]), _p(keep["val"]), _p(keep["sh"]),
                _p(xa), _p(keep["hal"]), _p(ya))
    else:
        f = getattr(plain, "dspmvm_nt_strided_%d_c" % nvec)
        f.argtypes = [i32, d] + [ct.c_void_p] * 6 + [i32, ct.c_void_p, ct.c_void_p, i32]
        args = (n, alpha, _p(keep["rp1"]), _p(keep["halo"]), _p(keep["col1"]), _p(keep["val"]), _p(keep["sh"]),
                _p(xa), nvec, _p(keep["hal"]), _p(ya), nvec)

    def run():
        f(*args)
    run.keep = (keep, xa)  # the buffers live as long as run
    return run, ya


def ref_ddot_prec(x, y):
    """PHIST's compensated dot (ddot_prec_<nvec>, dot_kernels_prec.c), nvec 1|2|4"""
    _, precl = ref_libs()
    # the kernels assume the row count padded to a multiple of 4 with zeros
    pad = (-x.shape[0]) % 4
    x = np.vstack([x, np.zeros((pad, x.shape[1]))])
    y = np.vstack([y, np.zeros((pad, y.shape[1]))])
    n, nvec = x.shape
    res = np.zeros(nvec)
    resC = np.zeros(nvec)
    raw = [np.zeros(x.size * 8 + 64, np.uint8) for _ in range(2)]
    bufs = []
    for r, a in zip(raw, (x, y)):
        off = (-r.ctypes.data) % 64
        b = r[off:off + a.size * 8].view(np.float64).reshape(a.shape)
        b[...] = a
        bufs.append(b)
    f = getattr(precl, "ddot_prec_%d" % nvec)
    f.argtypes = [ct.c_int] + [ct.c_void_p] * 4
    f(n, _p(bufs[0]), _p(bufs[1]), _p(res), _p(resC))
    return res, resC


def ref_gemm_sc_prec(V, W):
    """PHIST's compensated V'W (dgemm_sc_prec_<m>_k, gemm_kernels_sC_prec.c)
    for V with m in {1, 2, 4} columns, W with k columns; returns the
    double-double result as its high and low parts (m x k each)"""
    _, precl = ref_libs()
    n, m = V.shape
    k = W.shape[1]
    assert m in (1, 2, 4)
    bufs = []
    for a in (V, W):
        raw = np.zeros(a.size * 8 + 64, np.uint8)
        off = (-raw.ctypes.data) % 64
        b = raw[off:off + a.size * 8].view(np.float64).reshape(a.shape)
        b[...] = a
        bufs.append((raw, b))
    res = np.zeros(m * k)
    resC = np.zeros(m * k)
    f = getattr(precl, "dgemm_sc_prec_%d_k" % m)
    f.argtypes = [ct.c_int, ct.c_int] + [ct.c_void_p] * 4
    f(n, k, _p(bufs[0][1]), _p(bufs[1][1]), _p(res), _p(resC))
    # res[j*m + r] holds the (r, j) entry
    return res.reshape(k, m).T.copy(), resC.reshape(k, m).T.copy()


def jada_gmres(A, Q, R, sigma, tol, max_iter, max_bas, res_index=None):
    """GMRES for the Jacobi-Davidson correction equations, restated in numpy
    from PHIST's blocked GMRES as jadaCorrectionSolver_run drives it
    (src/jada/phist_jadaCorrectionSolver_def.hpp:372-583,
    src/krylov/phist_blockedgmres_def.hpp): per system s, operator
    P (A - sigma_s I) with P = I - Q Q', x_0 = 0, Arnoldi (here Gram-Schmidt
    twice), Givens rotations, convergence when the residual estimate is below
    1000 eps or tol_s * ||b_s|| (blockedgmres_def.hpp:604-606), restart after
    max_bas steps, at most max_iter steps, the solutions scaled to unit norm.
    A: dense n x n.  Returns (t, converged flags)."""
    A = np.asarray(A, np.float64)
    n = A.shape[0]
    k = len(sigma)
    P = np.eye(n) - (Q @ Q.T if Q is not None and Q.shape[1] else 0.0)
    eps = 1000 * np.finfo(np.float64).eps
    T = np.zeros((n, k))
    conv = np.zeros(k, bool)
    m = max(1, min(max_bas if max_bas > 0 else max_iter, max_iter, 63))
    for s in range(k):
        b = R[:, res_index[s] if res_index is not None else s].astype(np.float64)
        op = P @ (A - sigma[s] * np.eye(n))
        x = np.zeros(n)
        bnorm = np.linalg.norm(b)
        done = bnorm < eps
        total = 0
        while total < max_iter and not done:
            r = b - op @ x
            beta = np.linalg.norm(r)
            V = np.zeros((n, m + 1))
            H = np.zeros((m + 1, m))
            cs, sn = np.zeros(m), np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            V[:, 0] = r / beta if beta > 0 else 0.0
            jc = 0
            for j in range(min(m, max_iter - total)):
                w = op @ V[:, j]
                for _ in range(2):
                    h = V[:, :j + 1].T @ w
                    w = w - V[:, :j + 1] @ h
                    H[:j + 1, j] += h
                hn = np.linalg.norm(w)
                V[:, j + 1] = w / hn if hn > 0 else 0.0
                for i in range(j):
                    a, bb = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * bb, -sn[i] * a + cs[i] * bb
                a = H[j, j]
                rr = np.hypot(a, hn)
                c, sg = (a / rr, hn / rr) if rr > 0 else (1.0, 0.0)
                cs[j], sn[j] = c, sg
                H[j, j] = rr
                g[j], g[j + 1] = c * g[j], -sg * g[j]
                jc = j + 1
                res = abs(g[j + 1])
                if res < eps or (bnorm > 0 and res / bnorm < tol[s]):
                    done = True
                    break
            y = np.zeros(jc)
            for i in range(jc - 1, -1, -1):
                y[i] = (g[i] - H[i, i + 1:jc] @ y[i + 1:jc]) / H[i, i] if H[i, i] != 0 else 0.0
            x = x + V[:, :jc] @ y
            total += jc
        nx = np.linalg.norm(x)
        T[:, s] = x / nx if nx > 0 else 0.0
        conv[s] = done
    return T, conv


def jada_minres(A, Q, R, sigma, tol, max_iter, max_bas, res_index=None):
    """MINRES for the Jacobi-Davidson correction equations, restated in numpy
    from PHIST's blocked MINRES as jadaCorrectionSolver_run drives it
    (src/jada/phist_jadaCorrectionSolver_def.hpp:499-503,
    src/krylov/phist_blockedminres_def.hpp:185-277): per system s, operator
    P (A - sigma_s I) with P = I - Q Q', x_0 = 0, the Lanczos recurrence
    w = op v_j, alpha = v_j'w, w -= alpha v_j, w -= beta v_{j-1} (beta the
    previous norm), beta' = ||w||, H tridiagonal; the basis kept, Givens
    rotations and least squares as in jada_gmres; convergence when the
    residual estimate is below 100 eps or tol_s * ||b_s||
    (blockedminres_def.hpp:157), restart after max_bas steps, at most
    max_iter steps, the solutions scaled to unit norm.  A: dense symmetric
    n x n.  Returns (t, converged flags)."""
    A = np.asarray(A, np.float64)
    n = A.shape[0]
    k = len(sigma)
    P = np.eye(n) - (Q @ Q.T if Q is not None and Q.shape[1] else 0.0)
    eps = 100 * np.finfo(np.float64).eps
    T = np.zeros((n, k))
    conv = np.zeros(k, bool)
    m = max(1, min(max_bas if max_bas > 0 else max_iter, max_iter, 63))
    for s in range(k):
        b = R[:, res_index[s] if res_index is not None else s].astype(np.float64)
        op = P @ (A - sigma[s] * np.eye(n))
        x = np.zeros(n)
        bnorm = np.linalg.norm(b)
        done = bnorm < eps
        total = 0
        while total < max_iter and not done:
            r = b - op @ x
            beta = np.linalg.norm(r)
            V = np.zeros((n, m + 1))
            H = np.zeros((m + 1, m))
            cs, sn = np.zeros(m), np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            V[:, 0] = r / beta if beta > 0 else 0.0
            jc = 0
            bprev = 0.0
            for j in range(min(m, max_iter - total)):
                w = op @ V[:, j]
                alpha = V[:, j] @ w
                w = w - alpha * V[:, j]
                if j > 0:
                    w = w - bprev * V[:, j - 1]
                    H[j - 1, j] = bprev
                H[j, j] = alpha
                hn = np.linalg.norm(w)
                bprev = hn
                V[:, j + 1] = w / hn if hn > 0 else 0.0
                for i in range(j):
                    a, bb = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * bb, -sn[i] * a + cs[i] * bb
                a = H[j, j]
                rr = np.hypot(a, hn)
                c, sg = (a / rr, hn / rr) if rr > 0 else (1.0, 0.0)
                cs[j], sn[j] = c, sg
                H[j, j] = rr
                g[j], g[j + 1] = c * g[j], -sg * g[j]
                jc = j + 1
                res = abs(g[j + 1])
                if res < eps or (bnorm > 0 and res / bnorm < tol[s]):
                    done = True
                    break
            y = np.zeros(jc)
            for i in range(jc - 1, -1, -1):
                y[i] = (g[i] - H[i, i + 1:jc] @ y[i + 1:jc]) / H[i, i] if H[i, i] != 0 else 0.0
            x = x + V[:, :jc] @ y
            total += jc
        nx = np.linalg.norm(x)
        T[:, s] = x / nx if nx > 0 else 0.0
        conv[s] = done
    return T, conv


def carp_cgmn(rowptr, col, val, sigma, b, iters, order=None):
    """CGMN (CARP-CG) for the shifted systems (A - sigma_j I) x_j = b_j, one
    per column, restated from PHIST's carp_cg
    (src/krylov/phist_carp_cg_def.hpp:440-690): CG on (I - Q) x = Q(0, b),
    Q(x, b) the forward-backward Kaczmarz sweep over `order` with relaxation
    1, x_0 = 0, `iters` iterations; per column
        r = Q(0, b), p = r
        q = p - Q(p, 0), alpha = r'r / p'q, x += alpha p, r -= alpha q,
        beta = r'r_new / r'r, p = r + beta p.
    Returns x (n x nsys)."""
    b = np.ascontiguousarray(b, np.float64)
    n, w = b.shape
    sig = np.asarray(sigma, np.float64)
    om = np.ones(w)
    x = np.zeros((n, w))
    r = carp_sweep(rowptr, col, val, sig, b, np.zeros((n, w)), om, order)
    p = r.copy()
    rr = (r * r).sum(axis=0)
    for _ in range(iters):
        q = p - carp_sweep(rowptr, col, val, sig, None, p.copy(), om, order)
        pq = (p * q).sum(axis=0)
        alpha = np.where(pq != 0, rr / np.where(pq != 0, pq, 1.0), 0.0)
        x += alpha * p
        r -= alpha * q
        rr_new = (r * r).sum(axis=0)
        beta = np.where(rr != 0, rr_new / np.where(rr != 0, rr, 1.0), 0.0)
        p = r + beta * p
        rr = rr_new
    return x
