"""Per-kernel throughput of libphist_kernels_b200.so on the benchmark shapes.

    python -m phist_b200.bench_kernels [--suite spmmv,block,blas,carp] [--reps R] [--nvecs 1,...,32]

Every kernel is called through the C ABI on device-resident data, timed with
CUDA events on the library's stream, with the L2 flushed (256 MiB write)
before every call, outside the timed interval.  Each result line is JSON:
kernel, shape, algorithmic bytes and flops per call (the counts of
phist_kernel_perfmodels.hpp with the block-vector factors made explicit),
device time, GB/s, GFLOP/s and the fraction of the measured HBM peak.

Shapes: the 3D Anderson matrix, L=128 (n=2,097,152) for SpMMV; tall-skinny
n=2,097,152 blocks with m,k in {4,8,16,32,64} for the block products; the
1024x1024x2 honeycomb matrix with 8 shifts for the CARP sweep.
"""
import argparse
import ctypes as ct
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


class Timer:
    def __init__(self):
        import torch

        from .objects import stream_handle
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(stream_handle())
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def time(self, fn, reps):
        torch = self.torch
        fn()  # warm-up
        ts = []
        for r in range(reps):
            with torch.cuda.stream(self.stream):
                self.flush.fill_(r & 0xFF)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(self.stream)
            fn()
            e1.record(self.stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) * 1e-3 for a, b in ts]))


def report(kernel, shape, nbytes, flops, t, peak):
    line = {"kernel": kernel, "shape": shape, "bytes": int(nbytes), "flops": int(flops),
            "time_us": round(t * 1e6, 2), "GBs": round(nbytes / t / 1e9, 1),
            "GFLOPs": round(flops / t / 1e9, 1), "frac_hbm": round(nbytes / t / 1e9 / peak, 3)}
    print(json.dumps(line), flush=True)
    return line


def suite_spmmv(T, reps, peak, L=128):
    from . import kernels as K
    from .generators import random_block
    from .objects import Mvec, SdMat, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    A = SparseMat.from_problem("ANDERSON3D-%d-S1" % L, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n, nnz = A.nrows, A.nnz
    out = []
    for nv in NVECS:
        X = Mvec(A.domain_map, nv).set(random_block(n, nv, 3))
        Y = Mvec(A.row_map, nv)
        sh = np.linspace(-1, 1, nv)
        t = T.time(lambda: K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h), reps)
        b = nnz * 12 + 16 * n * nv + (-(-n // 32)) * 12
        out.append(report("spmmv", {"n": n, "nnz": nnz, "nvec": nv}, b, 2 * nnz * nv, t, peak))
        t = T.time(lambda: K.chk(K.phist_DsparseMat_times_mvec_vadd_mvec, 1.0, A.h, K.sptr(sh, np.float64),
                                 X.h, 1.0, Y.h), reps)
        out.append(report("spmmv_vadd_beta1", {"n": n, "nnz": nnz, "nvec": nv}, b + 8 * n * nv,
                          2 * nnz * nv + 4 * n * nv, t, peak))
        d1 = np.zeros(nv)
        d2 = np.zeros(nv)
        t = T.time(lambda: K.chk(K.phist_Dfused_spmv_mvdot, 1.0, A.h, X.h, 0.0, Y.h,
                                 K.sptr(d1, np.float64), K.sptr(d2, np.float64)), reps)
        out.append(report("fused_spmv_mvdot", {"n": n, "nnz": nnz, "nvec": nv}, b, 2 * nnz * nv + 4 * n * nv, t, peak))
        # W = A V with W'W and V'W in the same pass: the bytes of one SpMMV
        Gw, Gv = SdMat(nv, nv), SdMat(nv, nv)
        t = T.time(lambda: K.chk(K.phist_Dfused_spmv_mvTmv, 1.0, A.h, X.h, 0.0, Y.h, Gw.h, Gv.h,
                                 flags=K.PHIST_SDMAT_RUN_ON_DEVICE), reps)
        out.append(report("fused_spmv_mvTmv", {"n": n, "nnz": nnz, "nvec": nv}, b,
                          2 * nnz * nv + 4 * n * nv * nv, t, peak))
        Gw.delete()
        Gv.delete()
        X.delete()
        Y.delete()
    A.delete()
    return out


def suite_spmmv_tune(T, reps, peak, L=128):
    """every SpMMV launch shape (threads per row, unrolled or not) per width"""
    from . import kernels as K
    from .generators import random_block
    from .objects import Mvec, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    A = SparseMat.from_problem("ANDERSON3D-%d-S1" % L, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n, nnz = A.nrows, A.nnz
    opts = {1: (1,), 2: (1,), 4: (1, 2), 8: (1, 2, 4), 16: (2, 4, 8), 32: (4, 8, 16)}
    out = []
    for nv, tprs in opts.items():
        X = Mvec(A.domain_map, nv).set(random_block(n, nv, 3))
        Y = Mvec(A.row_map, nv)
        b = nnz * 12 + 16 * n * nv + (-(-n // 32)) * 12
        for tpr in tprs:
            for unroll in (1, 0):
                K.chk(K.phist_b200_set_spmv_config, nv, tpr, unroll)
                t = T.time(lambda: K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h), reps)
                out.append(report("spmmv_tpr%d_unroll%d" % (tpr, unroll), {"n": n, "nnz": nnz, "nvec": nv},
                                  b, 2 * nnz * nv, t, peak))
        X.delete()
        Y.delete()
    # back to the defaults
    for nv, tpr in ((4, 1), (8, 2), (16, 4), (32, 8)):
        K.chk(K.phist_b200_set_spmv_config, nv, tpr, 1)
    # shared-memory staged kernel on / off for the wide widths
    for nv in (8, 16, 32):
        X = Mvec(A.domain_map, nv).set(random_block(n, nv, 3))
        Y = Mvec(A.row_map, nv)
        b = nnz * 12 + 16 * n * nv + (-(-n // 32)) * 12
        for smin in (8, 99):
            K.chk(K.phist_b200_set_spmv_staged, smin)
            t = T.time(lambda: K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h), reps)
            out.append(report("spmmv_staged%d" % (smin <= 32), {"n": n, "nnz": nnz, "nvec": nv},
                              b, 2 * nnz * nv, t, peak))
        X.delete()
        Y.delete()
    K.chk(K.phist_b200_set_spmv_staged, 99)  # the library default
    A.delete()
    return out


def suite_block(T, reps, peak, n=1 << 21):
    from . import kernels as K
    from .generators import random_block
    from .objects import Map, Mvec, SdMat
    m_ = Map(n)
    out = []
    for m in (4, 8, 16, 32, 64):
        k = m
        V = Mvec(m_.h, m).set(random_block(n, m, 1))
        W = Mvec(m_.h, k).set(random_block(n, k, 2))
        C = SdMat(m, k).set(np.eye(m, k) + 0.01)
        G = SdMat(k, k)
        t = T.time(lambda: K.chk(K.phist_DmvecT_times_mvec, 1.0, V.h, W.h, 0.0, C.h), reps)
        out.append(report("mvecT_times_mvec", {"n": n, "m": m, "k": k}, 8 * n * (m + k), 2 * n * m * k, t, peak))
        # the same product with the result left on the device (no download, no host sync)
        t = T.time(lambda: K.chk(K.phist_DmvecT_times_mvec, 1.0, V.h, W.h, 0.0, C.h,
                                 flags=K.PHIST_SDMAT_RUN_ON_DEVICE), reps)
        out.append(report("mvecT_times_mvec_device", {"n": n, "m": m, "k": k}, 8 * n * (m + k), 2 * n * m * k,
                          t, peak))
        t = T.time(lambda: K.chk(K.phist_Dmvec_times_sdMat, 1.0, V.h, C.h, 0.0, W.h), reps)
        out.append(report("mvec_times_sdMat", {"n": n, "m": m, "k": k}, 8 * n * (m + k), 2 * n * m * k, t, peak))
        t = T.time(lambda: K.chk(K.phist_Dmvec_times_sdMat_inplace, W.h, C.h), reps)
        out.append(report("mvec_times_sdMat_inplace", {"n": n, "m": m, "k": k}, 8 * n * 2 * k, 2 * n * m * k, t, peak))
        t = T.time(lambda: K.chk(K.phist_Dfused_mvsd_mvTmv, 1.0, V.h, C.h, 0.0, W.h, G.h), reps)
        out.append(report("fused_mvsd_mvTmv", {"n": n, "m": m, "k": k}, 8 * n * (m + k),
                          2 * n * m * k + 2 * n * k * k, t, peak))
        # compensated (double-double) Gram product, PHIST_ROBUST_REDUCTIONS
        t = T.time(lambda: K.chk(K.phist_DmvecT_times_mvec, 1.0, V.h, W.h, 0.0, C.h,
                                 flags=K.PHIST_ROBUST_REDUCTIONS | K.PHIST_SDMAT_RUN_ON_DEVICE), reps)
        out.append(report("mvecT_times_mvec_robust", {"n": n, "m": m, "k": k}, 8 * n * (m + k),
                          2 * n * m * k, t, peak))
        for o in (V, W, C, G):
            o.delete()
    m_.delete()
    return out


def suite_blas(T, reps, peak, n=1 << 21):
    from . import kernels as K
    from .generators import random_block
    from .objects import Map, Mvec
    m_ = Map(n)
    out = []
    for nv in (1, 4, 8, 32):
        X = Mvec(m_.h, nv).set(random_block(n, nv, 1))
        Y = Mvec(m_.h, nv).set(random_block(n, nv, 2))
        d = np.zeros(nv)
        t = T.time(lambda: K.chk(K.phist_Dmvec_dot_mvec, X.h, Y.h, K.sptr(d, np.float64)), reps)
        out.append(report("mvec_dot_mvec", {"n": n, "nvec": nv}, 16 * n * nv, 2 * n * nv, t, peak))
        t = T.time(lambda: K.chk(K.phist_Dmvec_add_mvec, 0.5, X.h, 1.0, Y.h), reps)
        out.append(report("mvec_add_mvec", {"n": n, "nvec": nv}, 24 * n * nv, 2 * n * nv, t, peak))
        X.delete()
        Y.delete()
    m_.delete()
    return out


def suite_latency(T, reps, peak, n=262144):
    """host wall time per call, as a solver sees it, at the size of the 64^3
    Laplacian (no L2 flush; the median of 200 back-to-back calls)"""
    import time

    from . import kernels as K
    from .generators import random_block
    from .objects import Map, Mvec, SdMat, SparseMat, sync
    A = SparseMat.from_problem("LAPLACE3D-64")
    m_ = A.domain_map
    X1 = Mvec(m_, 1).set(random_block(n, 1, 1))
    Y1 = Mvec(m_, 1).set(random_block(n, 1, 2))
    X4 = Mvec(m_, 4).set(random_block(n, 4, 3))
    Y4 = Mvec(m_, 4).set(random_block(n, 4, 4))
    V = Mvec(m_, 40).set(random_block(n, 40, 5))
    C = SdMat(40, 4)
    C44 = SdMat(4, 4).set(np.eye(4))
    d = np.zeros(4)
    a4 = np.array([0.5, -0.25, 1.0, 2.0])
    calls = {
        "mvec_dot_mvec_nvec1": lambda: K.chk(K.phist_Dmvec_dot_mvec, X1.h, Y1.h, K.sptr(d, np.float64)),
        "mvec_dot_mvec_nvec4": lambda: K.chk(K.phist_Dmvec_dot_mvec, X4.h, Y4.h, K.sptr(d, np.float64)),
        "mvec_norm2_nvec4": lambda: K.chk(K.phist_Dmvec_norm2, X4.h, K.sptr(d, np.float64)),
        "mvec_vadd_mvec_nvec4": lambda: K.chk(K.phist_Dmvec_vadd_mvec, K.sptr(a4, np.float64), X4.h, 1.0, Y4.h),
        "mvec_add_mvec_nvec1": lambda: K.chk(K.phist_Dmvec_add_mvec, 0.5, X1.h, 1.0, Y1.h),
        "spmmv_nvec4": lambda: K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X4.h, 0.0, Y4.h),
        "mvecT_times_mvec_40x4": lambda: K.chk(K.phist_DmvecT_times_mvec, 1.0, V.h, X4.h, 0.0, C.h),
        "mvec_times_sdMat_40x4": lambda: K.chk(K.phist_Dmvec_times_sdMat, 1.0, V.h, C.h, 0.0, Y4.h),
        "mvec_times_sdMat_inplace_4x4": lambda: K.chk(K.phist_Dmvec_times_sdMat_inplace, Y4.h, C44.h),
    }
    out = []
    for name, f in calls.items():
        for _ in range(20):
            f()
        sync()
        ts = []
        for _ in range(200):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        sync()
        line = {"kernel": name, "n": n, "host_us_p50": round(float(np.median(ts)) * 1e6, 2),
                "host_us_p90": round(float(np.percentile(ts, 90)) * 1e6, 2)}
        print(json.dumps(line), flush=True)
        out.append(line)
    for o in (X1, Y1, X4, Y4, V, C, C44, A):
        o.delete()
    return out


def suite_autotune(T, reps, peak, L=128):
    """SpMMV before and after the autotuner (SELL C, sigma and kernel variant
    per width chosen by timing) on the Anderson L=128 matrix (7 entries in
    every row) and the Dirichlet Laplacian 128^3 (4 to 7 entries)"""
    out = []
    for prob in ("ANDERSON3D-%d-S1" % L, "LAPLACE3D-%d" % L):
        out += _autotune_one(T, reps, peak, prob)
    return out


def _autotune_one(T, reps, peak, prob):
    from . import kernels as K
    from .generators import random_block
    from .objects import Mvec, SparseMat
    K.chk(K.phist_b200_set_sell_params, 32, 256)
    A = SparseMat.from_problem(prob, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n, nnz = A.nrows, A.nnz
    widths = [1, 2, 4, 8, 16, 32]
    out = []

    def sweep(tag):
        for nv in widths:
            X = Mvec(A.domain_map, nv).set(random_block(n, nv, 3))
            Y = Mvec(A.row_map, nv)
            b = nnz * 12 + 16 * n * nv + (-(-n // 32)) * 12
            t = T.time(lambda: K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X.h, 0.0, Y.h), reps)
            out.append(report("spmmv_" + tag, {"problem": prob, "n": n, "nnz": nnz, "nvec": nv}, b, 2 * nnz * nv,
                              t, peak))
            X.delete()
            Y.delete()

    sweep("default")
    wd = np.array(widths, np.int32)
    best = np.zeros(len(widths))
    t0 = time.perf_counter()
    K.chk(K.phist_b200_DsparseMat_autotune, A.h, len(widths), K.ptr(wd), 5, K.ptr(best))
    wall = time.perf_counter() - t0
    C, sig = ct.c_int(), ct.c_int64()
    tpr, unr, stg = (np.zeros(6, np.int32) for _ in range(3))
    K.chk(K.phist_b200_DsparseMat_get_tuning, A.h, ct.byref(C), ct.byref(sig), K.ptr(tpr), K.ptr(unr), K.ptr(stg))
    line = {"autotune": {"problem": prob, "C": C.value, "sigma": sig.value, "tpr": tpr.tolist(), "unroll": unr.tolist(),
                         "staged": stg.tolist(), "tuner_us": [round(x, 2) for x in best], "wall_s": round(wall, 2)}}
    print(json.dumps(line), flush=True)
    sweep("tuned")
    A.delete()
    return out


def suite_carp(T, reps, peak):
    """double CARP sweep on the honeycomb matrix (1024 x 1024 cells, 2 sites),
    block-coloured layout (default) and row-colour layout, 8 and 16 shifts"""
    from . import kernels as K
    from .generators import random_block
    from .objects import Mvec, SparseMat
    A = SparseMat.from_problem("HONEYCOMB-1024-S4-W1")
    n, nnz = A.nrows, A.nnz
    out = []
    for blocks in (1, 0):
        K.chk(K.phist_b200_set_option, b"carp_blocks", blocks)
        for nv in (8, 16):
            sh = np.linspace(-2.5, 2.5, nv)
            om = np.ones(nv)
            work = ct.c_void_p()
            K.chk(K.phist_Dcarp_setup, A.h, nv, K.sptr(sh, np.float64), ct.byref(work))
            X = Mvec(A.row_map, nv)
            B = Mvec(A.row_map, nv).set(random_block(n, nv, 4))
            t = T.time(lambda: K.chk(K.phist_Dcarp_sweep, A.h, K.sptr(sh, np.float64), B.h, X.h, work,
                                     K.sptr(om, np.float64)), reps)
            nb = 2 * (nnz * 12 + 8 * n * nv * 3)
            nc = ct.c_int()
            K.chk(K.phist_b200_Dcarp_color_order, work, None, ct.byref(nc), None)
            out.append(report("carp_sweep", {"n": n, "nnz": nnz, "nvec": nv, "layout": "blocks" if blocks else "rowcolour",
                                             "segments": nc.value}, nb, 16 * nnz * nv, t, peak))
            K.chk(K.phist_Dcarp_destroy, A.h, work)
            X.delete()
            B.delete()
    K.chk(K.phist_b200_set_option, b"carp_blocks", 1)
    A.delete()
    return out


NVECS = (1, 2, 4, 8, 16, 32)


def main():
    global NVECS
    ap = argparse.ArgumentParser()
    ap.add_argument("--suite", default="spmmv,block,blas,carp")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--nvecs", default="1,2,4,8,16,32", help="block widths of the spmmv suite")
    args = ap.parse_args()
    NVECS = tuple(int(v) for v in args.nvecs.split(","))
    T = Timer()
    peak = _peak()
    for s in args.suite.split(","):
        globals()["suite_" + s](T, args.reps, peak)
    return 0


if __name__ == "__main__":
    sys.exit(main())
