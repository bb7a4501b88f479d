"""SpMMV HBM bandwidth on the 3D Anderson model, L=128 (n=2,097,152,
nnz=14,680,064), stored as SELL-32-sigma (sigma=256), FP64, row-major block
vectors of width nvec in {1,2,4,8,16,32}.

One step = one SpMMV Y = A X for every nvec of the sweep (the kernel sweep of
the benchmark configuration).  The metric is algorithmic bytes / device time,
summed over the sweep:
    bytes(nvec) = nnz*(8+4) + 8*n*nvec*2 + ceil(n/C)*(8+4)     (beta = 0)
(the SpMMV byte model of PHIST, src/kernels/phist_kernel_perfmodels.hpp:92-107,
with the block-vector term multiplied by nvec).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times PHIST's builtin SpMMV on all host cores, as PHIST
dispatches it: widths 1, 2, 4, 8 on PHIST's own C kernels (compiled from the
PHIST sources into oracle/_ref), the other widths on the oracle's C
restatement of the Fortran loop PHIST uses for them (its Fortran+MPI build
is not possible here), on a bounded sample of the same workload.  Under
torchrun only rank 0 runs that arm.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = 128
PROBLEM = "ANDERSON3D-%d-S1" % L
NVECS = [1, 2, 4, 8, 16, 32]
C_SELL = 32
SIGMA = 256
METRIC = "SpMMV HBM GB/s (algorithmic bytes / device time), FP64 SELL-32-256, nvec sweep 1..32"
UNIT = "GB/s"


def spmv_bytes(n, nnz, nvec, C=C_SELL):
    nch = -(-n // C)
    return nnz * 12 + 8 * n * nvec * 2 + nch * 12


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region"""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(steps_budget_s=12.0, nvecs=NVECS):
    """PHIST's SpMMV on all host cores, as PHIST dispatches it: widths 1, 2,
    4, 8 on PHIST's own C kernels (dspmvm_nt_*_c, spmvm_kernels_nt.c,
    compiled from the PHIST sources into oracle/_ref), the other widths on
    the oracle's C restatement of the Fortran loop they take
    (spmvm_kernels.F90:494-523); all widths on the restatement when the
    compiled kernels are absent"""
    from oracle import oracle as O
    from phist_b200 import generators as G
    O.set_threads(os.cpu_count() or 1)
    rp, c, v = G.anderson3d(L, 1)
    n = len(rp) - 1
    nnz = int(rp[-1])
    xs = {k: G.random_block(n, k, 3) for k in nvecs}
    ys = {k: np.zeros((n, k)) for k in nvecs}
    lib = O.lib()
    P = O._p
    have_ref = O.ref_available()
    runs = {}
    for k in nvecs:
        if have_ref and k in (1, 2, 4, 8):
            runs[k] = ("phist_c", O.ref_spmmv_nt_runner(rp, c, v, xs[k])[0])
        else:
            def port(k=k):
                lib.orc_spmmv(n, P(rp), P(c), P(v), k, 1.0, None, P(xs[k]), k, 0.0, P(ys[k]), k)
            runs[k] = ("port", port)
    for k in nvecs:  # warm-up
        runs[k][1]()
    tk = {k: 0.0 for k in nvecs}
    passes = 0
    t_end = time.perf_counter() + steps_budget_s
    while passes < 1 or time.perf_counter() < t_end:
        for k in nvecs:
            t0 = time.perf_counter()
            runs[k][1]()
            tk[k] += time.perf_counter() - t0
        passes += 1
        if passes >= 50:
            break
    total_t = sum(tk.values())
    total_b = passes * sum(spmv_bytes(n, nnz, k) for k in nvecs)
    widths = {str(k): {"impl": runs[k][0], "GBs": round(passes * spmv_bytes(n, nnz, k) / tk[k] / 1e9, 2)}
              for k in nvecs}
    ref_widths = [k for k in nvecs if runs[k][0] == "phist_c"]
    return {"value": round(total_b / total_t / 1e9, 3), "unit": UNIT, "cores": O.num_threads(),
            "kind": "reference" if ref_widths else "port",
            "sample": "%d full passes of the nvec sweep {%s} on the same L=128 Anderson matrix (CRS, columns "
                      "sorted), OpenMP static over rows; widths {%s} on PHIST's own C kernels (dspmvm_nt_*_c, "
                      "spmvm_kernels_nt.c, compiled from source), the others on the C restatement of PHIST's "
                      "Fortran loop (spmvm_kernels.F90:494-523), which those widths take in PHIST"
                      % (passes, ",".join(map(str, nvecs)), ",".join(map(str, ref_widths))),
            "widths": widths,
            "seconds": round(total_t, 3)}


def max_over_ranks(x, dist=None, device="cuda"):
    """The largest of the ranks' values of x (every rank gets it): the
    timing rule of the multi-replica runs, where the job takes as long as
    its slowest rank.  x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cb = cpu_baseline(steps_budget_s=max(3.0, 2.0 * args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, ANDERSON3D L=128 seed 1)",
            "config": {"workload": "spmmv_anderson3d_L128_nvec_sweep", "problem": PROBLEM,
                       "n": L ** 3, "nnz": 7 * L ** 3, "nvec": NVECS, "format": "CRS (host)"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "widths")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def jada_forms(timeout=300):
    """Time-to-solution of PHIST's unchanged subspacejada on this library
    (phist_b200/lib/jada_run): 7-point Dirichlet Laplacian 64^3, the 10
    smallest eigenpairs, block size 4, minBas 20, maxBas 40, tol 1e-10,
    start block uniform[-1,1) seed 0; the plain FP64 drop-in (PHIST's
    GMRES for the correction equations), the device-resident GMRES in FP64,
    FP32 correction equations on the device GMRES, and the same two on the
    device MINRES (innerSolvType=MINRES; the matrix is symmetric).  Each
    solve runs twice in one process; the second (warm) wall time is
    reported."""
    exe = os.path.join(ROOT, "phist_b200", "lib", "jada_run")
    if not os.path.exists(exe):
        return {"unavailable": "phist_b200/lib/jada_run is not built (phist_b200/solvers/Makefile)"}
    common = ["LAPLACE3D-64", "numEigs=10", "blockSize=4", "minBas=20", "maxBas=40", "convTol=1e-10",
              "which=SR", "seed=0", "reps=2"]
    forms = {}
    for name, extra in (("fp64_phist_gmres", []), ("fp64_device_gmres", ["devgmres=1"]),
                        ("mixed_device_gmres", ["mixed=1", "devgmres=1"]),
                        ("fp64_device_minres", ["devgmres=1", "innerSolvType=MINRES"]),
                        ("mixed_device_minres", ["mixed=1", "devgmres=1", "innerSolvType=MINRES"])):
        try:
            r = subprocess.run([exe] + common + extra, capture_output=True, text=True, timeout=timeout)
            d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        except Exception as e:  # a failed form is reported, not fatal to the bench line
            forms[name] = {"failed": str(e)[:200]}
            continue
        sec = d["wall"][-1]
        forms[name] = {"seconds": round(sec, 4), "solves_per_s": round(1.0 / sec, 3),
                       "outer_iterations": d["nIter"], "converged": d["nConv"],
                       "max_res_explicit": max(d["resExplicit"][:10]), "launches": d["launches"]}
    out = {"workload": "subspacejada_laplace3d_64_10eigs", "n": 262144, "tol": 1e-10, "forms": forms}
    # the same solve (PHIST's unchanged subspacejada, same options and start
    # block) on the host cores: the CPU restatement of PHIST's builtin kernels
    # (oracle/cpu_backend.cpp); one solve is the sample
    try:
        from oracle import oracle as O
        if os.path.exists(O.JADA_CPU):
            cores = os.cpu_count() or 1
            d = O.jada_cpu(common[:-1] + ["reps=1"], threads=cores, timeout=timeout)
            sec = d["wall"][-1]
            out["cpu_baseline"] = {
                "seconds": round(sec, 4), "solves_per_s": round(1.0 / sec, 4), "cores": cores, "kind": "port",
                "outer_iterations": d["nIter"], "converged": d["nConv"],
                "max_res_explicit": max(d["resExplicit"][:10]),
                "sample": "one FP64 solve of the same problem: PHIST's subspacejada (unchanged, from its "
                          "sources) on a host-core restatement of PHIST's builtin kernels, OpenMP"}
            for name, f in forms.items():
                if "seconds" in f:
                    f["speedup_vs_cpu"] = round(sec / f["seconds"], 2)
        else:
            out["cpu_baseline"] = {"unavailable": "oracle/_ref/jada_run_cpu is not built"}
    except Exception as e:  # reported, not fatal to the bench line
        out["cpu_baseline"] = {"failed": str(e)[:200]}
    return out


def served_forms(timeout=300):
    """A short served request stream (the served-stream configuration with
    fewer and smaller requests so that it fits the benchmark's time):
    Poisson arrivals at 200/s (stream seed 5) of eigen-solves, each the 8
    smallest eigenpairs (tol 1e-10) of a 7-point Laplacian + diag uniform[0,1)
    on an L^3 grid, L log-uniform in [24, 64], through
    phist_b200/lib/serve_run (PHIST's unchanged subspacejada per request).
    Forms: plain FP64 drop-in on one stream; FP64 and FP32-correction
    solves on the device GMRES served by 8 workers on their own lanes; the
    FP32-correction solves on the device MINRES (the matrices are
    symmetric)."""
    exe = os.path.join(ROOT, "phist_b200", "lib", "serve_run")
    if not os.path.exists(exe):
        return {"unavailable": "phist_b200/lib/serve_run is not built (phist_b200/solvers/Makefile)"}
    common = ["nreq=12", "rate=200", "lmin=24", "lmax=64", "seed=5", "numEigs=8", "tol=1e-10"]
    forms = {}
    for name, extra in (("fp64_one_stream", ["workers=1", "devgmres=0"]),
                        ("fp64_device_gmres_served", ["workers=8", "devgmres=1"]),
                        ("mixed_device_gmres_served", ["workers=8", "devgmres=1", "mixed=1"]),
                        ("mixed_device_minres_served", ["workers=8", "devgmres=1", "mixed=1", "minres=1"])):
        try:
            r = subprocess.run([exe] + common + extra, capture_output=True, text=True, timeout=timeout)
            d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        except Exception as e:  # a failed form is reported, not fatal to the bench line
            forms[name] = {"failed": str(e)[:200]}
            continue
        forms[name] = {k: d.get(k) for k in ("solves_per_s", "latency_p50", "latency_p99", "latency_mean", "wall",
                                             "failed", "unconverged", "max_resExplicit") if k in d}
    return {"workload": "served_laplace_diag_stream_12req_L24_64", "requests": 12, "forms": forms}


def carp_forms(reps=5):
    """Batched multi-shift CARP-CG on the 1024 x 1024 x 2 honeycomb lattice
    (n = 2,097,152, on-site uniform[-0.5,0.5) seed 4): device time of one
    iteration (forward+backward colour sweep and fused CG updates) per slot
    count 1..32, FP64 and with FP32 sweeps, from the library's slot tuner
    (phist_b200_DcarpCG_tune_block), and the slot count it picks for 32
    systems.  Solves to 1e-10 of these indefinite systems need far more
    iterations than a benchmark run allows, so the figure is per iteration."""
    import ctypes as ct

    from phist_b200 import kernels as K
    from phist_b200.objects import SparseMat
    A = SparseMat.from_problem("HONEYCOMB-1024-S4-W1")
    out = {"workload": "carpcg_honeycomb_1024x1024x2_32_shifts", "n": A.nrows, "nnz": A.nnz}
    for name, mixed in (("fp64", 0), ("fp32_sweeps", 1)):
        us = (ct.c_double * 6)()
        blk = ct.c_int(0)
        K.chk(K.phist_b200_DcarpCG_tune_block, A.h, 32, mixed, reps, ct.byref(blk), us)
        t = {str(1 << q): round(us[q], 1) for q in range(6) if us[q] > 0}
        best = blk.value
        out[name] = {"iteration_us": t, "block": best,
                     "system_iterations_per_s": round(best / (us[best.bit_length() - 1] * 1e-6), 1)}
    A.delete()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nvecs", default=",".join(map(str, NVECS)))
    ap.add_argument("--no-jada", action="store_true", help="skip the eigen-solve timings")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end runs through host buffers")
    ap.add_argument("--e2e-threads", type=int, default=4,
                    help="host threads of the end-to-end run (each on its own lane and stream)")
    ap.add_argument("--no-forms", action="store_true", help="skip the served-stream and CARP-CG timings")
    args = ap.parse_args()
    nvecs = [int(t) for t in args.nvecs.split(",")]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        rc = run_reference(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return rc

    import torch

    from phist_b200 import kernels as K
    from phist_b200.objects import Mvec, SparseMat, launch_count, stream_handle

    torch.cuda.set_device(local)
    K.chk(K.phist_b200_set_sell_params, C_SELL, SIGMA)
    A = SparseMat.from_problem(PROBLEM, flags=K.PHIST_SPARSEMAT_PERM_LOCAL)
    n, nnz = A.nrows, A.nnz
    info = A.sell_info()
    lib_stream = torch.cuda.ExternalStream(stream_handle())
    from phist_b200 import generators as G
    X = {k: Mvec(A.domain_map, k).set(G.random_block(n, k, 3)) for k in nvecs}
    Y = {k: Mvec(A.row_map, k) for k in nvecs}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 256 MiB > 126 MB L2

    def one_step(times):
        for k in nvecs:
            with torch.cuda.stream(lib_stream):
                flush.fill_(k & 0xFF)  # evict L2 (untimed)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(lib_stream)
            K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, X[k].h, 0.0, Y[k].h)
            e1.record(lib_stream)
            times.append((k, e0, e1))

    for _ in range(args.warmup):
        one_step([])
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = launch_count()
    ev = []
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        one_step(ev)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    launches = launch_count() - l0
    clk = clocks.stop()
    per = {k: 0.0 for k in nvecs}
    for k, e0, e1 in ev:
        per[k] += e0.elapsed_time(e1) * 1e-3
    dev_time = sum(per.values())
    if dist is not None:
        dev_time = max_over_ranks(dev_time, dist)
        dist.barrier()
    step_bytes = sum(spmv_bytes(n, nnz, k) for k in nvecs)
    value = world * step_bytes * args.steps / dev_time / 1e9
    detail = {str(k): round(spmv_bytes(n, nnz, k) * args.steps / per[k] / 1e9, 1) for k in nvecs}

    # ---- end to end through the C ABI with pinned host buffers -------------
    import ctypes

    def ct_ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    h2d = sum(8 * n * k for k in nvecs)
    d2h = h2d

    def e2e_run(nthreads, steps):
        """steps sweeps through the C ABI, split over nthreads host threads;
        each thread has its own lane (the library gives every calling
        thread its own stream), its own X/Y and pinned host buffers, and
        runs whole sweeps: upload X (phist_Dmvec_set_data), SpMMV, download
        Y (phist_Dmvec_get_data) per block width.  Returns GB/s of
        algorithmic bytes over the wall time, and the last thread's Y."""
        import threading
        per = [steps // nthreads + (1 if t < steps % nthreads else 0) for t in range(nthreads)]
        bufs = []
        for t in range(nthreads):
            hx = {k: torch.from_numpy(G.random_block(n, k, 3)).pin_memory() for k in nvecs}
            hy = {k: torch.empty((n, k), dtype=torch.float64).pin_memory() for k in nvecs}
            Xt = {k: Mvec(A.domain_map, k) for k in nvecs}
            Yt = {k: Mvec(A.row_map, k) for k in nvecs}
            bufs.append((hx, hy, Xt, Yt))
        bar = threading.Barrier(nthreads + 1)
        errs = []

        def sweep(b):
            hx, hy, Xt, Yt = b
            for k in nvecs:
                K.chk(K.phist_Dmvec_set_data, Xt[k].h, ct_ptr(hx[k]), k, 1)
                K.chk(K.phist_DsparseMat_times_mvec, 1.0, A.h, Xt[k].h, 0.0, Yt[k].h)
                K.chk(K.phist_Dmvec_get_data, Yt[k].h, ct_ptr(hy[k]), k, 1)

        def worker(t):
            try:
                sweep(bufs[t])  # warm-up: lane, stream and caches of this thread
                bar.wait()
                for _ in range(per[t]):
                    sweep(bufs[t])
                bar.wait()
            except Exception as e:  # reported after the join
                errs.append(e)
                bar.abort()

        ths = [threading.Thread(target=worker, args=(t,)) for t in range(nthreads)]
        for th in ths:
            th.start()
        bar.wait()
        t0 = time.perf_counter()
        bar.wait()
        wall = time.perf_counter() - t0
        for th in ths:
            th.join()
        if errs:
            raise errs[0]
        hy_last = bufs[-1][1]
        for hx, hy, Xt, Yt in bufs:
            for k in nvecs:
                Xt[k].delete()
                Yt[k].delete()
        return step_bytes * steps / wall / 1e9, wall, hy_last

    if args.no_e2e:
        e2e_1 = e2e_val = None
        hy = {k: torch.from_numpy(Y[k].get()) for k in nvecs}
    else:
        e2e_1, _, _ = e2e_run(1, args.steps)
        e2e_2, e2e_time, hy = e2e_run(max(1, args.e2e_threads), args.steps)
        e2e_time = max_over_ranks(e2e_time, dist)
        e2e_val = world * step_bytes * args.steps / e2e_time / 1e9
    ok = np.isfinite(hy[nvecs[-1]].numpy()).all()
    # the end-to-end result equals the device-resident one bit for bit
    e2e_same = bool(np.array_equal(hy[nvecs[-1]].numpy(), Y[nvecs[-1]].get()))

    peak, peak_kind = read_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "spmmv_traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                traffic = json.load(f)
        except Exception:
            traffic = None

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dev_time / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded counter-based generator: 3D Anderson L=128 periodic, on-site U[-8.25,8.25] seed 1; X uniform[-1,1) seed 3)",
        "config": {"workload": "spmmv_anderson3d_L128_nvec_sweep", "problem": PROBLEM, "n": n, "nnz": nnz,
                   "format": "SELL-%d-%d" % (info["C"], info["sigma"]), "nnz_padded": info["nnz_padded"],
                   "nvec": nvecs, "beta": 0.0, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed before every SpMMV (256 MiB write, outside the timed events)"},
        "per_nvec_gbs": detail,
        "roofline": {"bound": "hbm", "kernel": "k_sell_spmmv (all nvec instantiations)",
                     "achieved": round(step_bytes * args.steps / dev_time / 1e9, 2),
                     "peak": peak, "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, copy)",
                     "unit": "GB/s", "frac": round(step_bytes * args.steps / dev_time / 1e9 / peak, 4),
                     "traffic": traffic.get("bytes_per_step") if traffic else None,
                     "algorithmic_bytes_per_step": step_bytes},
        "e2e": {"value": None if e2e_val is None else round(e2e_val, 2), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "per block width: phist_Dmvec_set_data (pinned host X) -> phist_DsparseMat_times_mvec "
                        "-> phist_Dmvec_get_data (pinned host Y); wall time of the timed sweeps, split over %d "
                        "host threads (each on its own lane/stream), so uploads of some threads overlap "
                        "downloads of others" % max(1, args.e2e_threads),
                "threads": max(1, args.e2e_threads),
                "single_thread_value": None if e2e_1 is None else round(e2e_1, 2)},
        "gpu_launches": launches,
        "clocks": clk,
        "wall_s_timed": round(t_wall, 4),
        "finite": bool(ok),
        "e2e_equals_device_result": e2e_same,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline(steps_budget_s=12.0, nvecs=nvecs).items()
                                if k != "seconds"}
    if rank == 0 and world == 1 and not args.no_jada:
        line["jada"] = jada_forms()
    if rank == 0 and world == 1 and not args.no_forms:
        line["served"] = served_forms()
        try:
            line["carp_cg"] = carp_forms()
        except Exception as e:  # reported, not fatal to the bench line
            line["carp_cg"] = {"failed": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for k in nvecs:
        X[k].delete()
        Y[k].delete()
    A.delete()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
