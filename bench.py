#!/usr/bin/env python
"""Benchmark of the B200 multigrid solve phase (one JSON line on stdout, rank 0).

Workload (headline): smoothed-aggregation V-cycle PCG on the 2D five-point Poisson
problem, 500 x 500 grid (N = 250,000, nnz = 1,248,000), k = 64 right-hand sides
~ N(0, 1) from ``default_rng(0)`` stored [N, 64], damped Jacobi (omega = 2/3, 1+1
sweeps), pinv coarse solve, mixed precision: FP32 cycle and FP32 CG vectors (FP64 dots
and step lengths) with the FP64 solution and FP64 true residual refreshed on demand
(reliable updates), stopping at relative residual 1e-8 checked on the FP64 residual.  A
"step" is one such solve; the metric is ms per solve (lower is better).
Sub-measurements in ``variants``: the plain FP64 path, the FP64 CG around the FP32
cycle, k = 1, and the standalone (repeated-cycle) solve.

Timing: W untimed warm-up solves, then K solves each bracketed by CUDA events on the
launching stream, with a 256 MB L2 flush between solves outside the events; barrier +
synchronize around the timed block; max over ranks.  ``e2e`` repeats the headline
through the public API from pinned host buffers (H2D of B and D2H of X inside the
timed region).  ``roofline`` times every fine-level kernel of the CG step alone through
the C ABI (``amg_time_pcg_ops``) and reports the one with the largest time per solve.  ``cpu_baseline`` times the FP64 CPU
oracle (numpy/scipy restatement of AMJax's solve) on all k columns, one thread.
``--impl reference`` times that CPU restatement instead: all k columns per step, one
column per task over one single-threaded worker process per host core, set-up outside
the timer.

Multi-GPU (torchrun, one process per GPU): each rank solves its own 64 columns (seed =
rank) on a replicated hierarchy, no data-path collective (weak scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PUBLISHED = {"AMJax+PCG FP64 vmap k=64 N=250k (A100 80GB, omega=1/rho, U[0,1) rhs)": 295.15,
             "AMJax+PCG FP64 k=1 N=250k (A100 80GB)": 7.14}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=500)
    p.add_argument("--k", type=int, default=64)
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--no-variants", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--kernel-only", action="store_true",
                   help="only launch the dominant kernel (fine-level FP32 Jacobi sweep, k columns) a few "
                        "times: the command the ncu captures of that kernel run")
    p.add_argument("--kernel-reps", type=int, default=3)
    p.add_argument("--ragged", action="store_true",
                   help="config 3b: 24 SA hierarchies (2D, n ~ U{64..1024} from default_rng(1), odd i "
                        "rotated anisotropic), k_i ~ U{1..16}, mixed PCG to 1e-8 in one graph launch")
    p.add_argument("--cube", action="store_true",
                   help="config 4: 3D 7-point lognormal-kappa diffusion 128^3, V/W/F, k = 1 and 16, "
                        "FP32-cycle refinement to 1e-10 vs FP64; error vs a direct solve at 48^3")
    p.add_argument("--kernel", default="jacobi32", choices=["jacobi32", "pcg"],
                   help="--kernel-only target: the FP32 Jacobi sweep alone, or --kernel-reps CG steps of "
                        "the headline solve (every kernel of the CG loop)")
    return p.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(n, seed=0):
    from amjax_b200 import amg_setup, gallery
    A = gallery.poisson((n, n))
    host = amg_setup.smoothed_aggregation_solver(A)
    return A, host


# ---------------------------------------------------------------------------- clocks
class Clocks:
    Q = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, bus_id=None):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 10]
        if bus_id:
            mine = [r for r in rows if r[1].lower().endswith(bus_id.lower()[-12:])]
            rows = mine or rows
        if not rows:
            return None
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        pw = [float(r[4]) for r in rows if r[4].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower().startswith("active")})
        load = [s for s, p in zip(sm, pw) if p > 200] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


# ---------------------------------------------------------------------------- timing
def timed_steps(fn, steps, warmup, flush):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s, e in evs:
        flush()
        s.record()
        fn()
        e.record()
    torch.cuda.synchronize()
    ts = [s.elapsed_time(e) for s, e in evs]
    return ts


def cpu_oracle_columns(host, B, cols, tol, method, spec):
    """Wall time of the FP64 CPU oracle solving columns ``cols`` of B one after another on
    this thread (BLAS / OpenMP held to one thread); the oracle's hierarchy is built before
    the clock starts."""
    from threadpoolctl import threadpool_limits
    from oracle import amg_oracle as O
    oml = O.Hierarchy.from_host(host, presmoother=spec, postsmoother=spec, coarse_solver="pinv")
    A = host.levels[0].A
    M = O.aspreconditioner(oml)
    with threadpool_limits(1):
        t0 = time.perf_counter()
        for c in cols:
            if method == "pcg":
                O.cg(A, B[:, c], tol=tol, maxiter=500, M=M)
            else:
                O.solve_loop(oml, B[:, c], tol=tol, maxiter=500)
        return time.perf_counter() - t0


_REF = {}
_THREAD_VARS = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS")


def _ref_init(n, k, tol):
    """Worker set-up, once per process and outside every timed region: the hierarchy, the
    oracle's copy of it, the preconditioner and the k right-hand sides (seed 0, as rank 0
    of the GPU arm)."""
    from threadpoolctl import threadpool_limits
    from oracle import amg_oracle as O
    threadpool_limits(1)
    spec = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
    A, host = workload(n)
    oml = O.Hierarchy.from_host(host, presmoother=spec, postsmoother=spec, coarse_solver="pinv")
    _REF.update(A=A, M=O.aspreconditioner(oml), tol=tol,
                B=np.random.default_rng(0).standard_normal((A.shape[0], k)))


def _ref_column(c):
    from oracle import amg_oracle as O
    O.cg(_REF["A"], _REF["B"][:, c], tol=_REF["tol"], maxiter=500, M=_REF["M"])
    return c


# ---------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU path for the headline workload: every one of the k columns solved
    by the FP64 CPU restatement of AMJax's PCG (AMJax itself needs JAX and PyAMG, absent
    here), one column per task over a pool of one single-threaded process per host core.
    A step is one whole k-column solve, wall-clock timed; nothing is extrapolated."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0))
    k = args.k
    workers = max(1, min(k, cores))
    saved = {v: os.environ.get(v) for v in _THREAD_VARS}
    for v in _THREAD_VARS:  # inherited by the spawned workers before they import numpy
        os.environ[v] = "1"
    try:
        ctx = mp.get_context("spawn")
        with ctx.Pool(workers, initializer=_ref_init, initargs=(args.n, k, args.tol)) as pool:
            pool.map(_ref_column, range(workers), chunksize=1)  # every worker has finished its set-up
            times = []
            for step in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                pool.map(_ref_column, range(k), chunksize=1)
                dt = (time.perf_counter() - t0) * 1e3
                if step >= args.warmup:
                    times.append(dt)
    finally:
        for v, val in saved.items():
            if val is None:
                os.environ.pop(v, None)
            else:
                os.environ[v] = val
    v = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms/solve", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, "f64 (CPU restatement of AMJax's solve: FP64 numpy/scipy)"),
        "step_ms": {"min": min(times), "median": statistics.median(times)},
        "cpu_baseline": {"value": v, "unit": "ms/solve", "cores": workers, "kind": "port",
                         "sample": f"all {k} columns per step, one column per task over {workers} "
                                   f"single-threaded worker processes (BLAS/OpenMP 1 thread each); "
                                   f"hierarchy, oracle and right-hand sides built once per worker "
                                   f"outside the timer"},
        "e2e": {"value": v, "unit": "ms/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "JAX and PyAMG are not installed, so AMJax itself cannot run; this arm times the "
                "FP64 CPU restatement of its solve path (oracle/amg_oracle.py) on every host core.",
    }
    print(json.dumps(line), flush=True)
    return 0


METRIC = "ms/solve to 1e-8 rel resid, N=250k k=1/64: mixed-prec vs FP64 path; HBM GB/s"


def config_dict(args, precision):
    return {"workload": f"SA V-cycle PCG, 2D 5-point Poisson {args.n}x{args.n} (N={args.n * args.n}), "
                        f"k={args.k} RHS ~N(0,1) stored [N,k], Jacobi omega=2/3 1+1, pinv coarse, "
                        f"tol {args.tol:g}",
            "precision": precision, "hierarchy": "smoothed aggregation (host set-up, PyAMG defaults restated)",
            "global_batch": args.k * args.gpus, "parallelism": f"rhs-shard x{args.gpus}",
            "l2": "256 MB buffer written between timed solves (outside the events)"}


# ---------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from amjax_b200 import MultilevelSolver, bytemodel
    from amjax_b200 import _native as N
    import ctypes as C

    A, host = workload(args.n)
    Nn = A.shape[0]
    spec = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
    ml = MultilevelSolver.from_pyamg(host, presmoother=spec, postsmoother=spec, coarse_solver="pinv")
    k = args.k
    Bh = np.random.default_rng(rank).standard_normal((Nn, k))
    B = torch.as_tensor(Bh).cuda()
    flushbuf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def flush():
        flushbuf.fill_(1.0)

    prec_mixed = ml._precision("mixed")
    prec_f64cg = ml._precision("mixed-f64cg")
    prec_f64 = ml._precision("f64")

    def pcg(b, prec):
        return lambda: ml._pcg_dev(b, None, args.tol, 0.0, 500, "V", 1, prec)

    def solve(b, prec):
        return lambda: ml._solve_dev(b, None, args.tol, 500, "V", 1, prec)

    hbm_peak, peak_kind = load_peaks()
    bus = None
    try:
        bus = subprocess.run(["nvidia-smi", "--query-gpu=pci.bus_id", "--format=csv,noheader", "-i",
                              os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]],
                             capture_output=True, text=True, timeout=10).stdout.strip() or None
    except Exception:
        bus = None
    clocks = Clocks()
    clocks.start()

    # ---- headline: timed block bracketed by barrier + synchronize, max over ranks
    headline = pcg(B, prec_mixed)
    # first call: autotuning of every op layout, graph capture and instantiation (host wall
    # clock, synchronised); then a call on fresh B / X buffers: graphs are keyed by buffer
    # addresses, so it captures again (tuning is cached)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    headline()
    torch.cuda.synchronize()
    first_call_ms = (time.perf_counter() - t0) * 1e3
    B2 = B.clone()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ml._pcg_dev(B2, None, args.tol, 0.0, 500, "V", 1, prec_mixed)
    torch.cuda.synchronize()
    new_buffers_ms = (time.perf_counter() - t0) * 1e3
    del B2
    for _ in range(args.warmup):
        headline()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = N.kernel_launch_count()
    ts = timed_steps(headline, args.steps, 0, flush)
    launches = N.kernel_launch_count() - n0
    torch.cuda.synchronize()
    total = torch.tensor([sum(ts)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.barrier()
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    ms_per_step = float(total.item()) / args.steps
    value = float(total.item()) / (args.steps * world)
    x, info = headline()
    its = info["iterations"]
    stats = bytemodel.level_stats(ml)
    sbytes = bytemodel.solve_bytes(stats, k, max(its), method="pcg", cycle_s=4, outer_s=8)
    out = {"metric": METRIC, "value": value, "unit": "ms/solve", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 cycle / f64 outer", "data": "synthetic",
           "config": config_dict(args, "mixed: FP32 cycle (values, vectors, accumulation) and FP32 CG vectors "
                                       "with FP64 dots and step lengths; FP64 solution and FP64 true residual "
                                       "refreshed on demand (reliable updates), stop rule on the FP64 residual"),
           "iterations": {"min": min(its), "max": max(its)},
           "step_ms": {"min": min(ts), "median": statistics.median(ts)},
           "solve_bandwidth": {"bytes_per_solve_model": sbytes, "gbs": sbytes / (ms_per_step * 1e-3) / 1e9,
                               "frac_of_" + peak_kind: sbytes / (ms_per_step * 1e-3) / 1e9 / hbm_peak},
           "gpu_launches": int(launches),
           "first_call_ms": {"cold": first_call_ms, "new_buffers": new_buffers_ms,
                             "note": "host wall clock of the first call (autotuning + graph capture + solve) and "
                                     "of a call on new buffers (capture + solve); steady state is value"},
           "published_reference_ms": PUBLISHED}

    xh = x.cpu().numpy()
    res = np.linalg.norm(Bh - A @ xh, axis=0) / np.linalg.norm(Bh, axis=0)
    out["relres_fp64"] = {"max": float(res.max()), "mean": float(res.mean())}

    # ---- e2e through the public API from pinned host memory
    Bpin = torch.as_tensor(Bh).pin_memory()
    Xpin = torch.empty_like(Bpin).pin_memory()

    def e2e_step():
        ml.pcg(Bpin, tol=args.tol, maxiter=500, precision="mixed", out=Xpin)

    te = timed_steps(e2e_step, args.steps, args.warmup, flush)
    torch.cuda.synchronize()
    te_tot = torch.tensor([sum(te)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te_tot, op=dist.ReduceOp.MAX)
    out["e2e"] = {"value": float(te_tot.item()) / (args.steps * world), "unit": "ms/solve",
                  "h2d_bytes_per_step": int(Bpin.numel() * 8), "d2h_bytes_per_step": int(Xpin.numel() * 8),
                  "api": "MultilevelSolver.pcg(pinned host B, out=pinned host X, precision='mixed') -> "
                         "amg_pcg_host: two column blocks, each block's copies overlapped with the other's solve"}

    # ---- variants (rank 0 only does the bookkeeping; every rank runs the same work)
    if not args.no_variants:
        var = {}
        b1 = B[:, 0].contiguous()
        for name, fn, kk, meth, cs in [
            ("k64_pcg_f64", pcg(B, prec_f64), k, "pcg", 8),
            ("k64_pcg_mixed_f64cg", pcg(B, prec_f64cg), k, "pcg", 4),
            ("k1_pcg_mixed", pcg(b1, prec_mixed), 1, "pcg", 4),
            ("k1_pcg_mixed_f64cg", pcg(b1, prec_f64cg), 1, "pcg", 4),
            ("k1_pcg_f64", pcg(b1, prec_f64), 1, "pcg", 8),
            ("k64_solve_mixed", solve(B, prec_mixed), k, "solve", 4),
            ("k64_solve_f64", solve(B, prec_f64), k, "solve", 8),
            ("k1_solve_mixed", solve(b1, prec_mixed), 1, "solve", 4),
            ("k1_solve_f64", solve(b1, prec_f64), 1, "solve", 8),
        ]:
            t = timed_steps(fn, args.steps, args.warmup, flush)
            xv, inf = fn()
            ms = statistics.mean(t)
            its_v = inf["iterations"]
            bb = bytemodel.solve_bytes(stats, kk, max(its_v), method=meth, cycle_s=cs, outer_s=8)
            xr = xv.cpu().numpy().reshape(Nn, -1)
            Bv = Bh[:, :kk]
            rr = np.linalg.norm(Bv - A @ xr, axis=0) / np.linalg.norm(Bv, axis=0)
            var[name] = {"ms": ms, "ms_min": min(t), "iterations": max(its_v), "relres_max": float(rr.max()),
                         "gbs_model": bb / (ms * 1e-3) / 1e9}
        var["speedup_mixed_vs_f64_k64_pcg"] = var["k64_pcg_f64"]["ms"] / statistics.mean(ts)
        var["speedup_mixed_vs_f64_k1_pcg"] = var["k1_pcg_f64"]["ms"] / var["k1_pcg_mixed"]["ms"]
        var["speedup_mixed_f64cg_vs_f64_k64_pcg"] = var["k64_pcg_f64"]["ms"] / var["k64_pcg_mixed_f64cg"]["ms"]
        out["variants"] = var

    # ---- roofline: every fine-level kernel of the headline's CG step timed alone with CUDA
    # events (layouts as in the solve, L2 evicted before each launch); the dominant one is
    # the kernel with the largest time per solve (microseconds x launches per solve)
    it = max(its)
    per_solve = {"cg_direction_pAp": it, "cg_update": it, "post_smooth_with_dot": it + 1,
                 "residual_presmoothed": it + 1, "restriction": it + 1, "prolongation_correction": it + 1}
    rows = N.time_pcg_ops(ml._native(), k, reps=10)
    traffic_db = {}
    tpath = os.path.join(ROOT, "profiles", "pcg_mixed_k64_kernels_dram.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic_db = json.load(f).get("dram_bytes_per_launch", {})
    table = []
    for name, us_, by in rows:
        gbs = by / (us_ * 1e-6) / 1e9
        table.append({"kernel": name, "us": us_, "algorithmic_bytes": by, "gbs": gbs, "frac": gbs / hbm_peak,
                      "launches_per_solve": per_solve.get(name), "dram_bytes_ncu": traffic_db.get(name)})
    dom = max((r for r in table if r["launches_per_solve"]), key=lambda r: r["us"] * r["launches_per_solve"])
    out["roofline"] = {"bound": "hbm", "achieved": dom["gbs"], "peak": hbm_peak, "unit": "GB/s",
                       "frac": dom["frac"], "traffic": dom["dram_bytes_ncu"],
                       "peak_kind": peak_kind + " (burst copy)",
                       "kernel": f"{dom['kernel']} (fine level, N={Nn}, k={k}, FP32 vectors; the largest "
                                 f"microseconds x launches per solve)",
                       "algorithmic_bytes_per_launch": dom["algorithmic_bytes"], "launch_us": dom["us"],
                       "timing": "each launch alone between CUDA events on the launching stream, after a "
                                 "256 MB write that evicts L2; mean of 10",
                       "kernels": table}

    ck = clocks.stop(bus)
    out["clocks"] = ck

    # ---- CPU baseline (rank 0, N = 1): FP64 oracle on a sample of columns
    if rank == 0 and world == 1 and not args.no_cpu:
        t = cpu_oracle_columns(host, Bh, list(range(k)), args.tol, "pcg", spec)
        out["cpu_baseline"] = {"value": t * 1e3, "unit": "ms/solve", "cores": 1, "kind": "port",
                               "sample": f"all {k} columns, FP64 PCG one column at a time on one "
                                         f"thread (BLAS/OpenMP held to 1 thread)"}
        # true error against a direct FP64 solve on a few columns
        try:
            import scipy.sparse.linalg as spla
            lu = spla.splu(A.tocsc())
            xd = lu.solve(Bh[:, :4])
            err = np.linalg.norm(xh[:, :4] - xd, axis=0) / np.linalg.norm(xd, axis=0)
            out["rel_err_vs_spsolve"] = float(err.max())
        except Exception as ex:
            out["rel_err_vs_spsolve"] = f"unavailable: {ex}"
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_kernel_only(args):
    import torch
    from amjax_b200 import CSRMatrix, gallery, inverse_diagonal
    from amjax_b200 import _native as N
    if args.kernel == "pcg":
        from amjax_b200 import MultilevelSolver
        A, host = workload(args.n)
        spec = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
        ml = MultilevelSolver.from_pyamg(host, presmoother=spec, postsmoother=spec)
        B = torch.as_tensor(np.random.default_rng(0).standard_normal((A.shape[0], args.k))).cuda()
        ml._pcg_dev(B, None, 0.0, 0.0, args.kernel_reps, "V", 1, ml._precision("mixed"))
        torch.cuda.synchronize()
        print(json.dumps({"kernel_only": "pcg", "n": A.shape[0], "k": args.k, "steps": args.kernel_reps}))
        return 0
    A = gallery.poisson((args.n, args.n))
    Ad = CSRMatrix.from_scipy(A)
    Dinv = inverse_diagonal(Ad).to(torch.float32)
    k = args.k
    xs = torch.randn(A.shape[0], k, dtype=torch.float32, device="cuda")
    bs = torch.randn(A.shape[0], k, dtype=torch.float32, device="cuda")
    ys = torch.empty_like(xs)
    for _ in range(args.kernel_reps):
        N.call("amg_jacobi", Ad.desc(), 1, N.ptr(xs), N.ptr(bs), N.ptr(Dinv), N.ptr(ys), k, 1, 2.0 / 3.0,
               N.stream_ptr())
    torch.cuda.synchronize()
    print(json.dumps({"kernel_only": True, "n": A.shape[0], "k": k, "reps": args.kernel_reps}))
    return 0


def _time_ms(fn, steps, warmup):
    import torch
    ts = timed_steps(fn, steps, warmup, lambda: None)
    return statistics.mean(ts), min(ts)


def run_ragged(args):
    """Config 3b.  Draw order: for i in 0..23, n_i then k_i from default_rng(1); system i's
    right-hand sides from default_rng(100 + i).  Even i: 5-point Poisson n_i^2; odd i: rotated
    (45 degree) anisotropic diffusion with epsilon 1e-2 (i = 1, 5, 9, ...) or 1e-3."""
    import torch
    from amjax_b200 import MultilevelSolver, amg_setup, gallery, pcg_batch
    rng = np.random.default_rng(1)
    draws = [(int(rng.integers(64, 1025)), int(rng.integers(1, 17))) for _ in range(24)]
    spec = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
    mls, rhs, mats = [], [], []
    t0 = time.perf_counter()
    for i, (n, k) in enumerate(draws):
        A = gallery.poisson((n, n)) if i % 2 == 0 else gallery.anisotropic_diffusion_2d(
            n, 1e-2 if (i // 2) % 2 == 0 else 1e-3, np.pi / 4)
        mls.append(MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A),
                                               presmoother=spec, postsmoother=spec))
        rhs.append(torch.as_tensor(np.random.default_rng(100 + i).standard_normal((A.shape[0], k))).cuda())
        mats.append(A)
    setup_s = time.perf_counter() - t0
    batch = lambda: pcg_batch(mls, rhs, tol=1e-8, maxiter=500, precision="mixed")
    seq = lambda: [m.pcg(b, tol=1e-8, maxiter=500, precision="mixed") for m, b in zip(mls, rhs)]
    tb, tbmin = _time_ms(batch, args.steps, args.warmup)
    tsq, tsqmin = _time_ms(seq, args.steps, args.warmup)
    X, info = pcg_batch(mls, rhs, tol=1e-8, maxiter=500, precision="mixed", return_info=True)
    rel = []
    for A, b, x in zip(mats, rhs, X):
        bn, xn = b.cpu().numpy(), x.cpu().numpy()
        rel.append(float((np.linalg.norm(bn - A @ xn, axis=0) / np.linalg.norm(bn, axis=0)).max()))
    # the byte model of every system's solve (as for the headline: FP32 cycle, FP64-outer model
    # of the CG vectors) at its iteration count, summed: the batch's HBM floor
    from amjax_b200 import bytemodel
    model = sum(bytemodel.solve_bytes(bytemodel.level_stats(m), int(b.shape[1]), max(d["iterations"]),
                                      method="pcg", cycle_s=4, outer_s=8)
                for m, b, d in zip(mls, rhs, info))
    peak, _ = load_peaks()
    line = {"mode": "ragged", "metric": "ms per batch of 24 hierarchies (mixed PCG to 1e-8)",
            "value": tb, "unit": "ms/batch", "ms_min": tbmin, "sequential_ms": tsq,
            "speedup_vs_sequential": tsq / tb, "systems": 24,
            "bytes_model": model, "gbs_model_batch": model / (tbmin * 1e-3) / 1e9,
            "gbs_model_sequential": model / (tsqmin * 1e-3) / 1e9, "peak_gbs": peak,
            "rows": [A.shape[0] for A in mats], "rhs": [k for _, k in draws],
            "total_rows": int(sum(A.shape[0] for A in mats)), "total_rhs": int(sum(k for _, k in draws)),
            "iterations_max": [max(d["iterations"]) for d in info], "relres_fp64_max": max(rel),
            "host_setup_s": setup_s, "data": "synthetic"}
    print(json.dumps(line), flush=True)
    return 0


def run_cube(args):
    """Config 4: -div(kappa grad u) on 128^3 cells (N = 2,097,152), kappa = exp(g), g ~ N(0,1)
    from default_rng(2), harmonic face means, Dirichlet; SA; Jacobi 2/3; pinv.  Standalone
    solves to 1e-10: FP64 cycle vs FP32 cycle inside FP64 refinement, V / W / F, k = 1 and
    16.  True error against a direct solve on the 48^3 subsize."""
    import torch
    import scipy.sparse.linalg as spla
    from amjax_b200 import MultilevelSolver, amg_setup, gallery
    spec = ("jacobi", {"iterations": 1, "omega": 2.0 / 3.0})
    out = {"mode": "cube", "data": "synthetic", "tol": 1e-10}
    t0 = time.perf_counter()
    A = gallery.variable_diffusion_3d(128, sigma=1.0, seed=2)
    ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=spec, postsmoother=spec)
    out["host_setup_s"] = time.perf_counter() - t0
    out["levels"] = [l.A.shape[0] for l in ml.levels]
    res = {}
    for k in (1, 16):
        Bh = np.random.default_rng(2).standard_normal((A.shape[0], k) if k > 1 else A.shape[0])
        B = torch.as_tensor(Bh).cuda()
        for cyc in "VWF":
            for prec in ("f64", "mixed"):
                p = ml._precision(prec)
                f = lambda: ml._solve_dev(B, None, 1e-10, 300, cyc, 1, p)
                ms, msmin = _time_ms(f, max(2, args.steps // 3), 1)
                x, info = f()
                xn = x.cpu().numpy()
                r = np.linalg.norm((Bh - A @ xn).reshape(A.shape[0], -1), axis=0) / \
                    np.linalg.norm(Bh.reshape(A.shape[0], -1), axis=0)
                res[f"k{k}_{cyc}_{prec}"] = {"ms": ms, "iterations": max(info["iterations"]),
                                             "relres_fp64_max": float(r.max())}
    for k in (1, 16):
        for cyc in "VWF":
            a, b = res[f"k{k}_{cyc}_f64"]["ms"], res[f"k{k}_{cyc}_mixed"]["ms"]
            res[f"k{k}_{cyc}_speedup_mixed"] = a / b
    out["solves"] = res
    As = gallery.variable_diffusion_3d(48, sigma=1.0, seed=2)
    ms_ = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(As), presmoother=spec, postsmoother=spec)
    bs = np.random.default_rng(2).standard_normal(As.shape[0])
    xd = spla.splu(As.tocsc()).solve(bs)
    for prec in ("f64", "mixed"):
        xs = ms_.solve(bs, tol=1e-10, maxiter=300, precision=prec)
        out[f"err_vs_direct_48cube_{prec}"] = float(np.linalg.norm(xs - xd) / np.linalg.norm(xd))
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.ragged:
        return run_ragged(args)
    if args.cube:
        return run_cube(args)
    if args.kernel_only:
        return run_kernel_only(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
