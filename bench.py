#!/usr/bin/env python
"""Benchmark: AMEn time-to-1e-8 residual on one B200 (and N independent replicas).

Workload (one "step" = one full AMEn solve to tol 1e-8 from the same seeded
initial guess): d=10, n=64 anisotropic diffusion + separable reaction TT
operator (rank 3), seeded rank-4 Gaussian right-hand side, rmax 128,
amen_solve2 default options otherwise.  Inputs are synthetic (seeded numpy
PCG64), generated by ``ttgpu.workloads``.

Prints ONE JSON line (rank 0).  ``value`` is the device time of one solve
(CUDA events on the library's stream, inputs resident in HBM, L2 flushed
between steps); ``e2e`` is the same solve through the C ABI with host
buffers (upload + solve + download, host clock).  ``--impl reference`` times
the reference algorithm's CPU restatement (the FP64 oracle) instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tt-toolbox_b200"))

WORKLOAD = dict(d=10, n=64, rmax=128, tol=1e-8, seed=3)
METRIC = "AMEn time-to-1e-8 residual (d=10, n=64, rank-3 TT operator, rmax 128)"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-compare", action="store_true",
                   help="skip timing the other precision")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the rounding, gradient and batched configurations")
    p.add_argument("--no-batch", action="store_true",
                   help="skip the batched configuration in the configs block")
    p.add_argument("--workload", default="amen", choices=["amen", "batch"],
                   help="amen: the headline single solve; batch: 512 independent systems "
                        "(one timed batch; --steps/--warmup do not apply)")
    p.add_argument("--batch-count", type=int, default=512)
    p.add_argument("--batch-workers", type=int, default=8)
    p.add_argument("--batch-form", default="grouped", choices=["grouped", "streams"])
    p.add_argument("--batch-sample", type=int, default=32,
                   help="systems solved one by one (GPU FP64) and by the CPU oracle")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only: no data-path collective)
# ---------------------------------------------------------------------------

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            # The library is loaded before torch so that its CUDA 12.9
            # cuBLAS/cuSOLVER are the ones the process uses.
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group("gloo", timeout=timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# correctness check of the measured run (host numpy, outside the timed region)
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def load_peaks():
    try:
        with open(PEAKS_FILE) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def load_traffic():
    """The committed ncu figure (profiles/roofline_traffic.json): DRAM bytes
    of one BF16 local matvec at r = 64 (the solve's largest local system),
    or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def blas_threads():
    """Threads of the BLAS library numpy uses (what the CPU leg actually ran on)."""
    try:
        from threadpoolctl import threadpool_info
        n = [i["num_threads"] for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(n) if n else os.cpu_count()
    except Exception:
        return os.cpu_count()


def cpu_baseline_run(W, reps=1, threads=None):
    """The FP64 oracle (reference algorithm restated) on the same workload;
    ``threads`` caps the BLAS threads (1 matches the reference tests'
    ``maxNumCompThreads(1)``), None leaves all of them."""
    sys.path.insert(0, ROOT)
    from contextlib import nullcontext
    from oracle.amen import amen_solve2 as ref_solve
    from oracle.builders import aniso_config
    A, y, x0, z0 = aniso_config(d=W["d"], n=W["n"], seed=W["seed"])
    limit = nullcontext()
    if threads is not None:
        from threadpoolctl import threadpool_limits
        limit = threadpool_limits(threads)
    times = []
    info = None
    with limit:
        for _ in range(reps):
            t = time.perf_counter()
            x, info = ref_solve(A, y, W["tol"], x0, z0, rmax=W["rmax"], nswp=50)
            times.append(time.perf_counter() - t)
    return times, info


def single_thread_baseline(W):
    t1, info = cpu_baseline_run(W, reps=1, threads=1)
    return {"value": t1[0], "unit": "s", "cores": 1,
            "sample": "one full FP64 oracle solve, BLAS limited to one thread (%d sweeps)"
                      % info["sweeps"]}


def run_reference(args, dist):
    if dist.rank != 0:
        return None
    W = WORKLOAD
    n_total = args.warmup + args.steps
    times, info = cpu_baseline_run(W, reps=max(1, n_total))
    timed = times[-args.steps:] if args.steps > 0 else times
    v = statistics.mean(timed)
    cores = blas_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
        "config": {"workload": "amen_solve2 d=10 n=64 rank-3 anisotropic operator, rank-4 rhs, "
                               "rmax 128, tol 1e-8", "parallelism": "replicas", "sweeps": info["sweeps"]},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port",
                         "sample": "full FP64 oracle solve of the workload (numpy/OpenBLAS, all threads)",
                         "single_thread": single_thread_baseline(W)},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_ours(args, dist):
    import ttgpu
    from ttgpu import workloads
    ttgpu.lib()
    W = WORKLOAD
    dev = dist.local if dist.world > 1 else int(os.environ.get("TTG_DEVICE", "0"))
    ctx = ttgpu.Context(dev)
    A, y, x0, z0 = workloads.aniso(d=W["d"], n=W["n"], seed=W["seed"])
    dA, dy = ttgpu.DeviceTT.upload(ctx, A), ttgpu.DeviceTT.upload(ctx, y)
    dx0, dz0 = ttgpu.DeviceTT.upload(ctx, x0), ttgpu.DeviceTT.upload(ctx, z0)
    opts = dict(rmax=W["rmax"], nswp=50)

    def solve(prec, st, timing=False):
        out = ttgpu.amen_solve2(dA, dy, W["tol"], x0=dx0, z0=dz0, ctx=ctx, stats=st,
                                precision=prec, timing=timing, **opts)
        return out

    agg = {}

    def timed_steps(prec, K, timing=False):
        ms, launches, sweeps, gflop = [], 0, [], 0.0
        last = None
        acc = {"gflop_lp": 0.0, "ms_lp": 0.0, "gflop_fp64": 0.0, "ms_fp64": 0.0, "gbyte_lp": 0.0,
               "matvecs_lp": 0, "matvecs": 0}
        for _ in range(K):
            ctx.flush_l2()
            st = {}
            out = solve(prec, st, timing)
            ms.append(st["ms_total"])
            launches += st["launches"]
            sweeps.append(st["sweeps"])
            gflop += st["matvec_gflop"]
            for k in acc:
                acc[k] += st[k]
            if last is not None:
                last.free()
            last = out
        agg[prec] = acc
        return ms, launches, sweeps, gflop, last

    for _ in range(args.warmup):
        st = {}
        solve(args.precision, st).free()
    dist.barrier()
    ctx.sync()
    clocks = Clocks(dev)
    clocks.start()
    t0 = time.perf_counter()
    # The headline solves run without per-matvec events; the roofline comes
    # from a separate instrumented solve after the timed region.
    ms, launches, sweeps, gflop, xdev = timed_steps(args.precision, args.steps)
    ctx.sync()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    dist.barrier()
    # Instrumented pass (outside the timed region): every local matvec is
    # bracketed by CUDA events on the library's stream.
    timed_steps(args.precision, 1, timing=True)[-1].free()
    ms_step = statistics.mean(ms)
    ms_step_max = dist.max(ms_step)
    x = xdev.download()
    xdev.free()
    res = ttgpu.true_residual(A, x, y, ctx=ctx)

    # end to end through the C ABI with host buffers
    e2e_t = []
    h2d = 8 * (A.core.size + y.core.size + x0.core.size + z0.core.size)
    d2h = 0
    for _ in range(max(1, args.steps)):
        ctx.flush_l2()
        t = time.perf_counter()
        xh = ttgpu.amen_solve2(A, y, W["tol"], x0=x0, z0=z0, ctx=ctx, precision=args.precision,
                               **opts)
        e2e_t.append(time.perf_counter() - t)
        d2h = 8 * xh.core.size
    e2e_v = dist.max(statistics.mean(e2e_t))

    other = None
    if not args.no_compare:
        op = "fp64" if args.precision == "mixed" else "mixed"
        try:
            oms, _, osw, _, ox = timed_steps(op, args.steps)
            xo = ox.download()
            ox.free()
            timed_steps(op, 1, timing=True)[-1].free()
            a = agg[op]
            other = {"precision": op, "ms_per_step": statistics.mean(oms), "sweeps": osw,
                     "true_residual": ttgpu.true_residual(A, xo, y, ctx=ctx),
                     "speedup_of_headline": statistics.mean(oms) / ms_step}
            if a["ms_fp64"] > 0:
                other["fp64_matvec_tflops"] = a["gflop_fp64"] / a["ms_fp64"]
        except ttgpu.TTGError as e:
            other = {"precision": op, "unavailable": str(e)}

    peaks, peaks_kind = load_peaks()
    a = agg[args.precision]
    if args.precision == "mixed" and a["ms_lp"] > 0:
        # BF16 tcgen05 local matvec: average over the solve's matvecs of
        # algorithmic FLOPs (and bytes) per launch / CUDA-event duration.
        nlp = max(1, a["matvecs_lp"])
        per_launch_tflop = a["gflop_lp"] / nlp * 1e-3
        per_launch_ms = a["ms_lp"] / nlp
        alg_bytes = a["gbyte_lp"] / nlp * 1e9
        achieved = per_launch_tflop / (per_launch_ms * 1e-3)
        peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1590.0))
        tr = load_traffic()
        fused = os.environ.get("TTG_FUSED_MV", "0") == "1"
        # ncu measures one fixed shape; its DRAM bytes over the algorithmic
        # bytes of that shape, times the in-solve algorithmic bytes per
        # launch, gives the in-solve traffic (DRAM traffic of this kernel
        # scales with the operand and result sizes).
        traffic = None
        form = "fused" if fused else "split"
        ratio = (tr.get("ratio") or {}).get(form) if tr else None
        if ratio:
            traffic = ratio * alg_bytes
        roof = {"kernel": ("local matvec, BF16 tcgen05, one persistent launch (k_mv_fused)"
                           if fused else "local matvec, BF16 tcgen05, three GEMM launches"),
                "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic,
                "traffic_basis": (("ncu DRAM bytes / algorithmic bytes = %.3f at %s, times the "
                                   "in-solve algorithmic bytes per launch"
                                   % (ratio, tr.get("shape"))) if traffic else None),
                "alg_bytes_per_launch": alg_bytes,
                "hbm_gbs_per_launch": alg_bytes / (per_launch_ms * 1e-3) * 1e-9,
                "peak_kind": "bf16 sustained, %s" % peaks_kind,
                "launch_ms": per_launch_ms, "gflop_per_launch": per_launch_tflop * 1e3}
    else:
        per_launch_ms = a["ms_fp64"] / max(1, a["matvecs"])
        achieved = a["gflop_fp64"] / max(a["ms_fp64"], 1e-9)
        roof = {"kernel": "local matvec, FP64 DMMA (3 launches)", "bound": "tensor",
                "achieved": achieved, "peak": None, "unit": "TFLOP/s", "frac": None,
                "traffic": None, "peak_kind": "no measured FP64 peak", "launch_ms": per_launch_ms}
    line = {
        "metric": METRIC, "value": ms_step_max / 1e3, "unit": "s", "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step_max,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "bf16/f32 matvec + f64 refinement",
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": "amen_solve2 d=10 n=64 rank-3 anisotropic operator, rank-4 rhs, "
                               "rmax 128, tol 1e-8", "precision": args.precision,
                   "parallelism": "replicas" if dist.world > 1 else "single",
                   "l2": "flushed between steps (256 MiB memset)",
                   "sweeps": sweeps, "true_residual": res},
        "e2e": {"value": e2e_v, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk,
        "matvec_gflop_per_step": gflop / max(1, args.steps),
        "wall_s_timed": wall,
        "peaks_source": peaks_kind,
    }
    if other is not None:
        line["compare"] = other
    if dist.rank == 0 and not args.no_configs:
        # The other configurations of the hot path, measured in the same run
        # (not part of the headline value).
        line["configs"] = {"round": run_round_config(ctx, cpu=dist.world == 1
                                                     and not args.no_cpu_baseline),
                           "grad": run_grad_config(ctx)}
        if not args.no_batch:
            bargs = argparse.Namespace(batch_count=args.batch_count,
                                       batch_workers=args.batch_workers,
                                       batch_form=args.batch_form,
                                       batch_sample=min(args.batch_sample, 16),
                                       no_cpu_baseline=args.no_cpu_baseline or dist.world > 1)
            line["configs"]["batch"] = run_batch(bargs, dist)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        times, info = cpu_baseline_run(W, reps=1)
        line["cpu_baseline"] = {"value": times[0], "unit": "s", "cores": blas_threads(),
                                "kind": "port",
                                "sample": "one full FP64 oracle solve of the same workload "
                                          "(numpy/OpenBLAS, all threads; %d sweeps)" % info["sweeps"],
                                "single_thread": single_thread_baseline(W)}
    for h in (dA, dy, dx0, dz0):
        h.free()
    ctx.close()
    return line


def round_flops(n, r):
    """Algorithmic FLOPs of rounding a TT with mode sizes n and ranks r: per
    core the left-to-right QR (4 m p^2 - 4/3 p^3, m = r_k n_k, p = r_{k+1}) and
    R * core product, the right-to-left SVD of the r_k x (n_k r_{k+1})
    unfolding (6 (n r) r^2 + 20 r^3, QR-based) and the core * (U S) product."""
    d = len(n)
    fl = 0.0
    for k in range(d - 1):
        m, p = r[k] * n[k], r[k + 1]
        fl += 4.0 * m * p * p - 4.0 / 3.0 * p ** 3 + 2.0 * p * p * n[k + 1] * r[k + 2]
    for k in range(d - 1, 0, -1):
        rk, cols = r[k], n[k] * r[k + 1]
        fl += 6.0 * cols * rk * rk + 20.0 * rk ** 3 + 2.0 * r[k - 1] * n[k - 1] * rk * rk
    return fl


def run_round_config(ctx, reps=3, cpu=True):
    """Rounding of the sum of four rank-64 Gaussian TTs (d=20, n=16, internal
    ranks 256) to eps 1e-8 on the device: the FP64 form and the mixed form
    (R * core and core * (U S) on BF16 tensor cores, FP64 QR/SVD)."""
    import ttgpu
    from ttgpu import workloads
    W = dict(d=20, n=16, r=64, terms=4, seed=2, eps=1e-8)
    X = workloads.round_input(d=W["d"], n=W["n"], r=W["r"], terms=W["terms"], seed=W["seed"])
    dX = ttgpu.DeviceTT.upload(ctx, X)
    fl = round_flops([int(v) for v in X.n], [int(v) for v in X.r])
    out = {"workload": "round: d=20 n=16, sum of 4 rank-64 Gaussian TTs (ranks 256), eps 1e-8",
           "gflop": fl * 1e-9}
    xnorm = ttgpu.tt_norm(dX, ctx=ctx)
    for prec in ("fp64", "mixed"):
        ms, st = [], {}
        Y = None
        for it in range(reps + 1):
            if Y is not None:
                Y.free()
            ctx.flush_l2()
            st = {}
            Y = ttgpu.round(dX, W["eps"], precision=prec, ctx=ctx, stats=st)
            if it:
                ms.append(st["ms_total"])
        ranks = [int(v) for v in Y.shape()[2]]
        D = ttgpu.tt_axpby(1.0, Y, -1.0, dX, ctx=ctx)
        err = ttgpu.tt_norm(D, ctx=ctx) / xnorm
        D.free()
        Y.free()
        v = statistics.median(ms) * 1e-3
        out[prec] = {"value": v, "unit": "s", "gflops": fl / v * 1e-9,
                     "ms_qr_sweep": st["ms_qr_sweep"], "ms_svd_sweep": st["ms_svd_sweep"],
                     "ranks_max": max(ranks), "rel_err": err}
    t0 = time.perf_counter()
    ttgpu.round(X, W["eps"], ctx=ctx)
    out["fp64"]["e2e_s"] = time.perf_counter() - t0
    dX.free()
    if cpu:
        sys.path.insert(0, ROOT)
        from oracle.builders import round_config
        from oracle.round import tt_round
        Xo = round_config(d=W["d"], n=W["n"], r=W["r"], terms=W["terms"], seed=W["seed"])
        t0 = time.perf_counter()
        tt_round(Xo, W["eps"])
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": cpu_s, "unit": "s", "cores": blas_threads(),
                               "kind": "port", "sample": "one full FP64 oracle rounding"}
    return out


def run_grad_config(ctx, reps=5):
    """Gradients of <x,Ax>, <x,b> and the 1e6-sample loss with respect to every
    core (d=12, n=32, rank-64 x, rank-3 operator), FP64 on the device."""
    import ttgpu
    from ttgpu import workloads
    x, A, b, idx, y = workloads.grad_inputs()
    dx, dA, db = (ttgpu.DeviceTT.upload(ctx, t) for t in (x, A, b))
    ss = ttgpu.SampleSet(ctx, idx, y)
    g = ttgpu.DeviceArray(ctx, None, x.core.size)
    out = {"workload": "grad: d=12 n=32 rank-64 x, rank-3 operator, rank-4 b, 1e6 samples"}
    runs = [("xAx", lambda: ttgpu.grad_xAx(dx, dA, ctx=ctx, out=g)),
            ("xb", lambda: ttgpu.grad_xb(dx, db, ctx=ctx, out=g)),
            ("sampled", lambda: ttgpu.grad_sampled(dx, ss, ctx=ctx, out=g))]
    for name, fn in runs:
        fn()
        ctx.sync()
        ts = []
        for _ in range(reps):
            ctx.flush_l2()
            ctx.sync()
            t0 = time.perf_counter()
            fn()
            ctx.sync()
            ts.append(time.perf_counter() - t0)
        out[name + "_ms"] = statistics.median(ts) * 1e3
    g.free()
    ss.free()
    for h in (dx, dA, db):
        h.free()
    return out


BATCH_METRIC = "batched AMEn: independent Laplacian systems to tol 1e-8, total time"


def run_batch(args, dist):
    """``count`` independent seeded Laplacian systems (d U{6..14},
    n in {8,16,32,64}, rmax U{8..64}, all-ones right-hand sides, tol 1e-8)
    through the grouped batch ``ttg_amen_solve_grouped`` (every system's
    launches merged kernel by kernel into grouped launches), mixed precision
    (the value) and FP64, against the same systems solved one after another
    in FP64 on the GPU and by the CPU oracle (both on the first
    ``batch_sample`` systems, scaled to the whole batch by count).
    ``--batch-form streams`` times ``ttg_amen_solve_batch`` (worker host
    threads, one stream each) instead."""
    if dist.rank != 0:
        return None
    import numpy as np
    import ttgpu
    from ttgpu import workloads
    ctx = ttgpu.Context(int(os.environ.get("TTG_DEVICE", "0")))
    As, ys, rmaxs, shapes = workloads.batch_systems(count=args.batch_count, seed=4)
    dAs = [ttgpu.DeviceTT.upload(ctx, a) for a in As]
    dys = [ttgpu.DeviceTT.upload(ctx, y) for y in ys]
    per = [dict(rmax=r) for r in rmaxs]
    k = min(args.batch_sample, args.batch_count)
    grouped = args.batch_form == "grouped"
    width = 0 if grouped else args.batch_workers

    def run(prec, lo=0, hi=None, stats=None, gs=None):
        hi = len(dAs) if hi is None else hi
        return ttgpu.amen_solve2_batch(dAs[lo:hi], dys[lo:hi], 1e-8, workers=width, ctx=ctx,
                                       stats=stats, per_system=per[lo:hi], precision=prec,
                                       grouped=grouped, group_stats=gs)

    # warm-up: kernels loaded, tile widths tuned and allocator slabs grown
    for prec in ("mixed", "fp64"):
        for x in run(prec, 0, 32):
            x.free()
    ctx.sync()
    forms = {}
    clk = None
    res, conv, st_mixed = [], 0, None
    for prec in ("mixed", "fp64"):
        if prec == "mixed":
            clocks = Clocks(0)
            clocks.start()
        st, gs = [], {}
        t0 = time.perf_counter()
        xs = run(prec, stats=st, gs=gs)
        ctx.sync()
        wall = time.perf_counter() - t0
        # grouped: launches the executor issued; streams: each solve's own
        launches = gs["launches"] if grouped else sum(q["launches"] for q in st)
        if prec == "mixed":
            clk = clocks.stop()
            st_mixed = st
        c = sum(1 for q in st if q["sweeps"] and q["max_res"][q["sweeps"] - 1] < 1e-8)
        gflop = sum(q["matvec_gflop"] for q in st)
        rs = [ttgpu.true_residual(dAs[i], xs[i], dys[i], ctx=ctx) for i in range(k)]
        for x in xs:
            x.free()
        forms[prec] = {"value": wall, "unit": "s", "converged": c,
                       "true_residual_max_of_sample": max(rs), "gpu_launches": launches,
                       "recorded_launches": gs.get("records"),
                       "matvec_gflop": gflop, "matvec_tflops": gflop / wall * 1e-3}
        if grouped:  # where the executor's time went (host ms, summed over threads)
            forms[prec]["executor"] = {k: gs[k] for k in (
                "flushes", "grouped_records", "ms_record", "ms_plan", "ms_issue",
                "ms_issue_wait", "ms_alloc", "lanes_max", "tc_launches", "tc_records")}
        if prec == "mixed":
            res, conv = rs, c
    wall = forms["mixed"]["value"]
    roof = None
    if grouped:
        # Instrumented pass (outside the timed region): CUDA events around
        # every grouped launch of the BF16 tcgen05 GEMM (the local matvec
        # stages), each launch carrying the GEMMs of many systems.
        os.environ["TTG_GROUP_TIME"] = "1"
        try:
            gs = {}
            for x in run("mixed", gs=gs):
                x.free()
        finally:
            os.environ.pop("TTG_GROUP_TIME", None)
        if gs.get("tc_ms", 0) > 0 and gs.get("tc_launches", 0) > 0:
            peaks, peaks_kind = load_peaks()
            peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1590.0))
            achieved = gs["tc_gflop"] / gs["tc_ms"]  # GFLOP/ms = TFLOP/s
            roof = {"kernel": "grouped BF16 tcgen05 GEMM launches (k_umma_group: the local "
                              "matvec stages of many systems per launch)",
                    "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "peak_kind": "bf16 sustained, %s" % peaks_kind,
                    "launches": gs["tc_launches"], "gemms": gs["tc_records"],
                    "gemms_per_launch": gs["tc_records"] / gs["tc_launches"],
                    "gflop_per_launch": gs["tc_gflop"] / gs["tc_launches"],
                    "launch_ms": gs["tc_ms"] / gs["tc_launches"],
                    "note": "event-timed launches on concurrent lanes (contention included); "
                            "algorithmic FLOPs of the GEMMs that ran (skipped Krylov steps "
                            "taken out)"}
    # systems that stop short of 1e-8: at their rank cap or the sweep limit
    capped = [i for i, q in enumerate(st_mixed)
              if not (q["sweeps"] and q["max_res"][q["sweeps"] - 1] < 1e-8)]
    t0 = time.perf_counter()
    for i in range(k):
        ttgpu.amen_solve2(dAs[i], dys[i], 1e-8, ctx=ctx, rmax=rmaxs[i], precision="fp64").free()
    ctx.sync()
    serial = (time.perf_counter() - t0) / k * args.batch_count
    line = {
        "metric": BATCH_METRIC, "value": wall, "unit": "s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": wall * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16/f32 matvec + f64 refinement",
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": "%d Laplacian systems, d U{6..14}, n in {8,16,32,64}, rmax "
                               "U{8..64}, ones rhs, tol 1e-8" % args.batch_count,
                   "form": ("grouped launches (ttg_amen_solve_grouped)" if grouped else
                            "worker streams (ttg_amen_solve_batch, %d workers)"
                            % args.batch_workers),
                   "converged": conv, "stopped_short": len(capped),
                   "true_residual_max_of_sample": max(res)},
        "gpu_launches": forms["mixed"]["gpu_launches"],
        "matvec_tflops": forms["mixed"]["matvec_tflops"], "clocks": clk,
        "roofline": roof,
        "forms": forms,
        "compare": {"serial_fp64_gpu_s": serial,
                    "speedup_vs_serial_fp64_gpu": serial / wall,
                    "speedup_vs_same_form_fp64": forms["fp64"]["value"] / wall,
                    "sample": "first %d systems one by one, scaled by count" % k},
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle.amen import amen_solve2 as ref_solve
        from oracle.tt import TT, TTMatrix, tt_randn
        t0 = time.perf_counter()
        kc = max(1, k // 4)
        for i in range(kc):
            A, y = As[i], ys[i]
            Ao = TTMatrix.from_flat(A.n, A.m, A.r, A.core)
            yo = TT.from_flat(y.n, y.r, y.core)
            rng = np.random.default_rng(i)
            x0 = tt_randn([int(v) for v in A.n], A.d, 2, rng)
            ref_solve(Ao, yo, 1e-8, x0, None, rmax=rmaxs[i], nswp=20)
        cpu = (time.perf_counter() - t0) / kc * args.batch_count
        line["cpu_baseline"] = {"value": cpu, "unit": "s", "cores": blas_threads(),
                                "kind": "port",
                                "sample": "FP64 oracle on the first %d systems, scaled by count"
                                          % kc}
    for h in dAs + dys:
        h.free()
    ctx.close()
    return line


def main():
    args = parse()
    if args.impl == "ours":
        import ttgpu
        ttgpu.lib()  # before torch (see Dist)
    dist = Dist()
    try:
        if args.workload == "batch":
            line = run_batch(args, dist) if args.impl == "ours" else None
        else:
            line = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
        if dist.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
