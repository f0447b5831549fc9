"""Fixed-shape runs of the hot kernels through the C ABI.

``python -m ttgpu.kernel_bench matvec --r 64 --n 64 --ra 3 --reps 20``
    runs ``ttg_local_matvec`` (``bfun3``, ``solve/amen_solve2.m:924-951``) on
    seeded operands of one shape, in FP64 and in mixed (BF16 tcgen05)
    precision, and prints the mean wall time per call.  The call is
    synchronous, so the time includes the call's own conversions (FP64 ->
    BF16 operands, natural <-> reversed vector layout) and one stream
    synchronisation; it is the target of the kernel-level ncu captures.

``python -m ttgpu.kernel_bench round --d 20 --n 16 --r 64 --terms 4``
    rounds a sum of ``terms`` rank-``r`` Gaussian TTs (``@tt_tensor/round.m``)
    on the device and prints the time, ranks and the relative error of the
    rounded tensor against the input.

``python -m ttgpu.kernel_bench grad --d 12 --n 32 --r 64 --samples 1000000``
    gradients of <x,Ax>, <x,b> and the sampled-entry loss with respect to
    every core, inputs resident on the device; time and FLOP/s (parity at
    this size is checked in the GPU tests).

``python -m ttgpu.kernel_bench batch --count 512 --workers 8``
    the batched AMEn workload (uneven d, n, rmax; Laplacian systems, ones
    right-hand sides, tol 1e-8) through ``ttg_amen_solve_batch``, against
    the same systems solved one after another (the first ``--serial``).

``python -m ttgpu.kernel_bench amen --precision fp64,mixed``
    one solve of the anisotropic d=10, n=64 workload per precision (set
    TTG_PROFILE=1 for the per-phase breakdown on stderr).  With
    ``--kernel-table`` the last repetition runs under the CUDA activity
    tracer (CUPTI through ``torch.profiler``): per kernel its launches and
    device time in that warm solve, the idle gaps between consecutive
    kernels, and the top launch shapes (grid, block, shared memory).

``python -m ttgpu.kernel_bench svd --n 256,160,64``
    the device SVD (``ttg_dense_svd``; square inputs go straight to the
    Jacobi kernels) of seeded n x n Gaussian matrices: time per SVD, and the
    time of one sweep alone (sweep limit 1, the call then reports its
    non-convergence), so that time / sweep time estimates the sweeps run.

``python -m ttgpu.kernel_bench dgemm``
    cuBLAS FP64 GEMM throughput (torch.matmul, 8192^3) as the measured FP64
    tensor-core reference for the FP64 kernels.
"""

import argparse
import json
import time

import numpy as np

from . import (Context, DeviceArray, DeviceTT, _check, _PREC, lib, round as tt_round,
               workloads)


def matvec(args):
    ctx = Context(args.device)
    rng = np.random.default_rng(args.seed)
    r1 = r2 = args.r
    n, ra = args.n, args.ra
    P1 = DeviceArray(ctx, rng.standard_normal(r1 * r1 * ra))
    A = DeviceArray(ctx, rng.standard_normal(ra * n * n * ra))
    P2 = DeviceArray(ctx, rng.standard_normal(r2 * ra * r2))
    x = DeviceArray(ctx, rng.standard_normal(r1 * n * r2))
    y = DeviceArray(ctx, None, r1 * n * r2)
    flops = 2.0 * n * r1 * r2 * (r1 * ra + ra * ra * n + r2 * ra)
    out = {"shape": {"r1": r1, "n": n, "r2": r2, "ra1": ra, "ra2": ra}, "gflop": flops * 1e-9}
    for prec in args.precision.split(","):
        def call():
            _check(lib().ttg_local_matvec(ctx.h, r1, n, r2, ra, ra, P1.p, A.p, P2.p, x.p, y.p,
                                          _PREC[prec]))
        for _ in range(3):
            call()
        ctx.sync()
        t = time.perf_counter()
        for _ in range(args.reps):
            call()
        ctx.sync()
        ms = (time.perf_counter() - t) / args.reps * 1e3
        out[prec] = {"ms_per_call": ms, "tflops_per_call": flops / (ms * 1e-3) * 1e-12}
    print(json.dumps(out))
    ctx.close()


def round_bench(args):
    ctx = Context(args.device)
    X = workloads.round_input(d=args.d, n=args.n, r=args.r, terms=args.terms, seed=args.seed)
    dX = DeviceTT.upload(ctx, X)
    out = {"workload": "round: d=%d n=%d, sum of %d rank-%d Gaussian TTs, eps=%g"
                       % (args.d, args.n, args.terms, args.r, args.eps)}
    for prec in args.precision.split(","):
        times, st = [], {}
        for it in range(args.reps + 1):
            ctx.flush_l2()
            ctx.sync()
            t = time.perf_counter()
            Y = tt_round(dX, args.eps, precision=prec, ctx=ctx, stats=st)
            ctx.sync()
            if it:
                times.append(time.perf_counter() - t)
            if it < args.reps:
                Y.free()
        r = Y.shape()[2]
        Yh = Y.download()
        Y.free()
        out[prec] = {"ms": float(np.median(times)) * 1e3, "ranks": [int(v) for v in r],
                     "ms_qr_sweep": st["ms_qr_sweep"], "ms_svd_sweep": st["ms_svd_sweep"]}
        if args.check:
            out[prec]["rel_err"] = _rel_diff(X, Yh)
        if args.kernel_table:
            out[prec]["kernel_table"] = _kernel_table(
                lambda: tt_round(dX, args.eps, precision=prec, ctx=ctx).free())
    tables = {p: out[p].pop("kernel_table") for p in list(out) if isinstance(out[p], dict)
              and "kernel_table" in out[p]}
    print(json.dumps(out))
    for prec, tab in tables.items():
        print("\n# kernels of one rounding, precision %s\n%s" % (prec, tab))
    dX.free()
    ctx.close()


def _time(ctx, fn, reps):
    fn()
    ctx.sync()
    ts = []
    for _ in range(reps):
        ctx.flush_l2()
        ctx.sync()
        t = time.perf_counter()
        fn()
        ctx.sync()
        ts.append(time.perf_counter() - t)
    return float(np.median(ts)) * 1e3


def grad_bench(args):
    from . import SampleSet, grad_sampled, grad_xAx, grad_xb
    ctx = Context(args.device)
    x, A, b, idx, y = workloads.grad_inputs(d=args.d, n=args.n, r=args.r, nsamples=args.samples,
                                            seed=args.seed)
    dx, dA, db = DeviceTT.upload(ctx, x), DeviceTT.upload(ctx, A), DeviceTT.upload(ctx, b)
    ss = SampleSet(ctx, idx, y)
    g = DeviceArray(ctx, None, x.core.size)
    r, n, ra, rb = list(x.r), list(x.n), list(A.r), list(b.r)
    d = len(n)
    f_mv = [2.0 * n[k] * r[k] * r[k + 1] * (r[k] * ra[k + 1] + ra[k] * ra[k + 1] * n[k]
                                             + r[k + 1] * ra[k]) for k in range(d)]
    # two interface sweeps (d updates each, same flop formula) + two local matvecs per core
    fl_xAx = 2 * sum(f_mv) + 2 * sum(f_mv)
    fl_xb = sum(2.0 * n[k] * (r[k] * rb[k] * rb[k + 1] + 2 * r[k] * r[k + 1] * rb[k + 1]
                              + rb[k] * rb[k + 1] * r[k + 1] + r[k] * rb[k] * r[k + 1])
                for k in range(d))
    fl_s = 6.0 * args.samples * sum(r[k] * r[k + 1] for k in range(d))
    out = {"workload": "grad: d=%d n=%d rank-%d x, rank-3 operator, rank-%d b, %d samples"
                       % (args.d, args.n, args.r, rb[1], args.samples)}
    runs = [("xAx", lambda: grad_xAx(dx, dA, ctx=ctx, out=g), fl_xAx),
            ("xb", lambda: grad_xb(dx, db, ctx=ctx, out=g), fl_xb),
            ("sampled", lambda: grad_sampled(dx, ss, ctx=ctx, out=g), fl_s)]
    for name, fn, fl in runs:
        ms = _time(ctx, fn, args.reps)
        out[name] = {"ms": ms, "gflop": fl * 1e-9, "tflops": fl / (ms * 1e-3) * 1e-12}
    print(json.dumps(out))
    g.free()
    ss.free()
    for h in (dx, dA, db):
        h.free()
    ctx.close()


def batch_bench(args):
    from . import amen_solve2, amen_solve2_batch
    ctx = Context(args.device)
    As, ys, rmaxs, shapes = workloads.batch_systems(count=args.count, seed=args.seed)
    dAs = [DeviceTT.upload(ctx, a) for a in As]
    dys = [DeviceTT.upload(ctx, y) for y in ys]
    per = [dict(rmax=r) for r in rmaxs]
    out = {"workload": "batch: %d Laplacian systems, d U{6..14}, n in {8,16,32,64}, "
                       "rmax U{8..64}, ones rhs, tol %g" % (args.count, args.tol),
           "workers": args.workers}
    tables = {}
    for prec in args.precision.split(","):
        st = []
        ctx.sync()
        t = time.perf_counter()
        gs = {}
        res = {}

        def run():
            res["xs"] = amen_solve2_batch(dAs, dys, args.tol, workers=args.workers, ctx=ctx,
                                          stats=st, per_system=per, precision=prec,
                                          grouped=args.grouped, group_stats=gs)
            ctx.sync()

        table = None
        if args.kernel_table:
            table = _kernel_table(run)
        else:
            run()
        xs = res["xs"]
        wall = time.perf_counter() - t
        conv = sum(1 for s in st if s["sweeps"] and s["max_res"][s["sweeps"] - 1] < args.tol)
        fl = sum(s["matvec_gflop"] for s in st)
        for x in xs:
            x.free()
        k = min(args.serial, args.count)
        t = time.perf_counter()
        for i in range(k):
            amen_solve2(dAs[i], dys[i], args.tol, ctx=ctx, rmax=rmaxs[i], precision=prec).free()
        ctx.sync()
        ser = time.perf_counter() - t
        out[prec] = {"batch_s": wall, "converged": conv, "matvec_gflop": fl,
                     "matvec_tflops": fl / wall * 1e-3}
        if table is not None:
            tables[prec] = table
        if args.grouped:
            out[prec]["group"] = gs
            if gs.get("tc_ms"):
                out[prec]["tc_tflops_per_launch"] = gs["tc_gflop"] / gs["tc_ms"]
        if k:
            out[prec].update(serial_first_k_s=ser, serial_k=k,
                             batch_speedup_est=(ser / k * args.count) / wall)
    print(json.dumps(out))
    for prec, tab in tables.items():
        print("\n# kernels of the batch, precision %s\n%s" % (prec, tab))
    for h in dAs + dys:
        h.free()
    ctx.close()


def amen_bench(args):
    from . import amen_solve2
    ctx = Context(args.device)
    A, y, x0, z0 = workloads.aniso(d=args.d, n=args.n, seed=3)
    dA, dy = DeviceTT.upload(ctx, A), DeviceTT.upload(ctx, y)
    dx0, dz0 = DeviceTT.upload(ctx, x0), DeviceTT.upload(ctx, z0)
    out = {"workload": "amen_solve2 aniso d=%d n=%d rmax %d tol %g" % (args.d, args.n, args.rmax,
                                                                     args.tol)}
    tables = {}
    for prec in args.precision.split(","):
        for rep in range(args.reps):
            st = {}

            def solve():
                x = amen_solve2(dA, dy, args.tol, x0=dx0, z0=dz0, ctx=ctx, stats=st,
                                rmax=args.rmax, nswp=50, precision=prec, timing=args.timing)
                ctx.sync()
                x.free()

            if args.kernel_table and rep == args.reps - 1:
                tables[prec] = _kernel_table(solve)
            else:
                solve()
        out[prec] = {k: st[k] for k in ("ms_total", "sweeps", "matvecs", "matvecs_fp64",
                                        "gmres_iters", "launches", "max_rank")}
        if args.timing:  # per-matvec CUDA events: average in-solve matvec
            n_lp = max(1, st["matvecs_lp"])
            out[prec]["lp_matvec_us"] = st["ms_lp"] / n_lp * 1e3
            out[prec]["lp_matvec_gflop"] = st["gflop_lp"] / n_lp
            out[prec]["fp64_matvec_us"] = st["ms_fp64"] / max(1, st["matvecs_fp64"]) * 1e3
    print(json.dumps(out))
    for prec, tab in tables.items():
        print("\n# kernels of one warm solve, precision %s\n%s" % (prec, tab))
    for h in (dA, dy, dx0, dz0):
        h.free()
    ctx.close()


def _kernel_table(run, top=30, top_shapes=25):
    """Run ``run()`` under the CUDA activity tracer and summarise its kernels."""
    import collections
    import os
    import re
    import tempfile

    import torch
    from torch.profiler import ProfilerActivity, profile

    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        run()
        torch.cuda.synchronize()
    fd, path = tempfile.mkstemp(suffix=".json")
    os.close(fd)
    try:
        prof.export_chrome_trace(path)
        with open(path) as f:
            events = [e for e in json.load(f)["traceEvents"] if e.get("cat") == "kernel"]
    finally:
        os.remove(path)

    def short(name):
        name = name.replace("(anonymous namespace)::", "").replace("ttg::", "")
        name = re.sub(r"^void ", "", name)
        # cut at the parameter list: the first '(' outside template brackets
        depth = 0
        for i, ch in enumerate(name):
            if ch == "<":
                depth += 1
            elif ch == ">":
                depth -= 1
            elif ch == "(" and depth == 0:
                name = name[:i]
                break
        # grouped / plain entries of a kernel body: name the body
        m = re.match(r"k_(plain|group)_(?:no)?lb<&\(?(\w+?)_body(<[^>]*>)?", name)
        if m:
            return "%s%s%s" % (m.group(2), m.group(3) or "", " [grouped]" if m.group(1) == "group"
                                else "")
        return name

    tot, cnt = collections.defaultdict(float), collections.Counter()
    shp, shc = collections.defaultdict(float), collections.Counter()
    for e in events:
        k = short(e["name"])
        tot[k] += e["dur"]
        cnt[k] += 1
        a = e.get("args", {})
        key = "%s grid=%s block=%s smem=%s" % (k, a.get("grid"), a.get("block"),
                                               a.get("shared memory"))
        shp[key] += e["dur"]
        shc[key] += 1
    spans = sorted((e["ts"], e["ts"] + e["dur"]) for e in events)
    busy = sum(tot.values())
    span = spans[-1][1] - spans[0][0] if spans else 0.0
    gaps = [max(0.0, b[0] - a[1]) for a, b in zip(spans, spans[1:])]
    edges = [0, 2, 5, 10, 20, 50, 100, float("inf")]
    lines = ["launches %d, kernel time %.2f ms, first-to-last span %.2f ms (idle %.2f ms)"
             % (len(events), busy / 1e3, span / 1e3, (span - busy) / 1e3)]
    lines.append("idle gaps between consecutive kernels (us): " + ", ".join(
        "[%g,%g) %d = %.1f ms" % (lo, hi, sum(1 for g in gaps if lo <= g < hi),
                                  sum(g for g in gaps if lo <= g < hi) / 1e3)
        for lo, hi in zip(edges, edges[1:])))
    lines.append("| kernel | launches | total ms | share | us/launch |")
    lines.append("|---|---:|---:|---:|---:|")
    for k, v in sorted(tot.items(), key=lambda kv: -kv[1])[:top]:
        lines.append("| `%s` | %d | %.2f | %.1f%% | %.2f |" % (k[:70], cnt[k], v / 1e3,
                                                               100 * v / busy, v / cnt[k]))
    lines.append("\n| launch shape | launches | total ms | us/launch |")
    lines.append("|---|---:|---:|---:|")
    for k, v in sorted(shp.items(), key=lambda kv: -kv[1])[:top_shapes]:
        lines.append("| `%s` | %d | %.2f | %.2f |" % (k[:100], shc[k], v / 1e3, v / shc[k]))
    return "\n".join(lines)


def svd_bench(args):
    from . import TTGError, dense_svd
    ctx = Context(args.device)
    rng = np.random.default_rng(args.seed)
    out = {"workload": "device SVD of seeded n x n Gaussian matrices"}
    for n in [int(v) for v in args.n.split(",")]:
        A = rng.standard_normal((n, n))
        dense_svd(A, ctx=ctx)
        ts = []
        for _ in range(args.reps):
            t0 = time.perf_counter()
            dense_svd(A, ctx=ctx)
            ts.append(time.perf_counter() - t0)
        ctx.set_option(Context.OPT_JACOBI_MAX_SWEEPS, 1)
        t1 = []
        try:
            for _ in range(args.reps):
                t0 = time.perf_counter()
                try:
                    dense_svd(A, ctx=ctx)
                except TTGError:
                    pass
                t1.append(time.perf_counter() - t0)
        finally:
            ctx.set_option(Context.OPT_JACOBI_MAX_SWEEPS, 40)
        med, med1 = float(np.median(ts)), float(np.median(t1))
        out[str(n)] = {"ms": med * 1e3, "ms_one_sweep": med1 * 1e3,
                       "sweeps_est": med / med1 if med1 > 0 else None,
                       "us_per_round_est": med1 * 1e6 / max(1, n - 1 + n % 2)}
    print(json.dumps(out))
    ctx.close()


def dgemm_bench(args):
    import torch
    n = args.size
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(3):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(args.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    print(json.dumps({"dgemm": {"n": n, "ms": best, "tflops": 2.0 * n ** 3 / (best * 1e-3) * 1e-12}}))


def _rel_diff(X, Y):
    """||Y - X|| / ||X|| in FP64 on the host: the difference as one TT (rank
    concatenation) orthogonalised left to right; the norm is that of the last
    core.  (An inner-product formula would lose everything below 1e-8 to
    cancellation.)"""
    xs, ys = X.cores(), Y.cores()
    d = len(xs)

    def norm(cores):
        R = np.ones((1, 1))
        for k, c in enumerate(cores):
            r1, n, r2 = c.shape
            c = np.tensordot(R, c, axes=([1], [0])).reshape(-1, r2, order="F")
            if k == d - 1:
                return float(np.linalg.norm(c))
            q, R = np.linalg.qr(c)

    diff = []
    for k, (a, b) in enumerate(zip(xs, ys)):
        if k == 0:
            diff.append(np.concatenate([a, -b], axis=2))
        elif k == d - 1:
            diff.append(np.concatenate([a, b], axis=0))
        else:
            c = np.zeros((a.shape[0] + b.shape[0], a.shape[1], a.shape[2] + b.shape[2]))
            c[:a.shape[0], :, :a.shape[2]] = a
            c[a.shape[0]:, :, a.shape[2]:] = b
            diff.append(c)
    return norm(diff) / norm(xs)


def main():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    sub = p.add_subparsers(dest="what", required=True)
    m = sub.add_parser("matvec")
    m.add_argument("--r", type=int, default=64)
    m.add_argument("--n", type=int, default=64)
    m.add_argument("--ra", type=int, default=3)
    m.add_argument("--reps", type=int, default=20)
    m.add_argument("--precision", default="fp64,mixed")
    r = sub.add_parser("round")
    r.add_argument("--d", type=int, default=20)
    r.add_argument("--n", type=int, default=16)
    r.add_argument("--r", type=int, default=64)
    r.add_argument("--terms", type=int, default=4)
    r.add_argument("--eps", type=float, default=1e-8)
    r.add_argument("--reps", type=int, default=3)
    r.add_argument("--precision", default="fp64")
    r.add_argument("--check", action="store_true")
    r.add_argument("--kernel-table", action="store_true")
    g = sub.add_parser("grad")
    g.add_argument("--d", type=int, default=12)
    g.add_argument("--n", type=int, default=32)
    g.add_argument("--r", type=int, default=64)
    g.add_argument("--samples", type=int, default=1_000_000)
    g.add_argument("--reps", type=int, default=5)
    b = sub.add_parser("batch")
    b.add_argument("--count", type=int, default=512)
    b.add_argument("--workers", type=int, default=8)
    b.add_argument("--grouped", action="store_true",
                   help="grouped batch (workers = systems in flight, 0: all)")
    b.add_argument("--kernel-table", action="store_true",
                   help="run under the CUDA activity tracer and summarise the kernels")
    b.add_argument("--serial", type=int, default=64)
    b.add_argument("--tol", type=float, default=1e-8)
    b.add_argument("--precision", default="fp64,mixed")
    am = sub.add_parser("amen")
    am.add_argument("--d", type=int, default=10)
    am.add_argument("--n", type=int, default=64)
    am.add_argument("--rmax", type=int, default=128)
    am.add_argument("--tol", type=float, default=1e-8)
    am.add_argument("--reps", type=int, default=2)
    am.add_argument("--precision", default="fp64,mixed")
    am.add_argument("--kernel-table", action="store_true")
    am.add_argument("--timing", action="store_true",
                    help="time every local matvec with CUDA events (slows the solve)")
    dg = sub.add_parser("dgemm")
    dg.add_argument("--size", type=int, default=8192)
    dg.add_argument("--reps", type=int, default=10)
    sv = sub.add_parser("svd")
    sv.add_argument("--n", default="256,200,160,128,96,64")
    sv.add_argument("--reps", type=int, default=5)
    for s in (m, r, g, b, am, dg, sv):
        s.add_argument("--device", type=int, default=0)
        s.add_argument("--seed", type=int, default=5)
    args = p.parse_args()
    {"matvec": matvec, "round": round_bench, "grad": grad_bench, "batch": batch_bench,
     "amen": amen_bench, "dgemm": dgemm_bench, "svd": svd_bench}[args.what](args)


if __name__ == "__main__":
    main()
