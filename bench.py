#!/usr/bin/env python
"""Benchmark of the FMM hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c3|c2|c1|c4|c5|tree|nrnmm|cheb] [--precision tf32x3|bf16x3|fp64]

One step = one fmm solve (tree build + sweep; operator tables cached across
steps) over one synthetic batch.  Default workload: 4,194,304 targets and
sources from 16 clustered Gaussians in 3-D, 1/r (0 at coincidence), 6 nodes
per dimension, leaves of <= 128 points.  Prints one JSON line (rank 0).

`value` is targets/s with inputs resident in HBM (the mixed-precision solve);
`e2e` is the same metric through the C ABI with pinned host buffers, the
host<->device copies inside the timed region.  The plain FP64 GPU FMM is
timed on the same inputs and reported beside it, with both errors against the
FP64 exact sum on 4096 sampled targets.  Under torchrun each rank runs an
independent replica (the single-problem solve does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c1": dict(name="1-D 1/(x-y), 4096+4096 uniform points, 8 nodes, leaves<=64", d=1, n=4096,
               kernel="inv_diff", p0=0.0, poly_ord=7, cap=64, dist="uniform", wdist="uniform"),
    # TF32x3 by default: BF16x3 products (~2^-17) sit at the 2x-of-plain error bar here (2.00x measured)
    "c2": dict(name="2-D log r, 1,000,000+1,000,000 uniform points, 6 nodes/dim, leaves<=64", d=2,
               n=1_000_000, kernel="log_r", p0=0.0, poly_ord=5, cap=64, dist="uniform", wdist="normal",
               precision="tf32x3"),
    "c5": dict(name="512 independent 2-D multiquadric problems (sizes log-uniform in [1e3, 2e5], boxes of side "
                    "U[0.5, 2]), 16 right-hand sides, 5 nodes/dim, leaves<=64", d=2, n=512, kernel="multiquadric",
               p0=1e-4, poly_ord=4, cap=64, dist="forest", wdist="normal", nrhs=16),
    "c3": dict(name="3-D 1/r, 4,194,304+4,194,304 points from 16 Gaussians (sigma 0.02), 6 nodes/dim, "
                    "leaves<=128", d=3, n=4_194_304, kernel="inv_r_safe", p0=0.0, poly_ord=5, cap=128,
               dist="clustered", wdist="uniform"),
    "c4": dict(name="3-D adjoint: Gaussian exp(-r^2/0.01), 1,048,576+1,048,576 uniform points, weights N(0,1), "
                    "5 nodes/dim, Depth 6; one step = forward + backward (dL/dx, dL/dy, dL/dw of L = g.c) through "
                    "torch.autograd", d=3, n=1 << 20, kernel="gaussian", p0=0.01, poly_ord=4, cap=0, depth=6,
               dist="uniform", wdist="normal", adjoint=True),
    # the reference's other two approximate solvers, FP64 (src/tree.cpp, src/nrnmm.cpp)
    "tree": dict(name="tree solver: 3-D 1/r, 1,000,000+1,000,000 uniform points, 6 nodes/dim, default Depth",
                 d=3, n=1_000_000, kernel="inv_r_safe", p0=0.0, poly_ord=5, cap=0, dist="uniform",
                 wdist="uniform", solver="tree", sample=20_000),
    "cheb": dict(name="Chebyshev approximation (CHEBYSHEV_APPROX): 1/(1+|x|^2) on [-1,1]^3, Nth 15 (4096 "
                      "coefficients), fit + evaluation at 8,388,608 uniform points", d=3, n=8_388_608, nth=15,
                 dist="cheb", sample=2_000),
    "nrnmm": dict(name="nrnmm solver: 3-D 1/r, 1,000,000+1,000,000 uniform points, 6 nodes/dim, default nrn_N",
                  d=3, n=1_000_000, kernel="inv_r_safe", p0=0.0, poly_ord=5, cap=0, dist="uniform",
                  wdist="uniform", solver="nrnmm", sample=8_000),
}


def make_points(w, seed_t=1, seed_s=2, seed_w=3, seed_c=7):
    d, n = w["d"], w["n"]
    if w["dist"] == "uniform":
        t = np.random.default_rng(seed_t).random((n, d))
        s = np.random.default_rng(seed_s).random((n, d))
    else:
        cen = np.random.default_rng(seed_c).uniform(0.1, 0.9, (16, d))

        def blob(seed):
            r = np.random.default_rng(seed)
            k = r.integers(0, 16, n)
            return np.clip(cen[k] + 0.02 * r.standard_normal((n, d)), 0.0, 1.0)
        t, s = blob(seed_t), blob(seed_s)
    r = np.random.default_rng(seed_w)
    wt = r.uniform(-1, 1, n) if w["wdist"] == "uniform" else r.standard_normal(n)
    return t, s, wt


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        # nvidia-smi numbers GPUs by physical index and ignores
        # CUDA_VISIBLE_DEVICES: name the device by its UUID (else its PCI bus id)
        self.index = self.gpu_id(index)
        self.samples = []
        self.proc = None
        self.thread = None

    @staticmethod
    def gpu_id(index):
        try:
            import torch
            p = torch.cuda.get_device_properties(index)
            u = str(getattr(p, "uuid", "") or "")
            if u:
                return u if u.startswith(("GPU-", "MIG-")) else "GPU-" + u
            return "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        except Exception:  # no torch device properties: the ordinal is the best left
            return str(index)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        after = False
        if not self.samples:  # a timed region shorter than the sampling interval: one query right after it
            try:
                q = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
                parts = [x.strip() for x in q.stdout.strip().split(",")]
                if len(parts) >= 9:
                    self.samples.append(parts)
                    after = True
            except (OSError, subprocess.TimeoutExpired):
                pass
        sm = [float(p[1]) for p in self.samples if p[1].replace(".", "").isdigit()]
        mx = [float(p[2]) for p in self.samples if p[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for p in self.samples for i in range(4) if p[5 + i].lower() == "active"})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
               "reasons": reasons, "samples": len(self.samples), "gpu": self.index}
        if after:
            out["sampled"] = "once, right after the timed region (shorter than the 200 ms interval)"
        return out


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def tensor_peak(peaks, timed_s, precision):
    """The BF16 (TF32: half) dense tensor peak that bounds the M2L: the
    sustained figure (a matmul loop of seconds under the power cap) when the
    timed region keeps the GPU loaded for a second or more, else the burst
    figure.  Returns (peak, regime, burst peak)."""
    sustained = timed_s >= 1.0
    burst = peaks.get("bf16_tflops", 1590.0)
    bf16 = peaks.get("bf16_tflops_sustained", 1400.0) if sustained else burst
    div = 1.0 if precision == "bf16x3" else 2.0
    regime = (f"sustained (timed region {timed_s:.1f} s under load)" if sustained
              else f"burst (timed region {timed_s:.2f} s)")
    return bf16 / div, regime, burst / div


def add_peak_fields(roof, regime, burst):
    roof["peak_regime"] = regime
    if roof.get("achieved"):
        roof["frac_of_burst"] = roof["achieved"] / burst


def cpu_reference_baseline(wl, budget_s=20.0, with_error=True):
    """The reference fmm (compiled from its sources, oracle/_ref) on the host
    cores over a bounded sample of the workload: the same distribution and
    kernel at a reduced size that its dense uniform grid can hold."""
    from oracle.oracle import REF_SO, ORACLE_SO
    kind = "reference" if os.path.exists(REF_SO) else "port"
    if kind == "reference":
        from oracle.oracle import Reference as Impl
        impl = Impl()
    else:
        from oracle.oracle import Oracle as Impl
        impl = Impl()
    d = wl["d"]
    cores = os.cpu_count() or 1
    if wl["dist"] == "forest":
        return forest_reference_baseline(wl, impl, kind, cores)
    if wl.get("solver"):
        return solver_reference_baseline(wl, impl, kind, cores)
    if wl["dist"] == "cheb":
        return cheb_reference_baseline(wl, impl, kind, cores)
    # the largest sample whose solve stays within a few seconds on 16 host
    # cores (3-D: 65,536 clustered points at Depth 5, ~6 s; 131,072 at Depth 6
    # already takes ~60 s on 8 cores, the dense grid's M2L and P2P growing)
    n = {1: 4096, 2: 65536, 3: 65536}[d]
    sample = dict(wl)
    sample["n"] = n
    t, s, w = make_points(sample)
    depth = {1: 8, 2: 7, 3: 5}[d]
    kid = {"inv_diff": 2, "log_r": 3, "inv_r_safe": 1, "gaussian": 4, "multiquadric": 5}[wl["kernel"]]
    times = []
    out = None
    t_end = time.time() + budget_s
    while time.time() < t_end or not times:
        t0 = time.time()
        if kind == "reference":
            out, _ = impl.solve(d, "fmm", kid, wl["p0"], wl["poly_ord"], depth, 1, t, s, w)
        else:
            out, _ = impl.fmm(d, kid, wl["p0"], wl["poly_ord"], depth, 1, t, s, w)
        times.append(time.time() - t0)
        if len(times) >= 3:
            break
    best = min(times)
    rel = None
    if with_error:
        # its error against the FP64 exact sum on 1024 sampled targets (oracle restatement of exact)
        from oracle.oracle import Oracle
        rows = np.random.default_rng(11).choice(n, min(n, 1024), replace=False)
        ex = Oracle().exact_rows(d, kid, wl["p0"], rows, t, s, w)
        rel = float(np.linalg.norm(out[rows] - ex) / np.linalg.norm(ex))
    return {"value": n / best, "unit": "targets/s", "cores": cores, "kind": kind,
            "sample": f"{n} targets and {n} sources of the same distribution, Depth {depth}, trans_sym_flag 1, "
                      f"OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS', cores)}, best of {len(times)}",
            "seconds": best, "rel_l2_vs_fp64_exact": rel}


def forest_reference_baseline(wl, impl, kind, cores):
    """The reference's only route for a forest: one fmm call per problem and
    per right-hand side.  Sample: the first 8 problems of the forest, one
    right-hand side each, each at the depth the forest solve uses for it
    (the smallest with at most `cap` points per leaf, uniform estimate)."""
    tgt, toff, src, soff, W, sizes = make_forest(wl["n"], wl["d"], R=1)
    d = wl["d"]
    n_done, secs = 0, 0.0
    for p in range(8):
        a, b = int(toff[p]), int(toff[p + 1])
        m = b - a
        depth = max(3, int(np.ceil(np.log(max(m / wl["cap"], 1.0)) / np.log(2 ** d))) + 1)
        t, s, w = (np.ascontiguousarray(x) for x in (tgt[a:b], src[a:b], W[0, a:b]))
        t0 = time.time()
        if kind == "reference":
            impl.solve(d, "fmm", 5, wl["p0"], wl["poly_ord"], depth, 1, t, s, w)
        else:
            impl.fmm(d, 5, wl["p0"], wl["poly_ord"], depth, 1, t, s, w)
        secs += time.time() - t0
        n_done += m
    return {"value": n_done / secs, "unit": "targets*rhs/s", "cores": cores, "kind": kind,
            "sample": f"first 8 problems of the forest ({n_done} targets), 1 right-hand side, one fmm call per "
                      f"problem, OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS', cores)}",
            "seconds": secs}


def solver_reference_baseline(wl, impl, kind, cores):
    """The reference's tree / nrnmm solver on a sample of the workload's
    distribution (default Depth / nrn_N for the sample size)."""
    sample = dict(wl)
    sample["n"] = wl["sample"]
    t, s, w = make_points(sample)
    d, po, solver = wl["d"], wl["poly_ord"], wl["solver"]
    t0 = time.time()
    if kind == "reference":
        _, used = impl.solve(d, solver, 1, wl["p0"], po, -1, 0, t, s, w)
    elif solver == "tree":
        _, used = impl.tree(d, 1, wl["p0"], po, -1, t, s, w)
    else:
        _, used = impl.nrnmm(d, 1, wl["p0"], po, -1, t, s, w)
    secs = time.time() - t0
    what = "Depth" if solver == "tree" else "nrn_N"
    return {"value": sample["n"] / secs, "unit": "targets/s", "cores": cores, "kind": kind,
            "sample": f"{sample['n']} targets and {sample['n']} sources of the same distribution, {solver} solver, "
                      f"{what} {used}, OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS', cores)}",
            "seconds": secs}


def cheb_reference_baseline(wl, impl, kind, cores):
    """The reference's CHEBYSHEV_APPROX predict (one point per call, as its
    API offers) on a sample of the points; its fit is not timed (GCR on the
    4096 x 4096 system)."""
    d, nth = wl["d"], wl["nth"]
    x = np.cos((2 * np.arange(nth + 1) + 1) / (2 * (nth + 1)) * np.pi)
    n = nth + 1
    idx = np.arange(n ** d)
    nodes = np.stack([x[(idx // n ** q) % n] for q in range(d)], axis=1)
    from oracle.oracle import Oracle
    coef = Oracle().cheb_fit(d, nth, 1.0 / (1.0 + np.sum(nodes * nodes, axis=1)))
    pts = np.random.default_rng(5).uniform(-1, 1, (wl["sample"], d))
    t0 = time.time()
    if kind == "reference":
        impl.cheb_predict(d, nth, coef, pts)
    else:
        impl.cheb_eval(d, nth, coef, pts)
    secs = time.time() - t0
    return {"value": wl["sample"] / secs, "unit": "points/s", "cores": 1 if kind == "reference" else cores,
            "kind": kind, "sample": f"{wl['sample']} points, predict called once per point (single thread)",
            "seconds": secs}


def run_cheb(args, wl):
    """CHEBYSHEV_APPROX on the GPU: one step = fit from the node values +
    evaluation at every point (inputs resident on the device)."""
    import torch

    import fmma_b200
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    torch.cuda.set_device(dev)
    d, nth = wl["d"], wl["nth"]
    ctx = fmma_b200.Context(dev)
    ctx.set_m2l_options(pair=args.m2l_pair, stages=args.m2l_stages, group=args.m2l_group, units=args.m2l_units)
    nodes = fmma_b200.cheb_points(d, nth)
    values = torch.from_numpy(1.0 / (1.0 + np.sum(nodes * nodes, axis=1))).cuda(dev)
    pts_h = np.random.default_rng(1 + 100 * rank).uniform(-1, 1, (wl["n"], d))
    pts = torch.from_numpy(pts_h).cuda(dev)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")

    def step():
        c = ctx.cheb_fit(values, d, nth)
        return ctx.cheb_eval(c, pts, nth)

    out = step()
    sub = np.random.default_rng(2).choice(wl["n"], 4096, replace=False)
    exact = 1.0 / (1.0 + np.sum(pts_h[sub] ** 2, axis=1))
    err = float(np.max(np.abs(out.cpu().numpy()[sub] - exact)))
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    e0.record(stream)
    for _ in range(args.steps):
        step()
        launches += ctx.last_launch_count()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    # end to end with host arrays
    vh, ph = values.cpu().numpy(), torch.from_numpy(pts_h).pin_memory().numpy()
    t0 = time.perf_counter()
    ctx.cheb_eval(ctx.cheb_fit(vh, d, nth), ph, nth)
    e2e = (time.perf_counter() - t0) * 1e3
    if rank == 0:
        size = (nth + 1) ** d
        flops = 2.0 * size * wl["n"]  # Clenshaw / recurrences: 2 FP64 operations per coefficient and point
        cpu = None if args.no_cpu else cpu_reference_baseline(wl)
        line = {
            "metric": metric_of(wl), "value": wl["n"] / (ms / 1e3),
            "unit": "points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "coefficients": size, "l2": "points larger than L2"},
            "max_abs_err_vs_f": err,
            "roofline": {"bound": "fp64", "kernel": "k_cheb_eval", "achieved": flops / (ms / 1e3) / 1e12,
                         "unit": "TFLOP/s", "peak": None, "frac": None, "traffic": None,
                         "note": "2 FP64 operations per coefficient and point; FP64 pipe utilisation from ncu"},
            "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                                         "rel_l2_vs_fp64_exact") if k in cpu},
            "e2e": {"value": wl["n"] / (e2e / 1e3), "unit": "points/s",
                    "h2d_bytes_per_step": int(vh.nbytes + ph.nbytes), "d2h_bytes_per_step": int(wl["n"] * 8)},
            "gpu_launches": int(launches), "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def run_solver(args, wl):
    """The tree or nrnmm solver (FP64) on one GPU per rank (replicas): one
    step = one solve, tree/grid build included."""
    import torch
    import torch.distributed as dist

    import fmma_b200
    from fmma_b200.sharding import max_over_ranks
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    t, s, w = make_points(wl, seed_t=1 + 100 * rank, seed_s=2 + 100 * rank, seed_w=3 + 100 * rank)
    ctx = fmma_b200.Context(dev)
    ctx.set_m2l_options(pair=args.m2l_pair, stages=args.m2l_stages, group=args.m2l_group, units=args.m2l_units)
    ctx.set_kernel(wl["kernel"], wl["p0"])
    tt, ss, ww = (torch.from_numpy(a).cuda(dev) for a in (t, s, w))
    out = torch.empty(wl["n"], dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")
    solver = wl["solver"]

    def solve(o=out):
        return ctx.solve(tt, ss, ww, solver=solver, poly_ord=wl["poly_ord"], depth=-1, out=o)

    _, used = solve()
    rows = np.random.default_rng(11).choice(wl["n"], 4096, replace=False)
    exact = ctx.exact_rows(rows, t, s, w)
    a = out.cpu().numpy()[rows]
    err = float(np.linalg.norm(a - exact) / np.linalg.norm(exact))
    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    e0.record(stream)
    for _ in range(args.steps):
        solve()
        launches += ctx.last_launch_count()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    stages = ctx.stage_times()
    th, sh, wh = (torch.from_numpy(x).pin_memory().numpy() for x in (t, s, w))
    ah = torch.empty(wl["n"], dtype=torch.float64).pin_memory().numpy()
    ctx.solve(th, sh, wh, solver=solver, poly_ord=wl["poly_ord"], depth=-1, out=ah)
    t0 = time.perf_counter()
    ctx.solve(th, sh, wh, solver=solver, poly_ord=wl["poly_ord"], depth=-1, out=ah)
    e2e = (time.perf_counter() - t0) * 1e3
    ms, e2e = max_over_ranks([ms, e2e], device=f"cuda:{dev}")
    if rank == 0:
        d, P = wl["d"], (wl["poly_ord"] + 1) ** wl["d"]
        far_ms = stages.get("M2L", 0.0)
        if solver == "nrnmm":
            far_pairs = wl["n"] * (used ** d - 3 ** d) * P  # uniform points: every box holds sources
            kern = "k_nrn_far"
        else:
            # upper bound: 6^d - 3^d far boxes at each level 2 .. Depth-1
            far_pairs = wl["n"] * (6 ** d - 3 ** d) * P * max(used - 2, 0)
            kern = "k_m2p_f64"
        n_total = wl["n"] * world
        cpu = None if args.no_cpu else cpu_reference_baseline(wl)
        line = {
            "metric": metric_of(wl), "value": n_total / (ms / 1e3), "unit": "targets/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], ("depth" if solver == "tree" else "nrn_N"): used,
                       "nodes_per_dim": wl["poly_ord"] + 1, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2"},
            "rel_l2_vs_fp64_exact": err,
            "stage_ms": {k: round(v, 3) for k, v in stages.items() if v},
            "roofline": {"bound": "fp64", "kernel": kern, "achieved": far_pairs / (far_ms / 1e3) if far_ms else None,
                         "unit": "kernel evaluations/s", "peak": None, "frac": None, "traffic": None,
                         "note": "FP64-issue bound; pipe utilisation from ncu in profiles/"},
            "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                                         "rel_l2_vs_fp64_exact") if k in cpu},
            "e2e": {"value": n_total / (e2e / 1e3), "unit": "targets/s",
                    "h2d_bytes_per_step": int(t.nbytes + s.nbytes + w.nbytes), "d2h_bytes_per_step": int(ah.nbytes)},
            "gpu_launches": int(launches), "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def run_adjoint(args, wl):
    """C4: one step = the FMM forward pass and its hand-written adjoint through
    torch.autograd (pyfmma.torch.fmm): a forward solve, the transposed solve
    with its gradient (dL/dw, dL/dy) and the forward gradient (dL/dx).  Trees
    are rebuilt in every solve.  Inputs are device-resident for `value`; `e2e`
    copies them from pinned host memory and the three gradients back."""
    import torch
    import torch.distributed as dist

    import fmma_b200
    import pyfmma
    from fmma_b200.sharding import max_over_ranks
    from pyfmma.torch import fmm
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    t, s, w = make_points(wl, seed_t=1 + 100 * rank, seed_s=2 + 100 * rank, seed_w=3 + 100 * rank)
    g = np.random.default_rng(4 + 100 * rank).standard_normal(wl["n"])
    ctx = fmma_b200.Context(dev)
    ctx.set_m2l_options(pair=args.m2l_pair, stages=args.m2l_stages, group=args.m2l_group, units=args.m2l_units)
    kern = pyfmma.kernels.gaussian(wl["p0"])
    depth, po = wl["depth"], wl["poly_ord"]
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")
    x = torch.from_numpy(t).cuda(dev).requires_grad_(True)
    y = torch.from_numpy(s).cuda(dev).requires_grad_(True)
    wt = torch.from_numpy(w).cuda(dev).requires_grad_(True)
    gd = torch.from_numpy(g).cuda(dev)

    def step(prec, xx=x, yy=y, ww=wt, gg=gd):
        for a in (xx, yy, ww):
            a.grad = None
        c = fmm(xx, yy, ww, kernel=kern, poly_ord=po, depth=depth, precision=prec, context=ctx)
        (gg * c).sum().backward()
        return c

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            step(prec)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        torch.cuda.current_stream(dev).synchronize()
        e0.record(stream)
        for _ in range(steps):
            step(prec)
            launches += ctx.last_launch_count()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        return e0.elapsed_time(e1) / steps, launches

    # accuracy: the gradients on 2048 sampled points against the exact solver's
    rows = np.sort(np.random.default_rng(12).choice(wl["n"], 2048, replace=False))
    ri = torch.from_numpy(rows).cuda(dev)
    ctx.set_kernel("gaussian", wl["p0"])
    X, Y, W = x.detach(), y.detach(), wt.detach()
    ce, cg, _ = ctx.solve_grad(X[ri].contiguous(), Y, W, solver="exact")
    u, ug, _ = ctx.solve_grad(Y[ri].contiguous(), X, gd, solver="exact")

    def errors(prec):
        c = step(prec).detach()
        want = {"c": ce, "dL/dx": gd[ri].unsqueeze(-1) * cg, "dL/dy": W[ri].unsqueeze(-1) * ug, "dL/dw": u}
        got = {"c": c[ri], "dL/dx": x.grad[ri], "dL/dy": y.grad[ri], "dL/dw": wt.grad[ri]}
        return {k: float(torch.linalg.norm(got[k] - want[k]) / torch.linalg.norm(want[k])) for k in want}

    err = errors(args.precision)
    clocks = ClockSampler(dev)
    clocks.start()
    ms, launches = timed(args.precision, args.steps, args.warmup)
    clk = clocks.stop()
    plain = None
    if args.precision != "fp64" and not args.no_plain:
        pms, _ = timed("fp64", max(1, min(args.steps, 3)), 1)
        plain = {"ms_per_step": pms, "value": wl["n"] / (pms / 1e3), "rel_l2_vs_exact": errors("fp64")}
    # the three solves of a step one by one through the C ABI, for the stage split and the M2L roofline
    ctx.set_kernel("gaussian", wl["p0"])
    split = {}
    m2l_ms = m2l_fl = 0.0
    for name, call in (("forward", lambda: ctx.solve(X, Y, W, poly_ord=po, depth=depth, precision=args.precision)),
                       ("transposed+grad", lambda: ctx.solve_grad(Y, X, gd, poly_ord=po, depth=depth,
                                                                  precision=args.precision)),
                       ("forward grad", lambda: ctx.solve_grad(X, Y, W, poly_ord=po, depth=depth,
                                                               precision=args.precision, want_potential=False))):
        call()
        st = ctx.m2l_stats()
        m2l_ms += st["kernel_ms"]
        m2l_fl += st["flops"]
        split[name] = {k: round(v, 3) for k, v in ctx.stage_times().items() if v}
    # end to end: host arrays in pinned memory, copied in and the gradients copied out inside the timed region
    th, sh, wh, gh = (torch.from_numpy(a).pin_memory() for a in (t, s, w, g))
    outs = [torch.empty(sh_, dtype=torch.float64).pin_memory() for sh_ in ((wl["n"], 3), (wl["n"], 3), (wl["n"],))]

    def e2e_step():
        xx = th.cuda(dev, non_blocking=True).requires_grad_(True)
        yy = sh.cuda(dev, non_blocking=True).requires_grad_(True)
        ww = wh.cuda(dev, non_blocking=True).requires_grad_(True)
        gg = gh.cuda(dev, non_blocking=True)
        step(args.precision, xx, yy, ww, gg)
        for o, a in zip(outs, (xx, yy, ww)):
            o.copy_(a.grad, non_blocking=True)
        torch.cuda.synchronize(dev)

    e2e_step()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        e2e_step()
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = statistics.median(e2e)
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], device=f"cuda:{dev}")
    if rank == 0:
        n_total = wl["n"] * world
        peaks, peak_src = measured_peaks()
        if args.precision == "fp64":
            achieved = m2l_fl / (m2l_ms / 1e3) / 1e12 if m2l_ms else None
            roof = {"bound": "fp64", "kernel": "k_m2l_f64 (FP64 DMMA), the three solves of a step",
                    "achieved": achieved, "peak": 37.0, "unit": "TFLOP/s",
                    "frac": achieved / 37.0 if achieved else None, "traffic": None,
                    "peak_source": "nominal B200 FP64 tensor"}
        else:
            tpk, regime, burst = tensor_peak(peaks, ms * args.steps / 1e3, args.precision)
            achieved = 3 * m2l_fl / (m2l_ms / 1e3) / 1e12 if m2l_ms else None
            roof = {"bound": "tensor", "kernel": "k_m2l_tc2 + k_m2l_tc (tensor-core M2L), the three solves of a step",
                    "achieved": achieved,
                    "peak": tpk, "unit": "TFLOP/s", "frac": achieved / tpk if achieved else None, "traffic": None,
                    "peak_source": f"{peak_src} bf16 cuBLAS" + ("" if args.precision == "bf16x3" else " / 2 (TF32)")}
            add_peak_fields(roof, regime, burst)
        roof["m2l_kernel_ms_per_step"] = m2l_ms
        cpu = None if args.no_cpu else cpu_reference_baseline(wl)
        line = {
            "metric": metric_of(wl), "value": n_total / (ms / 1e3), "unit": "targets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+" + args.precision, "data": "synthetic",
            "config": {"workload": wl["name"], "depth": depth, "nodes_per_dim": po + 1, "precision": args.precision,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2",
                       "operator_tables": "cached across steps"},
            "rel_l2_vs_exact_on_2048_points": err, "plain_fp64": plain,
            "stage_ms_per_solve": split, "roofline": roof,
            "cpu_baseline": None if cpu is None else dict(
                {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "rel_l2_vs_fp64_exact") if k in cpu},
                note="the reference has no gradients: its forward fmm alone"),
            "e2e": {"value": n_total / (e2e_ms / 1e3), "unit": "targets/s",
                    "h2d_bytes_per_step": int(t.nbytes + s.nbytes + w.nbytes + g.nbytes),
                    "d2h_bytes_per_step": int(sum(o.numel() * 8 for o in outs))},
            "gpu_launches": int(launches), "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    vals = []
    base = None
    err = None
    for i in range(args.warmup + args.steps):
        base = cpu_reference_baseline(wl, budget_s=0.0, with_error=(i == 0))
        if i == 0:
            err = base.get("rel_l2_vs_fp64_exact")
        if i >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    unit = base["unit"]
    line = {"impl": "reference", "metric": metric_of(wl), "value": v, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": base["seconds"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "sample": base["sample"]},
            "cpu_baseline": {"value": v, "unit": unit, "cores": base["cores"], "kind": base["kind"],
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if err is not None:
        line["rel_l2_vs_fp64_exact"] = err
        line["rel_l2_scope"] = "1024 sampled targets of the sample against the FP64 exact sum"
    print(json.dumps(line), flush=True)


METRIC = "targets/s at matched rel-L2 err vs FP64 oracle: mixed+batched vs plain FP64 GPU FMM"


def ncu_kernel_dram_bytes(path, name, launches_per_step):
    """DRAM bytes (read + write) per step of the kernels whose name contains
    `name`, from an ncu --csv launch list of this same command captured with
    the metrics dram__bytes_read.sum and dram__bytes_write.sum: the sum over
    the captured launches, scaled to `launches_per_step` launches."""
    import csv
    tot, ids = 0.0, set()
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}
    with open(path, newline="") as f:
        rows = [r for r in csv.reader(f) if r]
    hdr = next(i for i, r in enumerate(rows) if "Metric Name" in r)
    cols = rows[hdr]
    iid, ik, im, iu, iv = (cols.index(c) for c in ("ID", "Kernel Name", "Metric Name", "Metric Unit", "Metric Value"))
    for r in rows[hdr + 1:]:
        if len(r) <= iv or name not in r[ik] or r[im] not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            continue
        ids.add(r[iid])
        tot += float(r[iv].replace(",", "")) * scale.get(r[iu], 1.0)
    return tot / len(ids) * launches_per_step if ids else None


def metric_of(wl):
    if wl.get("adjoint"):
        return "targets/s, FMM forward + adjoint (dL/dx, dL/dy, dL/dw) through torch.autograd"
    if wl.get("solver"):
        return f"targets/s, {wl['solver']} solver (FP64)"
    if wl["dist"] == "cheb":
        return "points/s, Chebyshev approximation fit + evaluation (FP64)"
    return METRIC


def make_forest(nprob, d=2, seed=11, lo=1e3, hi=2e5, R=16):
    r = np.random.default_rng(seed)
    sizes = np.exp(r.uniform(np.log(lo), np.log(hi), nprob)).astype(np.int64)
    tg, sr = [], []
    for m in sizes:
        side = r.uniform(0.5, 2.0)
        corner = r.uniform(-10, 10, d)
        tg.append(corner + side * r.random((m, d)))
        sr.append(corner + side * r.random((m, d)))
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    W = r.standard_normal((R, off[-1]))
    return np.concatenate(tg), off, np.concatenate(sr), off.copy(), W, sizes


def stage_roofline(wl, stages, tree, levels, depth, peaks):
    """Algorithmic bytes (HBM-bound stages) or interactions (P2P) per step,
    by the per-stage formulas of the measurement plan, over the stage's
    CUDA-event time; bandwidth against the measured copy peak."""
    d, n, R = wl["d"], wl["poly_ord"] + 1, 1
    P = n ** d
    N = M = wl["n"]
    B, rows = levels["boxes"], levels["rows"]
    leaves = B[0]
    key_bits = d * (depth - 1)
    passes = -(-key_bits // 8)
    hbm = peaks.get("hbm_gbs", 6650.0)
    nb = {
        "tree": (N + M) * (d * 8 + 8) + passes * (N + M) * 2 * (8 + 4) + sum(b * 16 for b in B)
                + sum(r * 189 * 4 for r in rows) + rows[0] * (3 ** d) * 4,
        "P2M": M * (d + 1) * 8 + leaves * P * 8 * R,
        "L2P": N * d * 8 + rows[0] * P * 8 * R + N * 8 * R,
        "M2M": sum(2 * b * P * 8 * R for b in B[:-1]),
        "L2L": sum(2 * r * P * 8 * R for r in rows[:-1]),
    }
    out = {}
    for k, v in nb.items():
        ms = stages.get(k, 0.0)
        gbs = v / (ms / 1e3) / 1e9 if ms else None
        out[k] = {"bytes": int(v), "ms": round(ms, 3), "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm if gbs else None}
    ms = stages.get("P2P", 0.0)
    c_f = 9  # 1/r: 3 sub, 3 fma, rsqrt, select, weight fma
    inter = tree["p2p_pairs"]
    out["P2P"] = {"interactions": int(inter), "ms": round(ms, 3),
                  "g_interactions_per_s": inter / (ms / 1e3) / 1e9 if ms else None,
                  "declared_flops_per_interaction": c_f,
                  "tflops_declared": inter * c_f / (ms / 1e3) / 1e12 if ms else None}
    out["hbm_peak_gbs"] = hbm
    return out


def run_forest(args, wl):
    """C5: the whole forest in one sweep (tree build included) against looping
    the plain FP64 single-problem solve per problem and per right-hand side."""
    import torch
    import torch.distributed as dist

    import fmma_b200
    from fmma_b200.sharding import forest_shard, max_over_ranks, sub_forest
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    R = wl["nrhs"]
    tgt, toff, src, soff, W, sizes = make_forest(wl["n"], wl["d"], R=R)
    nt_all = int(toff[-1])
    if world > 1:  # independent problems: each rank takes its share, no collective on the data path
        mine = forest_shard(sizes, world, rank)
        toff, soff, ti, si = sub_forest(toff, soff, mine)
        tgt, src, W, sizes = tgt[ti], src[si], np.ascontiguousarray(W[:, si]), sizes[mine]
    ctx = fmma_b200.Context(dev)
    ctx.set_m2l_options(pair=args.m2l_pair, stages=args.m2l_stages, group=args.m2l_group, units=args.m2l_units)
    ctx.set_kernel(wl["kernel"], wl["p0"])
    tt, ss, ww = (torch.from_numpy(a).cuda(dev) for a in (tgt, src, W))
    depths = ctx.forest_depths(tt, toff, ss, soff, wl["cap"])
    out = torch.empty((R, int(toff[-1])), dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    def step(prec):
        return ctx.forest_solve(tt, toff, ss, soff, ww, depths, poly_ord=wl["poly_ord"], precision=prec, out=out)

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            step(prec)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m2l_ms = m2l_fl = 0.0
        launches = 0
        e0.record(stream)
        for _ in range(steps):
            step(prec)
            st = ctx.m2l_stats()
            m2l_ms += st["kernel_ms"]
            m2l_fl += st["flops"]
            launches += ctx.last_launch_count()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps, m2l_ms / steps, m2l_fl / steps, launches, ctx.stage_times()

    # errors: a few problems against the FP64 exact sum (first right-hand side)
    def errors(prec):
        o = step(prec)
        errs = []
        for p in np.random.default_rng(3).choice(len(sizes), 6, replace=False):
            a, b = int(toff[p]), int(toff[p + 1])
            rows = np.arange(a, b)[:: max(1, (b - a) // 256)]
            ex = ctx.exact_rows(rows - a, np.ascontiguousarray(tgt[a:b]), np.ascontiguousarray(src[soff[p]:soff[p + 1]]),
                                np.ascontiguousarray(W[0, soff[p]:soff[p + 1]]))
            got = o[0, rows].cpu().numpy()
            errs.append(np.linalg.norm(got - ex) / np.linalg.norm(ex))
        return float(np.max(errs))

    err_mixed = errors(args.precision)
    clocks = ClockSampler(dev)
    clocks.start()
    ms, m2l_ms, m2l_fl, launches, stages = timed(args.precision, args.steps, args.warmup)
    clk = clocks.stop()
    err_plain = errors("fp64")
    pms, _, _, _, _ = timed("fp64", max(1, min(args.steps, 3)), 1)
    # graph-captured sweep for new right-hand sides on the same forest (autotuned)
    plan = ctx.plan(tt, toff, ss, soff, R, depths, poly_ord=wl["poly_ord"], precision=args.precision)
    for _ in range(3):
        plan.execute(ww, out)
    pex = []
    for _ in range(5):
        plan.execute(ww, out)
        pex.append(plan.stats()["last_exec_ms"])
    pst = plan.stats()
    plan.close()
    # baseline: the plain FP64 single-problem solve looped per problem and per RHS (subset, extrapolated)
    sub = np.random.default_rng(5 + rank).choice(len(sizes), min(32, len(sizes)), replace=False)
    loop_t, loop_n = 0.0, 0
    for p in sub:
        a, b = int(toff[p]), int(toff[p + 1])
        t1 = tt[a:b].contiguous()
        s1 = ss[int(soff[p]):int(soff[p + 1])].contiguous()
        w1 = ww[0, int(soff[p]):int(soff[p + 1])].contiguous()
        ctx.solve(t1, s1, w1, poly_ord=wl["poly_ord"], depth=int(depths[p]))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.solve(t1, s1, w1, poly_ord=wl["poly_ord"], depth=int(depths[p]))
        torch.cuda.synchronize()
        loop_t += time.perf_counter() - t0
        loop_n += b - a
    loop_rate = loop_n / loop_t  # targets x RHS per second
    nt = int(toff[-1])
    peaks, peak_src = measured_peaks()
    tpk, regime, burst = tensor_peak(peaks, ms * args.steps / 1e3, args.precision)
    achieved = (3 * m2l_fl / (m2l_ms / 1e3)) / 1e12 if m2l_ms > 0 else None
    # end to end: host arrays through the C ABI
    th, sh, wh = (torch.from_numpy(a).pin_memory().numpy() for a in (tgt, src, W))
    ah = torch.empty((R, nt), dtype=torch.float64).pin_memory().numpy()
    ctx.forest_solve(th, toff, sh, soff, wh, depths, poly_ord=wl["poly_ord"], precision=args.precision, out=ah)
    e2e = []
    for _ in range(2):
        t0 = time.perf_counter()
        ctx.forest_solve(th, toff, sh, soff, wh, depths, poly_ord=wl["poly_ord"], precision=args.precision, out=ah)
        e2e.append((time.perf_counter() - t0) * 1e3)
    # times are the maximum over ranks; each rank solved its own share of the problems
    ms, pms, pexm, e2em, loop_s = max_over_ranks(
        [ms, pms, float(np.median(pex)), float(np.median(e2e)), loop_n / loop_rate / max(loop_n, 1)],
        device=f"cuda:{dev}")
    loop_rate = 1.0 / loop_s
    nt = nt_all
    if rank != 0:
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": nt * R / (ms / 1e3), "unit": "targets*rhs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+" + args.precision, "data": "synthetic",
        "config": {"workload": wl["name"], "problems": int(wl["n"]), "targets_total": nt, "nrhs": R,
                   "parallelism": f"problems split over {world} rank(s), no data-path collective",
                   "depths_min_max": [int(depths.min()), int(depths.max())], "precision": args.precision,
                   "l2": "inputs larger than L2", "operator_tables": "cached across steps"},
        "rel_l2_vs_fp64_exact_max_over_6_problems": err_mixed, "plain_fp64_forest": {
            "ms_per_step": pms, "rel_l2_max": err_plain},
        "loop_plain_fp64_per_problem_per_rhs": {"value": loop_rate, "unit": "targets*rhs/s",
                                                "sample": "32 random problems x 1 RHS, extrapolated"},
        "speedup_vs_loop": (nt * R / (ms / 1e3)) / loop_rate,
        "plan_graph_replay": {"ms_per_step": pexm, "value": nt * R / (pexm / 1e3),
                              "levels_tc": pst["levels_tc"], "levels_fp64": pst["levels_fp64"],
                              "graph_nodes": pst["graph_nodes"], "build_ms": pst["build_ms"]},
        "stage_ms": {k: round(v, 3) for k, v in stages.items() if v},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": tpk, "unit": "TFLOP/s",
                     "frac": achieved / tpk if achieved else None, "traffic": None,
                     "kernel": "k_m2l_tc2 (2-SM, levels with a 256-row tile per cluster) + k_m2l_tc (1-SM)",
                     "peak_source": f"{peak_src} bf16 cuBLAS" +
                     ("" if args.precision == "bf16x3" else " / 2 (TF32)"),
                     "peak_regime": regime, "frac_of_burst": achieved / burst if achieved else None},
        "cpu_baseline": None if (args.no_cpu or world > 1) else cpu_reference_baseline(wl),
        "e2e": {"value": nt * R / (e2em / 1e3), "unit": "targets*rhs/s",
                "h2d_bytes_per_step": int(tgt.nbytes + src.nbytes + W.nbytes), "d2h_bytes_per_step": int(ah.nbytes)},
        "gpu_launches": int(launches), "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=["tf32x3", "bf16x3", "fp64"],
                    help="mixed precision of the solve (default: the workload's, bf16x3 except c2)")
    ap.add_argument("--n", type=int, default=0, help="override the point count (profiling on a small case)")
    ap.add_argument("--depth", type=int, default=0,
                    help="fixed Depth instead of the leaf-capacity search (profiling: no search launches)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--traffic-csv", default="",
                    help="ncu --csv launch list (dram__bytes_read.sum, dram__bytes_write.sum) of this command: "
                         "fills roofline.traffic")
    ap.add_argument("--no-cold", action="store_true", help="skip the cold step on fresh inputs")
    ap.add_argument("--m2l-pair", type=int, default=-1, choices=[-1, 0, 1],
                    help="tensor-core M2L 2-SM kernel: -1 library default, 0 off, 1 on")
    ap.add_argument("--m2l-stages", type=int, default=0, help="tensor-core M2L pipeline depth cap (0: default)")
    ap.add_argument("--m2l-group", type=int, default=0, help="tensor-core M2L slots per drain (0: default)")
    ap.add_argument("--m2l-units", type=int, default=0,
                    help="tensor-core M2L (slot, K chunk) units per pipeline stage (0: default)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.precision is None:
        args.precision = wl.get("precision", "bf16x3")
    if args.n:
        wl["n"] = args.n
        wl["name"] = wl["name"] + f" [reduced to {args.n} points]"
    if args.impl == "reference":
        run_reference(args, wl)
        return
    if args.workload == "c5":
        run_forest(args, wl)
        return
    if wl.get("adjoint"):
        run_adjoint(args, wl)
        return
    if wl.get("solver"):
        run_solver(args, wl)
        return
    if wl["dist"] == "cheb":
        run_cheb(args, wl)
        return

    import torch
    import torch.distributed as dist

    import fmma_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    t, s, w = make_points(wl, seed_t=1 + 100 * rank, seed_s=2 + 100 * rank, seed_w=3 + 100 * rank)
    ctx = fmma_b200.Context(dev)
    ctx.set_m2l_options(pair=args.m2l_pair, stages=args.m2l_stages, group=args.m2l_group, units=args.m2l_units)
    ctx.set_kernel(wl["kernel"], wl["p0"])
    depth = args.depth if args.depth > 0 else fmma_b200.choose_depth(ctx, t, s, wl["cap"])
    tt = torch.from_numpy(t).cuda(dev)
    ss = torch.from_numpy(s).cuda(dev)
    ww = torch.from_numpy(w).cuda(dev)
    out = torch.empty(wl["n"], dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")

    def solve(prec, o=out):
        return ctx.solve(tt, ss, ww, poly_ord=wl["poly_ord"], depth=depth, precision=prec, out=o)

    m2l_launches = 0

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            solve(prec)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m2l_ms, m2l_flops, launches = 0.0, 0.0, 0
        nonlocal m2l_launches
        e0.record(stream)
        for _ in range(steps):
            solve(prec)
            st = ctx.m2l_stats()
            m2l_ms += st["kernel_ms"]
            m2l_flops += st["flops"]
            m2l_launches = st["launches"]
            launches += ctx.last_launch_count()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        return e0.elapsed_time(e1) / steps, m2l_ms / steps, m2l_flops / steps, launches, ctx.stage_times()

    # errors on 4096 sampled targets against the FP64 exact sum
    rows = np.random.default_rng(11).choice(wl["n"], 4096, replace=False)
    exact = ctx.exact_rows(rows, t, s, w)

    def err_of(prec):
        o, _ = solve(prec)
        a = o.cpu().numpy()[rows]
        return float(np.linalg.norm(a - exact) / np.linalg.norm(exact)), float(np.max(np.abs(a - exact)))

    def rel_rms_of(prec):
        """The reference tests' per-point relative RMS (test/src/fmma/fmm.cpp)."""
        o, _ = solve(prec)
        a = o.cpu().numpy()[rows]
        nz = exact != 0
        return float(np.sqrt(np.mean(((a[nz] - exact[nz]) / exact[nz]) ** 2)))

    err_mixed, maxerr_mixed = err_of(args.precision)
    rms_mixed = rel_rms_of(args.precision)

    clocks = ClockSampler(dev)
    clocks.start()
    ms, m2l_ms, m2l_flops, launches, stages = timed(args.precision, args.steps, args.warmup)
    clk = clocks.stop()
    tree = ctx.tree_stats()
    levels = ctx.tree_levels()

    # sweep only: the same solve as a plan (tree built once), replayed as a CUDA graph
    plan = ctx.plan(tt, [0, wl["n"]], ss, [0, wl["n"]], 1, [depth], poly_ord=wl["poly_ord"],
                    precision=args.precision, autotune=False)
    out_sweep = torch.empty_like(out)
    for _ in range(2):
        plan.execute(ww, out_sweep)
    sweep = []
    for _ in range(max(3, min(args.steps, 5))):
        plan.execute(ww, out_sweep)
        sweep.append(plan.stats()["last_exec_ms"])
    sweep_ms = float(np.median(sweep))
    plan.close()

    plain = None
    if not args.no_plain and args.precision != "fp64":
        err_plain, maxerr_plain = err_of("fp64")
        pms, pm2l_ms, _, _, pstages = timed("fp64", max(1, min(args.steps, 3)), 1)
        plain = {"value": wl["n"] / (pms / 1e3), "ms_per_step": pms, "rel_l2": err_plain, "max_abs_err": maxerr_plain,
                 "m2l_kernel_ms": pm2l_ms, "stage_ms": {k: round(v, 3) for k, v in pstages.items() if v}}

    # end-to-end through the C ABI with pinned host buffers
    th = torch.from_numpy(t).pin_memory().numpy()
    sh = torch.from_numpy(s).pin_memory().numpy()
    wh = torch.from_numpy(w).pin_memory().numpy()
    ah = torch.empty(wl["n"], dtype=torch.float64).pin_memory().numpy()
    for _ in range(1):
        ctx.solve(th, sh, wh, poly_ord=wl["poly_ord"], depth=depth, precision=args.precision, out=ah)
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        ctx.solve(th, sh, wh, poly_ord=wl["poly_ord"], depth=depth, precision=args.precision, out=ah)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_ms[-1] = max(e2e_ms[-1], ctx.stage_times()["total"])
    e2e = statistics.median(e2e_ms)

    # one cold step: freshly drawn inputs of the same distribution (another
    # cube, so every operator table is rebuilt), device-resident, CUDA events
    cold = None
    if not args.no_cold:
        tc_, sc_, wc_ = make_points(wl, seed_t=1001 + 100 * rank, seed_s=1002 + 100 * rank, seed_w=1003 + 100 * rank)
        tcd, scd, wcd = (torch.from_numpy(a).cuda(dev) for a in (tc_, sc_, wc_))
        torch.cuda.synchronize(dev)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        ctx.solve(tcd, scd, wcd, poly_ord=wl["poly_ord"], depth=depth, precision=args.precision, out=out)
        c1.record(stream)
        torch.cuda.synchronize(dev)
        cold = {"ms": c0.elapsed_time(c1), "stage_ms": {k: round(v, 3) for k, v in ctx.stage_times().items() if v},
                "what": "one solve on freshly drawn inputs (seeds 1001-1003): a new cube, so the operator tables "
                        "of every level are rebuilt inside the step"}
        del tcd, scd, wcd

    # max over ranks (replicas: every rank solved its own copy of the workload)
    from fmma_b200.sharding import max_over_ranks
    ms, e2e, sweep_ms = max_over_ranks([ms, e2e, sweep_ms], device=f"cuda:{dev}")

    if rank == 0:
        peaks, peak_src = measured_peaks()
        # TF32 dense tensor peak taken as half the measured BF16 one (nominal 1.1 vs 2.25 PF)
        tpk, regime, burst = tensor_peak(peaks, ms * args.steps / 1e3, args.precision)
        n_products = 3 if args.precision != "fp64" else 1
        achieved = (m2l_flops * n_products / (m2l_ms / 1e3)) / 1e12 if m2l_ms > 0 else None
        if args.precision == "fp64":
            roof = {"bound": "fp64", "achieved": achieved, "peak": 37.0, "unit": "TFLOP/s",
                    "frac": achieved / 37.0 if achieved else None, "traffic": None,
                    "kernel": "k_m2l_f64 (FP64 DMMA)", "peak_source": "nominal B200 FP64"}
        else:
            roof = {"bound": "tensor", "achieved": achieved, "peak": tpk, "unit": "TFLOP/s",
                    "frac": achieved / tpk if achieved else None, "traffic": None,
                    "kernel": f"k_m2l_tc2 (2-SM, large levels) + k_m2l_tc (small levels), {args.precision}",
                    "peak_source": f"{peak_src} bf16 cuBLAS" + ("" if args.precision == "bf16x3" else " / 2 (TF32)"),
                    "flops_per_launch_note": "3 split products x 2 P^2 per (target box, source box) pair",
                    "m2l_kernel_ms_per_step": m2l_ms, "m2l_pairs": tree["m2l_pairs"]}
            add_peak_fields(roof, regime, burst)
            # DRAM bytes of the M2L launches of one solve, from an ncu launch
            # list of this same command (given with --traffic-csv); else null
            if args.traffic_csv:
                roof["traffic"] = ncu_kernel_dram_bytes(args.traffic_csv, "k_m2l_tc", m2l_launches)
                roof["traffic_scope"] = f"DRAM read+write bytes, the {m2l_launches} M2L launches of one solve"
        cpu = None if args.no_cpu else cpu_reference_baseline(wl)
        n_total = wl["n"] * world
        line = {
            "metric": METRIC, "value": n_total / (ms / 1e3), "unit": "targets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+" + args.precision if args.precision != "fp64" else "f64",
            "data": "synthetic",
            "config": {"workload": wl["name"], "depth": depth, "nodes_per_dim": wl["poly_ord"] + 1, "nrhs": 1,
                       "precision": args.precision, "parallelism": f"replicas{world}",
                       "l2": "inputs and tree arrays larger than L2 (126 MB)",
                       "operator_tables": "cached across steps (built in warm-up)"},
            "rel_l2_vs_fp64_exact": err_mixed, "max_abs_err": maxerr_mixed, "rel_rms_per_point": rms_mixed,
            "cold_step": cold,
            "sweep_only": {"ms_per_step": sweep_ms, "value": n_total / (sweep_ms / 1e3),
                           "what": "same solve with the tree built once (plan), sweep replayed as a CUDA graph"},
            "stage_roofline": stage_roofline(wl, stages, tree, levels, depth, peaks),
            "plain_fp64": plain,
            "speedup_vs_plain": (plain["ms_per_step"] / ms) if plain else None,
            "stage_ms": {k: round(v, 3) for k, v in stages.items() if v},
            "tree": tree,
            "roofline": roof,
            "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                                         "rel_l2_vs_fp64_exact") if k in cpu},
            "e2e": {"value": n_total / (e2e / 1e3), "unit": "targets/s",
                    "h2d_bytes_per_step": int(t.nbytes + s.nbytes + w.nbytes), "d2h_bytes_per_step": int(ah.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
