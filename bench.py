"""Benchmark: box FGT leaf points/s on the adaptive order-16 configuration.

Workload (one "step" = one full boxfgt, steps 1-6, on the tree below, inputs
resident in HBM): density = sum of 20 seeded Gaussians (centres uniform in the
unit box, widths log-uniform in [1e-3, 1e-2], amplitudes N(0,1)); Legendre
order 16 leaves, periodic unit box; tree uniform to level 8 and refined
adaptively while the leaf Legendre tail exceeds 1e-10, max level 12 (~65.6k
leaves, 16.8M points); nd = 1, delta = 1e-4, eps = 1e-6.  Synthetic data.

Prints one JSON line (rank 0).  Under torchrun every rank runs its own
independent tree (seed + rank): weak scaling, no collective on the data path;
time = max over ranks of the device-timed region.

--impl reference times the reference's CPU algorithm (the oracle: a C
restatement of bfgt/boxfgt.f with the reference's OpenMP loops; no Fortran
compiler is available to build the reference itself) on the host's cores,
same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "boxfgt leaf points/s at rel err 1e-6: split-TC batched vs plain FP64; % roofline"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def make_tree(seed, small=False, minlev=None):
    """The adaptive order-16 workload tree: uniform to level 8 (6 with small),
    or to minlev when given (0: the purely adaptive tree of the tail
    criterion), then refined to a 1e-10 Legendre tail, max level 12."""
    import heat2d_per_box_b200 as hb
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.5, 0.5, (20, 2))
    w = np.exp(rng.uniform(np.log(1e-3), np.log(1e-2), 20))
    a = rng.standard_normal(20)
    g = hb.gauss_params(c, w, a)
    if minlev is None:
        minlev = 6 if small else 8
    return hb.build_adaptive(g, norder=16, ipoly=0, iperiod=1, eps=1e-10, eta=1.0, minlev=minlev, maxlev=12)


def base_level(args):
    """The uniform base level the arguments give the adaptive workload tree."""
    m = getattr(args, "minlev", None)
    return m if m is not None else (6 if getattr(args, "small", False) else 8)


def workload_config(tree, delta, eps, world, minlev=8):
    """The config of the adaptive order-16 workload, identical in both arms."""
    npts = len(tree.leaves()) * tree.npbox
    base = f"uniform to level {minlev} then " if minlev > 0 else ""
    return {"workload": "adaptive order-16 periodic tree, 20 Gaussians (w log-U[1e-3,1e-2], a~N(0,1)), "
                        f"{base}tail<1e-10, max level 12; nd=1",
            "leaves": int(len(tree.leaves())), "points_per_gpu": int(npts), "nd": 1, "delta": delta, "eps": eps,
            "norder": 16,
            "l2": ("inputs larger than L2 (leaf fvals + pot = %.0f MB per step)" if npts * 24 > 126e6 else
                   "inputs fit in L2 (leaf fvals + pot = %.0f MB per step; not flushed between steps)")
                  % (npts * 24 / 1e6),
            "parallelism": f"replicas x{world} (independent trees)"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), line.strip()))

    def mark(self, begin):
        if begin:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for t, r in self.rows if self.t0 is None or (self.t0 - 0.2 <= t <= (self.t1 or t) + 0.2)]
        if not rows:
            rows = [r for _, r in self.rows]
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            f = [x.strip() for x in r.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


def reduce_over_ranks(dist, points, seconds, device):
    """Whole-job figures for replicas: points summed over ranks (each rank has
    its own tree), time as the maximum over ranks.  dist None means one rank."""
    if dist is None:
        return float(points), float(seconds)
    import torch
    t = torch.tensor([float(points), float(seconds)], dtype=torch.float64, device=device)
    p = t[:1].clone()
    s = t[1:].clone()
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return float(p.item()), float(s.item())


def run_reference(args, rank, world):
    """CPU arm: the reference's algorithm (oracle) on the host cores, same workload."""
    from oracle import oracle
    if rank != 0:
        return
    t = make_tree(2, small=args.small, minlev=args.minlev)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    delta, eps = args.delta, args.eps
    for _ in range(args.warmup):
        oracle.boxfgt(t, t.fvals, delta, eps)
    npts = len(t.leaves()) * t.npbox
    # each step is one full transform; cap the number so the arm ends in minutes
    t0 = time.perf_counter()
    oracle.boxfgt(t, t.fvals, delta, eps)
    one = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(math.ceil(120.0 / max(one, 1e-3)))))
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.boxfgt(t, t.fvals, delta, eps)
    el = time.perf_counter() - t0
    v = npts * steps / el
    line = {"metric": METRIC, "value": v, "unit": "leaf points/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": el / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(t, delta, eps, world, base_level(args)),
            "cpu_baseline": {"value": v, "unit": "leaf points/s", "cores": threads, "kind": "port",
                             "sample": f"{steps} full transforms of the workload tree (oracle, OpenMP "
                                       f"{threads} threads; bfgt/boxfgt.f restated in C)"},
            "e2e": {"value": v, "unit": "leaf points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def make_uneven_trees(seed, ntrees=64, lo=1000, hi=50000):
    """Uneven-trees workload: order-8 periodic trees whose leaf counts follow
    targets drawn log-uniform in [lo, hi], each a sum of 5-30 Gaussians (widths
    log-uniform in [2e-3, 5e-2], N(0,1) amplitudes); delta log-uniform in
    [1e-5, 1e-1] per tree.  A tree is refined uniformly to level L or L+1
    (4^L <= target) and then adaptively by the Legendre-tail criterion with a
    tolerance of 1e-6, 1e-9 or 1e-12 (at most 4 more levels): of these six
    trees the one whose leaf count is nearest the target (in log) among those
    inside [lo, hi] is kept (the nearest overall if none is inside)."""
    import heat2d_per_box_b200 as hb
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ntrees):
        ng = int(rng.integers(5, 31))
        c = rng.uniform(-0.5, 0.5, (ng, 2))
        w = np.exp(rng.uniform(np.log(2e-3), np.log(5e-2), ng))
        a = rng.standard_normal(ng)
        target = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        L = max(1, int(np.floor(np.log(target) / np.log(4))))
        t, best = None, (True, np.inf)
        for minlev in (L, L + 1):
            for tail in (1e-6, 1e-9, 1e-12):
                cand = hb.build_adaptive(hb.gauss_params(c, w, a), norder=8, ipoly=0, iperiod=1, eps=tail,
                                         minlev=minlev, maxlev=minlev + 4)
                nl = len(cand.leaves())
                d = (not lo <= nl <= hi, abs(np.log(nl / target)))
                if d < best:
                    t, best = cand, d
        delta = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-1))))
        out.append((t, delta))
    return out


def run_uneven(args, rank, world):
    """64 uneven trees x nd=8 densities, one batch (split precision), captured
    as one CUDA graph, with every plan's kernel shapes autotuned first; also
    the untuned batch, the same plans executed one after another, and the
    batch in FP64 (tile shapes autotuned)."""
    import torch
    import heat2d_per_box_b200 as hb
    torch.cuda.set_device(0)
    nd, eps = 8, 1e-6
    trees = make_uneven_trees(6)[:max(1, min(args.trees, 64))]
    rng = np.random.default_rng(7)
    fv = []
    for t, _ in trees:
        f = np.repeat(t.fvals[:, :, None], nd, axis=2) * rng.uniform(0.5, 2.0, nd)[None, None, :]
        f[t.nchild() > 0] = 0.0
        fv.append(f.reshape(-1))
    F = torch.from_numpy(np.concatenate(fv)).cuda()
    P = torch.zeros_like(F)
    npts = sum(len(t.leaves()) * t.npbox * nd for t, _ in trees)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_graph(batch, steps):
        P.zero_()
        batch.graph_capture(F, P, stream)
        for _ in range(args.warmup):
            batch.graph_launch(stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            batch.graph_launch(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        batch.check()
        return e0.elapsed_time(e1) / steps

    plans = [hb.Plan(t, d, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT) for t, d in trees]
    untuned = hb.Batch(plans)
    ms_untuned = time_graph(untuned, args.steps)
    P_untuned = P.clone()
    untuned.close()
    for pl in plans:
        pl.autotune(stream)
    batch = hb.Batch(plans)
    off = batch.offsets
    ms = time_graph(batch, args.steps)
    same_bits = bool(torch.equal(P, P_untuned))
    # the same transforms as separate plan executes (4 launches per tree)
    fs = [F[off[i]:off[i + 1]] for i in range(len(plans))]
    ps = [P[off[i]:off[i + 1]] for i in range(len(plans))]
    for _ in range(args.warmup):
        for pl, f, p in zip(plans, fs, ps):
            pl.execute(f, p, stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        for pl, f, p in zip(plans, fs, ps):
            pl.execute(f, p, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1) / args.steps
    # per-stage device time of the batched execute (events, outside the graph)
    batch.stage_ms()
    for _ in range(max(3, min(args.steps, 10))):
        batch.execute(F, P, stream)
    st = batch.stage_ms()
    nst = max(st[6], 1)
    stage = {k: round(st[i] / nst, 4) for i, k in enumerate(["form", "reduce", "translate", "eval", "near"])}
    info = batch.info()
    leaves = [len(t.leaves()) for t, _ in trees]
    regimes = [pl.info()["regime"] for pl in plans]
    shapes = [pl.info()["split_shape"] for pl in plans]
    line = {"metric": METRIC, "value": npts / (ms * 1e-3), "unit": "leaf points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16-split/f32acc/f64", "data": "synthetic",
            "config": {"workload": f"{len(trees)} uneven periodic order-8 trees, nd=8, delta log-U[1e-5,1e-1] per tree, "
                                   "eps=1e-6, one batch captured as one CUDA graph, kernel shapes autotuned per plan",
                       "trees": len(trees), "leaves_total": int(sum(leaves)), "leaves_min": int(min(leaves)),
                       "leaves_max": int(max(leaves)), "points_x_nd": int(npts),
                       "regimes": {str(r): int(regimes.count(r)) for r in sorted(set(regimes))},
                       "launches_per_step": info["launches"], "form_items": info["form_items"]},
            "stage_ms": stage, "untuned_value": npts / (ms_untuned * 1e-3), "untuned_ms_per_step": ms_untuned,
            "tuned_same_bits": same_bits,
            "tuned_shapes": {str(k): shapes.count(k) for k in sorted(set(shapes))},
            "unbatched_value": npts / (ms_seq * 1e-3), "unbatched_ms_per_step": ms_seq,
            "batched_over_unbatched": ms_seq / ms}
    batch.close()
    for pl in plans:
        pl.close()
    # the same batch with every plan in FP64 (the plain GPU reference point of
    # the metric), tile shapes autotuned, captured the same way; fewer steps
    # (it is ~5x slower)
    plans64 = [hb.Plan(t, d, eps, nd=nd, precision=hb.BFGT_PREC_FP64) for t, d in trees]
    for pl in plans64:
        pl.autotune(stream)
    b64 = hb.Batch(plans64)
    ms64 = time_graph(b64, max(3, args.steps // 4))
    b64.close()
    for pl in plans64:
        pl.close()
    line["fp64_value"] = npts / (ms64 * 1e-3)
    line["fp64_ms_per_step"] = ms64
    line["split_over_fp64"] = ms64 / ms
    print(json.dumps(line), flush=True)


def run_uniform5(args):
    """Plain FP64 periodic boxfgt on a uniform level-5 quadtree (1024 leaves),
    Legendre order 8 (65,536 points), nd=1, delta=1e-3, eps=1e-9; density = 3
    Gaussians (seed 1, centres uniform in the box, widths uniform in
    [0.05, 0.1], amplitudes uniform in [-1, 1]).  FP64 and split plans, CUDA
    events over back-to-back executes, and the oracle on the host cores."""
    import torch
    import heat2d_per_box_b200 as hb
    from oracle import oracle
    torch.cuda.set_device(0)
    rng = np.random.default_rng(1)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (3, 2)), rng.uniform(0.05, 0.1, 3), rng.uniform(-1, 1, 3))
    t = hb.build_uniform(5, g, norder=8, ipoly=0, iperiod=1)
    delta, eps = 1e-3, 1e-9
    npts = len(t.leaves()) * t.npbox
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    stream = torch.cuda.current_stream()
    res = {}
    for prec in (hb.BFGT_PREC_FP64, hb.BFGT_PREC_SPLIT):
        plan = hb.Plan(t, delta, eps, precision=prec)
        plan.autotune(stream)
        p = torch.zeros_like(f)
        for _ in range(args.warmup):
            plan.execute(f, p, stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(f, p, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        res[prec] = (e0.elapsed_time(e1) / args.steps, plan.info())
        plan.close()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    oracle.boxfgt(t, t.fvals, delta, eps)
    reps, t0 = 0, time.perf_counter()
    while reps < 50 and time.perf_counter() - t0 < 5.0:
        oracle.boxfgt(t, t.fvals, delta, eps)
        reps += 1
    cpu_ms = (time.perf_counter() - t0) / reps * 1e3
    ms64, info = res[hb.BFGT_PREC_FP64]
    line = {"metric": METRIC, "value": npts / (ms64 * 1e-3), "unit": "leaf points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uniform level-5 periodic tree, Legendre order 8, 3 Gaussians (seed 1), nd=1, "
                                   "delta=1e-3, eps=1e-9", "leaves": int(len(t.leaves())), "points": int(npts),
                       "npw": info["npw"], "npwlevel": info["npwlevel"], "regime": info["regime"]},
            "split_value": npts / (res[hb.BFGT_PREC_SPLIT][0] * 1e-3),
            "split_ms_per_step": res[hb.BFGT_PREC_SPLIT][0],
            "cpu_baseline": {"value": npts / (cpu_ms * 1e-3), "unit": "leaf points/s", "cores": threads,
                             "kind": "port", "sample": f"{reps} full transforms (oracle, OpenMP {threads} threads)"}}
    print(json.dumps(line), flush=True)


def run_near16(args):
    """Regime C (near field only): a uniform level-8 periodic tree, Legendre
    order 16 (65,536 leaves, 16.8 M points, as many as the adaptive tree), 20
    Gaussians (seed 2, widths log-uniform in [1e-3, 1e-2], N(0,1)
    amplitudes), nd=1, delta=1e-6, eps=1e-6: every leaf interacts with its 8
    neighbours and itself through the near-field tables.  Device time of the
    near-field stage against the FP64 peak (it is FP64 work in both
    precisions) and against HBM."""
    import torch
    import heat2d_per_box_b200 as hb
    torch.cuda.set_device(0)
    rng = np.random.default_rng(2)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (20, 2)), np.exp(rng.uniform(np.log(1e-3), np.log(1e-2), 20)),
                        rng.standard_normal(20))
    t = hb.build_uniform(8, g, norder=16, ipoly=0, iperiod=1)
    delta, eps = 1e-6, 1e-6
    npts = len(t.leaves()) * t.npbox
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    stream = torch.cuda.current_stream()
    res = {}
    for prec in (hb.BFGT_PREC_FP64, hb.BFGT_PREC_SPLIT):
        plan = hb.Plan(t, delta, eps, precision=prec)
        plan.autotune(stream)
        p = torch.zeros_like(f)
        for _ in range(args.warmup):
            plan.execute(f, p, stream)
        plan.reserve_events(args.steps + 8)
        plan.stage_ms()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(f, p, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        st = plan.stage_ms()
        res[prec] = (e0.elapsed_time(e1) / args.steps, st[4] / max(st[6], 1), plan.info(), plan.work(), p.clone())
        plan.close()
    ms64, near64, info, work, p64 = res[hb.BFGT_PREC_FP64]
    mss, nears, _, _, ps = res[hb.BFGT_PREC_SPLIT]
    lv = t.leaves()
    a = ps.cpu().numpy().reshape(t.nboxes, -1)[lv]
    b = p64.cpu().numpy().reshape(t.nboxes, -1)[lv]
    hbm = peaks()[0]
    line = {"metric": METRIC, "value": npts / (mss * 1e-3), "unit": "leaf points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mss, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16-split/f32acc/f64", "data": "synthetic",
            "config": {"workload": "uniform level-8 periodic tree, Legendre order 16, 20 Gaussians (seed 2), nd=1, "
                                   "delta=1e-6, eps=1e-6 (regime C: near field only)",
                       "leaves": int(len(lv)), "points": int(npts), "regime": info["regime"],
                       "near_pairs": info["nnear_pairs"]},
            "fp64_value": npts / (ms64 * 1e-3), "fp64_ms_per_step": ms64,
            "near_ms": {"split": nears, "fp64": near64},
            "near_roofline": {"flop_per_launch": work["flops_near"], "bytes_per_launch": work["bytes_near"],
                              "fp64_tflops": work["flops_near"] / (near64 * 1e-3) / 1e12,
                              "frac_of_nominal_40tflops_fp64": work["flops_near"] / (near64 * 1e-3) / 40e12,
                              "hbm_gbs": work["bytes_near"] / (near64 * 1e-3) / 1e9,
                              "frac_of_hbm": work["bytes_near"] / (near64 * 1e-3) / 1e9 / hbm},
            "split_rel_l2_err_vs_fp64": float(np.linalg.norm(a - b) / np.linalg.norm(b))}
    print(json.dumps(line), flush=True)


def run_heat5(args):
    """The transforms of one time step of the reaction-diffusion / heat solvers
    (hpots2dadap.f:79, 329-346): the initial-value transform with delta = 4 dt
    and one volume transform per Gauss-Legendre node s_q of [t_n, t_n + dt]
    with delta = 4 (t_n + dt - s_q), 4 nodes, dt = 1e-3.  A uniform level-6
    periodic order-8 tree (4096 leaves), nd = 1, eps = 1e-6, split precision;
    the 5 plans in one batch, the step replayed as one CUDA graph, and the
    same 5 plans in FP64 executed one after another for comparison."""
    import torch
    import heat2d_per_box_b200 as hb
    torch.cuda.set_device(0)
    rng = np.random.default_rng(5)
    ng = 10
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (ng, 2)), np.full(ng, 0.02), rng.standard_normal(ng))
    t = hb.build_uniform(6, g, norder=8, ipoly=0, iperiod=1)
    dt, eps = 1e-3, 1e-6
    xq = (np.polynomial.legendre.leggauss(4)[0] + 1) / 2
    deltas = [4 * dt] + [4 * (1 - x) * dt for x in xq]
    npts = len(t.leaves()) * t.npbox * len(deltas)
    stream = torch.cuda.current_stream()
    res = {}
    for prec in (hb.BFGT_PREC_SPLIT, hb.BFGT_PREC_FP64):
        plans = [hb.Plan(t, d, eps if prec == hb.BFGT_PREC_SPLIT else 1e-9, precision=prec) for d in deltas]
        batch = hb.Batch(plans)
        off = batch.offsets
        F = torch.from_numpy(np.tile(t.fvals.reshape(-1), len(deltas))).cuda()
        P = torch.zeros_like(F)
        assert F.numel() == off[-1]
        batch.graph_capture(F, P, stream)
        for _ in range(args.warmup):
            batch.graph_launch(stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            batch.graph_launch(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        batch.check()
        # per-stage device time (events around plain executes, outside the graph)
        batch.stage_ms()
        for _ in range(10):
            batch.execute(F, P, stream)
        st = batch.stage_ms()
        nst = max(st[6], 1)
        stage = {k: round(st[i] / nst, 5) for i, k in enumerate(["form", "reduce", "translate", "eval", "near"])}
        res[prec] = (e0.elapsed_time(e1) / args.steps, batch.info(), stage)
        batch.close()
        for pl in plans:
            pl.close()
    ms, info, stage = res[hb.BFGT_PREC_SPLIT]
    line = {"metric": METRIC, "value": npts / (ms * 1e-3), "unit": "leaf points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16-split/f32acc/f64", "data": "synthetic",
            "config": {"workload": "one heat/reaction-diffusion time step: 5 transforms (delta = 4 dt and 4 dt (1 - x_q), "
                                   "4 Gauss-Legendre nodes, dt = 1e-3) on a uniform level-6 periodic order-8 tree, "
                                   "nd=1, eps=1e-6, one batch replayed as one CUDA graph",
                       "leaves": int(len(t.leaves())), "transforms": len(deltas), "points_x_transforms": int(npts),
                       "deltas": deltas, "launches_per_step": info["launches"]},
            "stage_ms": stage,
            "fp64_value": npts / (res[hb.BFGT_PREC_FP64][0] * 1e-3),
            "fp64_ms_per_step": res[hb.BFGT_PREC_FP64][0], "fp64_stage_ms": res[hb.BFGT_PREC_FP64][2]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--delta", type=float, default=1e-4)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "split"])
    ap.add_argument("--small", action="store_true", help="level-6 base tree (for profiler captures)")
    ap.add_argument("--minlev", type=int, default=None,
                    help="uniform base level of the adaptive tree (default 8; 0: purely adaptive)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="adaptive16", choices=["adaptive16", "uneven64", "uniform5", "heat5", "near16"],
                    help="adaptive16: one adaptive order-16 tree (default); uneven64: 64 uneven order-8 trees, "
                         "nd=8, batched in one graph; uniform5: the plain FP64 case on a uniform level-5 order-8 "
                         "tree; heat5: the 5 transforms of one heat-solver time step, batched in one graph; "
                         "near16: regime C (near field only) on a uniform level-8 order-16 tree")
    ap.add_argument("--trees", type=int, default=64,
                    help="uneven64: use only the first N of the 64 trees (for profiler captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "uneven64":
        run_uneven(args, rank, world)
        return
    if args.workload == "uniform5":
        run_uniform5(args)
        return
    if args.workload == "heat5":
        run_heat5(args)
        return
    if args.workload == "near16":
        run_near16(args)
        return

    import torch
    import heat2d_per_box_b200 as hb

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    tree = make_tree(2 + rank, small=args.small, minlev=args.minlev)
    leaves = tree.leaves()
    npts = len(leaves) * tree.npbox
    precs = {"fp64": [hb.BFGT_PREC_FP64], "split": [hb.BFGT_PREC_SPLIT]}.get(args.precision)
    if precs is None:
        precs = [hb.BFGT_PREC_FP64]
        try:
            hb.Plan(tree, args.delta, args.eps, precision=hb.BFGT_PREC_SPLIT).close()
            precs = [hb.BFGT_PREC_SPLIT, hb.BFGT_PREC_FP64]
        except hb.BfgtError:
            pass

    hbm, bf16, bf16s, peak_src = peaks()
    f = torch.from_numpy(tree.fvals.reshape(-1)).to(dev)
    results = {}
    stream = torch.cuda.current_stream()
    clocks = None
    for prec in precs:
        plan = hb.Plan(tree, args.delta, args.eps, precision=prec)
        plan.autotune(stream)  # fastest compiled shapes: FP64 tiles, or the split kernels' groups and staging
        pot = torch.zeros_like(f)
        for _ in range(args.warmup):
            plan.execute(f, pot, stream)
        plan.reserve_events(args.steps + 8)
        torch.cuda.synchronize()
        plan.stage_ms()
        sampler = ClockSampler(dev.index) if prec == precs[0] else None
        if sampler:
            sampler.start()
            time.sleep(0.4)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.mark(True)
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(f, pot, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if sampler:
            sampler.mark(False)
        ms = e0.elapsed_time(e1)
        job_points, sec = reduce_over_ranks(dist, npts * args.steps, ms * 1e-3, dev)
        ms = sec * 1e3
        st = plan.stage_ms()
        if sampler:
            clocks = sampler.stop()
        nst = max(st[6], 1)
        work = plan.work()
        info = plan.info()
        stage_names = ["form", "reduce", "translate", "eval", "near"]
        stage_avg = {nm: st[i] / nst for i, nm in enumerate(stage_names)}
        results[prec] = dict(ms=ms, job_points=job_points, stage=stage_avg, work=work, info=info, plan=plan)
        # correctness of this run against a fresh single execute is covered by the tests

    main_prec = precs[0]
    R = results[main_prec]
    ms_step = R["ms"] / args.steps
    value = R["job_points"] / (R["ms"] * 1e-3)
    # roofline of the dominant kernel (largest share of the step)
    stg = R["stage"]
    dom = max(("form", "eval", "near"), key=lambda k: stg[k])
    w = R["work"]
    dom_ms = stg[dom]
    fl = {"form": w["flops_form"], "eval": w["flops_eval"], "near": w["flops_near"]}[dom]
    by = {"form": w["bytes_form"], "eval": w["bytes_eval"], "near": w["bytes_near"]}[dom]
    tcf = {"form": w["tc_flops_form"], "eval": w["tc_flops_eval"], "near": 0.0}[dom]
    hbm_ach = by / (dom_ms * 1e-3) / 1e9
    if main_prec == hb.BFGT_PREC_SPLIT and tcf > 0:
        tc_ach = fl / (dom_ms * 1e-3) / 1e12
        if tc_ach / bf16 >= hbm_ach / hbm:
            roof = {"bound": "tensor", "achieved": tc_ach, "peak": bf16, "unit": "TFLOP/s", "frac": tc_ach / bf16}
        else:
            roof = {"bound": "hbm", "achieved": hbm_ach, "peak": hbm, "unit": "GB/s", "frac": hbm_ach / hbm}
        roof["tensor_flops_issued_per_launch"] = tcf
        roof["tensor_issue_rate_tflops"] = tcf / (dom_ms * 1e-3) / 1e12
    else:
        roof = {"bound": "hbm", "achieved": hbm_ach, "peak": hbm, "unit": "GB/s", "frac": hbm_ach / hbm}
        roof["fp64_tflops"] = fl / (dom_ms * 1e-3) / 1e12
        roof["fp64_frac_of_nominal_40tf"] = roof["fp64_tflops"] / 40.0
    roof.update({"kernel": dom, "kernel_ms": dom_ms, "algorithmic_flop_per_launch": fl,
                 "algorithmic_bytes_per_launch": by, "peak_source": peak_src, "traffic": None})
    prof = ROOT / "profiles" / "traffic.json"
    if prof.exists():
        try:
            tr = json.loads(prof.read_text()).get(f"{'split' if main_prec else 'fp64'}_{dom}")
            if tr:
                roof["traffic"] = tr
        except Exception:
            pass

    # end-to-end through the drop-in symbol boxfgt_ (the call a Fortran solver
    # makes) with pinned host arrays: the first call builds and caches the
    # plan (reported separately), the timed calls find it in the cache; the
    # host<->device copies and the step-0 lookup are inside the timed region.
    # As the reference's solvers do (hpots2dadap.f:97-101, 321-325), pot is
    # zeroed before each call; that fill is the caller's work and is outside
    # the timed calls (one event pair per call)
    e2e = None
    nelem = tree.nboxes * tree.npbox
    hf = torch.from_numpy(tree.fvals.reshape(-1).copy()).pin_memory()
    hp = torch.zeros(nelem, dtype=torch.float64).pin_memory()
    hf_np, hp_np = hf.numpy(), hp.numpy()
    itree = tree.itree.copy()
    ti = np.zeros(20)
    hb.plan_cache_clear()
    hb.set_default_precision(main_prec)

    def dropin():
        hb.boxfgt(1, 2, args.delta, args.eps, tree.ipoly, tree.iperiod, tree.norder, tree.npbox, tree.nboxes,
                  tree.nlevels, tree.ltree, itree, tree.iptr, tree.centers, tree.boxsize, hf_np, 1, hp_np, None, None,
                  0, 0, None, 0, None, None, None, ti)

    t0 = time.perf_counter()
    dropin()
    first_ms = (time.perf_counter() - t0) * 1e3
    first_pre_ms = ti[0] * 1e3
    ne = max(3, min(args.steps, 50))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ne)]
    for a, b in ev:
        hp_np.fill(0.0)
        a.record(stream)
        dropin()
        b.record(stream)
    torch.cuda.synchronize()
    t_calls = sum(a.elapsed_time(b) for a, b in ev) * 1e-3
    cache = hb.plan_cache_info()
    moved = hb.last_call_bytes()
    e2e_points, el = reduce_over_ranks(dist, npts * ne, t_calls, dev)
    e2e = {"value": e2e_points / el, "unit": "leaf points/s", "h2d_bytes_per_step": moved["h2d"],
           "d2h_bytes_per_step": moved["d2h"],
           "api": "boxfgt_ (gfortran-ABI drop-in; plan cached after the first call; pinned host arrays; pot zeroed "
                  "by the caller before each call, so only fvals goes up)",
           "ms_per_call": el / ne * 1e3, "lookup_ms_per_call": ti[0] * 1e3, "first_call_ms": first_ms,
           "first_call_precompute_ms": first_pre_ms, "cache_hits": cache["hits"],
           "pcie_gbs": (moved["h2d"] + moved["d2h"]) / (el / ne) / 1e9}
    # the same calls with ordinary (pageable) host arrays, as a Fortran solver
    # has them: the library stages them through pinned chunks
    pf = tree.fvals.reshape(-1).copy()
    pp = np.zeros(nelem)

    def dropin_pageable():
        hb.boxfgt(1, 2, args.delta, args.eps, tree.ipoly, tree.iperiod, tree.norder, tree.npbox, tree.nboxes,
                  tree.nlevels, tree.ltree, itree, tree.iptr, tree.centers, tree.boxsize, pf, 1, pp, None, None,
                  0, 0, None, 0, None, None, None, ti)

    dropin_pageable()
    evp = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ne)]
    for a, b in evp:
        pp.fill(0.0)
        a.record(stream)
        dropin_pageable()
        b.record(stream)
    torch.cuda.synchronize()
    t_pg = sum(a.elapsed_time(b) for a, b in evp) * 1e-3
    pg_points, pg_el = reduce_over_ranks(dist, npts * ne, t_pg, dev)
    e2e["pageable"] = {"value": pg_points / pg_el, "ms_per_call": pg_el / ne * 1e3,
                       "same_result_as_pinned": bool(np.array_equal(pp, hp_np))}
    hb.set_default_precision(hb.BFGT_PREC_FP64)
    hb.plan_cache_clear()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        ref = oracle.boxfgt(tree, tree.fvals, args.delta, args.eps).reshape(tree.nboxes, -1)[leaves]
        # accuracy of each measured GPU path against the oracle on this tree
        # (one more execute, outside the timed regions)
        for prec, r in results.items():
            p1 = torch.zeros_like(f)
            r["plan"].execute(f, p1, stream)
            r["plan"].check()
            got = p1.cpu().numpy().reshape(tree.nboxes, -1)[leaves]
            r["err_vs_oracle"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        reps = 0
        t0 = time.perf_counter()
        while True:
            oracle.boxfgt(tree, tree.fvals, args.delta, args.eps)
            reps += 1
            if time.perf_counter() - t0 > 10.0 or reps >= 20:
                break
        el = time.perf_counter() - t0
        cpu = {"value": npts * reps / el, "unit": "leaf points/s", "cores": threads, "kind": "port",
               "sample": f"{reps} full transforms of the same tree (oracle: bfgt/boxfgt.f restated in C, "
                         f"OpenMP {threads} threads)"}

    nlaunch_step = R["info"]["launches"]
    line = {
        "metric": METRIC, "value": value, "unit": "leaf points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if main_prec == hb.BFGT_PREC_FP64 else "f16-split/f32acc/f64",
        "data": "synthetic",
        "config": workload_config(tree, args.delta, args.eps, world, base_level(args)),
        "plan": {"npw": R["info"]["npw"], "npwlevel": R["info"]["npwlevel"],
                 "precision": "split" if main_prec == hb.BFGT_PREC_SPLIT else "fp64",
                 "tuned_shape": R["info"]["split_shape"] if main_prec == hb.BFGT_PREC_SPLIT else
                 [R["info"]["form_tile"], R["info"]["eval_tile"]]},
        "roofline": roof,
        "stage_ms": {k: round(v, 5) for k, v in stg.items()},
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": nlaunch_step * args.steps,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    for prec, r in results.items():
        if "err_vs_oracle" in r:
            key = "split" if prec == hb.BFGT_PREC_SPLIT else "fp64"
            line[f"{key}_rel_l2_err_vs_oracle"] = r["err_vs_oracle"]
    if hb.BFGT_PREC_FP64 in results and main_prec != hb.BFGT_PREC_FP64:
        F = results[hb.BFGT_PREC_FP64]
        line["fp64_value"] = F["job_points"] / (F["ms"] * 1e-3)
        line["split_over_fp64"] = value / line["fp64_value"]
        line["fp64_stage_ms"] = {k: round(v, 5) for k, v in F["stage"].items()}
        # accuracy of the measured split transform against the FP64 one on this
        # tree (one more execute of each, outside the timed regions; non-leaf
        # boxes hold zeros in both)
        outs = []
        for prec in (main_prec, hb.BFGT_PREC_FP64):
            p1 = torch.zeros_like(f)
            results[prec]["plan"].execute(f, p1, stream)
            outs.append(p1)
        torch.cuda.synchronize()
        line["split_rel_l2_err_vs_fp64"] = ((outs[0] - outs[1]).norm() / outs[1].norm()).item()
        # the FP64 reference point's own rate (form and eval FLOP of the FP64
        # plan over their stage times; 40 TFLOP/s is B200's nominal FP64 rate)
        fw = F["work"]
        tf = (fw["flops_form"] + fw["flops_eval"]) / ((F["stage"]["form"] + F["stage"]["eval"]) * 1e-3) / 1e12
        line["fp64_path"] = {"form_eval_tflops": tf, "frac_of_nominal_40tflops": tf / 40.0}
    for r in results.values():
        r["plan"].close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
