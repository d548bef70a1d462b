#!/usr/bin/env python
"""Benchmark of the delta-push centrality engine on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config cached-all|pr16]

Default workload (`cached-all`): `--measure all` -- PageRank d = 0.85 eps 1e-2,
Katz beta = 1, alpha = 0.9 / lambda1 eps 1e-6, eigenvector with lambda1 from FP64
power iteration eps 1e-6 -- over one stream of a seeded R-MAT graph of scale 24
(16.8M vertices), edge factor 16, (a, b, c, d) = (0.57, 0.19, 0.19, 0.05), seed
2, symmetric, fully cached in HBM, FP32 values and residuals. One step is one
solve from initialisation until no vertex is pending (time to eps). The
metric is GTEPS: adjacency entries pushed per second (an entry pushed in an
`all` run updates all three measures of its target).

`value` times solves with the graph already resident in HBM; `e2e` times the
same solve through the C ABI from pinned host buffers, with the offsets and
edge upload and the result readback inside the timed region. A solve does
not shard without a residual exchange, so N GPUs run N independent replicas
(weak scaling, no collective on the data path). `--impl reference` runs the
CPU port of the reference engine (oracle/) on the host cores for a bounded
sample (its first passes) of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
LOG_DIR = None   # --log-dir: where CLI runs leave their stdout
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (scale, edge_factor, seed, measure)
    "cached-all": (24, 16, 2, "all"),
    "pr24": (24, 16, 2, "pr"),
    "pr16": (16, 16, 1, "pr"),
    "ppr256": (24, 16, 2, "ppr"),
    "adjoint22": (22, 16, 4, "adjoint"),
    "ooc28": (28, 32, 3, "ooc"),
}


T_START = time.perf_counter()

# DRAM bytes (read + write) of the push kernels per solve, GB, from the ncu captures summarised in
# profiles/ (dram__bytes_read.sum + dram__bytes_write.sum, one pass per launch, three solves)
TRAFFIC_CAPTURES = {
    ("cached-all", 24): (307.0, "GB per solve: k_push 118.3 + k_segments 188.7, ncu over three solves of "
                                "`bench.py --steps 1 --warmup 0 --no-cpu-baseline --errors off --no-graph` "
                                "(profiles/traffic_all_rmat24.md); `achieved` and `traffic` are both per solve"),
}


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write("[bench %7.1fs] %s\n" % (time.perf_counter() - T_START, msg))
    sys.stderr.flush()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cached-all", choices=sorted(CONFIGS))
    ap.add_argument("--scale", type=int, default=None, help="override the graph scale (smaller test runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--errors", default="on", choices=["on", "off"],
                    help="error against the FP64 oracle solution, like-for-like run and the reference engine's error")
    ap.add_argument("--no-graph", action="store_true", help="host-driven pass loop instead of the CUDA graph")
    ap.add_argument("--ev-project", default="on", choices=["on", "off"],
                    help="FP64 eigenvector normalisation step (remove the principal-eigenvector component of the "
                         "eigenvector residual each pass); the `all` run does not reach eps 1e-6 at scale 24 without it")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="also run this repo's CLI and the reference CLI (built from source) on the same EGR file")
    ap.add_argument("--ref-passes", type=int, default=200, help="pass cap of the CLI runs for 'all'")
    ap.add_argument("--ooc-budget-gb", type=float, default=16.0,
                    help="device memory left to the CLIs in the out-of-core run (the rest is held as ballast)")
    ap.add_argument("--ooc-dir", default=None, help="directory for the out-of-core EGR file (default: temp dir)")
    ap.add_argument("--ooc-measures", default="pr", help="comma-separated measures of the out-of-core run")
    ap.add_argument("--ooc-mode", default="pinned", choices=["pinned", "pipeline"],
                    help="which of this repo's out-of-core arms is the headline")
    ap.add_argument("--ooc-pipeline", default="on", choices=["on", "off"],
                    help="also run this repo's CLI with the reference's stream/gather pipeline")
    ap.add_argument("--ooc-ref", default="on", choices=["on", "off"], help="also run the reference CLI out of core")
    ap.add_argument("--batch-width", type=int, default=0, choices=[0, 32, 64, 128, 256],
                    help="batched PPR: fixed batch width instead of the autotuner's")
    ap.add_argument("--ppr-eps", default="1e-4,2e-9",
                    help="batched PPR: eps points as multiples of the seed mass (the first is the headline; "
                         "2e-9 brings the L1 error against the FP64 oracle under 1e-2 on 16.8M vertices, where "
                         "1e-7 leaves about 0.2)")
    ap.add_argument("--ppr-seq-limit", type=int, default=64,
                    help="batched PPR: sequential solves timed at the points after the first (scaled to 256)")
    ap.add_argument("--dense-groups", type=int, default=-1,
                    help="batched PPR: active-group threshold of the group-parallel hub scatter (-1: default)")
    ap.add_argument("--greedy", default="off", choices=["on", "off"], help="with --batch-width: greedy row push")
    ap.add_argument("--list-frac", type=float, default=0.5,
                    help="per-chunk list/range rule of the device loop (the reference's --list-frac)")
    ap.add_argument("--log-dir", default=None, help="keep the stdout of every CLI run in this directory")
    ap.add_argument("--hub-order", default="auto", choices=["auto", "first", "last", "table", "launch-first"],
                    help="where the high-degree lists go in each pass of the device loop (auto: launch-first when "
                         "the chunks are swept one by one, else first)")
    ap.add_argument("--chunk-sweep", default="auto", choices=["auto", "on", "off"],
                    help="cached pushes one chunk per launch in chunk order (auto: when there are several chunks)")
    ap.add_argument("--error-runs", type=int, default=3,
                    help="solves per error figure (each engine's figure is the median over them)")
    ap.add_argument("--sweep-demand", type=float, default=0.5,
                    help="with a chunk sweep: sweep only the passes whose pending entries reach this fraction of m "
                         "(the others run as one launch); 0 sweeps every pass")
    ap.add_argument("--hub-targets", type=int, default=-1,
                    help="shared-memory aggregation of the k highest-degree targets (0: off; -1: 4096 for all; "
                         "for one measure 2048 with a chunk sweep, else 16384)")
    ap.add_argument("--ev-init", default="fp64", choices=["fp64", "reference"],
                    help="eigenvector initial residual from the FP64 lambda1 (default) or from lambda1 rounded to "
                         "float as the reference does")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [l.split(", ") for l in self.f.read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) >= 9 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local, dist


def push_bytes(nm, log):
    """Algorithmic bytes of the push kernels over the logged passes, counting only
    the measures that carry a nonzero weight: 4 E_p (indices) + 8 per entry and
    measure pushed (residual RMW) + 16 P (offsets pair) + 16 per vertex and measure
    taken (residual exchange, value RMW). With one measure this is the model
    4 E_p + 8 E_p + P (16 + 16)."""
    ep = sum(int(l.pushed) for l in log)
    pv = sum(int(l.pending) for l in log)
    lanes = sum(int(l.lanes) for l in log)
    taken = sum(int(l.taken) for l in log)
    return 4 * ep + 8 * lanes + 16 * pv + 16 * taken, ep, pv


def top_k(v, k):
    """Indices of the k largest entries of v, ties broken by the lower index."""
    k = min(k, len(v))
    if k == 0:
        return np.zeros(0, dtype=np.int64)
    kth = np.partition(v, len(v) - k)[len(v) - k]
    cand = np.nonzero(v >= kth)[0]
    return cand[np.lexsort((cand, -v[cand]))[:k]]


def unit_signed(v):
    """Unit L2 norm with the sign fixed by the sum, as the reference's comparison tool treats
    eigenvectors (tools/centrality_reference.cu:71-76)."""
    v = np.asarray(v, dtype=np.float64)
    s, t = float(np.dot(v, v)), float(v.sum())
    return v * ((-1.0 if t < 0 else 1.0) / np.sqrt(s)) if s > 0 else v


def error_vs_fp64(measure, ref, x):
    """L1 error relative to the FP64 solution's mass, max per-vertex error and top-1000 overlap."""
    r = np.asarray(ref, dtype=np.float64)
    xx = np.asarray(x, dtype=np.float32).astype(np.float64)
    if measure == "ev":
        r, xx = unit_signed(r), unit_signed(xx)
    d = np.abs(xx - r)
    return {"l1_rel": float(d.sum() / np.abs(r).sum()), "max_abs": float(d.max()),
            "top1000": int(len(np.intersect1d(top_k(r, 1000), top_k(xx, 1000))))}


def fp64_solutions(n, d_idx, d_adj, kinds, alpha, device):
    """FP64 Jacobi / power-iteration solutions on the device (tol 1e-9, as the reference's oracle)."""
    import excent_b200 as X
    out = {}
    for k in kinds:
        t0 = time.perf_counter()
        out[k], it = X.reference_fp64(n, d_idx, d_adj, k, alpha=alpha if k == "katz" else 0.0, beta=1.0, tol=1e-9,
                                      device=device)
        log(f"FP64 {k}: {it} iterations, {time.perf_counter() - t0:.1f}s")
    return out


def median_errors(runs):
    """Per measure and metric, the median over runs (each a {measure: error_vs_fp64} dict), with the
    L1 range of the runs."""
    out = {}
    for k in runs[0]:
        out[k] = {q: float(np.median([r[k][q] for r in runs])) for q in ("l1_rel", "max_abs", "top1000")}
        out[k]["l1_range"] = [min(r[k]["l1_rel"] for r in runs), max(r[k]["l1_rel"] for r in runs)]
        out[k]["max_abs_range"] = [min(r[k]["max_abs"] for r in runs), max(r[k]["max_abs"] for r in runs)]
    return out


def error_report(a, n, m, d_idx, d_adj, idx_np, adj_np, v0, e, eng, meas, measure, lam, device):
    """Error of this engine's results against the FP64 oracle solution, in the timed configuration and
    like for like with the reference engine (eigenvector initial residual from lambda1 rounded to float,
    no FP64 eigenvector step, the same pass cap), beside the reference engine's own error: its CLI
    (src/excent.cu built from source) on the same EGR file and constants, results through --dump
    (src/excent.cu:763-777). Both engines add FP32 residuals with atomics in a run-dependent order,
    so each figure is the median of --error-runs solves, with the range of their L1 errors."""
    import shutil

    import excent_b200 as X
    kinds = ["pr", "katz", "ev"] if measure == "all" else [measure]
    alpha = 0.9 / lam if lam else None
    ref = fp64_solutions(n, d_idx, d_adj, kinds, alpha, device)
    rep = {"oracle": "FP64 Jacobi (PageRank, Katz) and power iteration (eigenvector) on the device to a relative "
                     "change of 1e-9 (tools/centrality_reference.cu:184-214); the eigenvector is compared as a "
                     "unit vector with its sign fixed by its sum",
           "runs_per_figure": a.error_runs}
    ours = []
    for _ in range(a.error_runs):
        eng.solve(list_frac=a.list_frac, use_graph=not a.no_graph)
        ours.append({k: error_vs_fp64(k, ref[k], eng.read(i)) for i, k in enumerate(kinds)})
    rep["timed_config"] = median_errors(ours)
    if measure == "all":
        meas_l = X.measures("all", alpha=alpha, beta=1.0, lam=lam, eps_pr=1e-2, eps_katz=1e-6, eps_ev=1e-6,
                            ev_init_fp64=False)
        eng2 = X.Engine(n, m, meas_l, v0, e, device=device)
        eng2.upload_device(d_idx, d_adj)
        eng2.set_hub_targets(min(4096, n))
        eng2.set_hub_order(a.hub_order)
        eng2.set_chunk_sweep({"auto": "auto", "on": True, "off": False}[a.chunk_sweep])
        eng2.set_sweep_demand(a.sweep_demand)
        lfl = []
        for _ in range(a.error_runs):
            st = eng2.solve(list_frac=a.list_frac, max_passes=a.ref_passes)
            lfl.append({k: error_vs_fp64(k, ref[k], eng2.read(i)) for i, k in enumerate(kinds)})
        rep["like_for_like"] = {"ev_init": "lambda1 rounded to float", "ev_project": "off",
                                "max_passes": a.ref_passes, "passes": st.passes, **median_errors(lfl)}
        eng2.close()
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "excent")
    if not os.path.exists(ref_bin):
        rep["reference_engine"] = {"unavailable": "reference CLI not built (oracle/Makefile)"}
        return rep
    d = tempfile.mkdtemp(prefix="excent_err_")
    try:
        path = os.path.join(d, "g.egr")
        X.write_egr(path, idx_np, adj_np)
        args = [path, "--measure", measure, "--cache", "chunks", "--stream-ratio", "2", "--dump",
                os.path.join(d, "out"), "--max-passes", str(a.ref_passes), "--count-pushes"]
        if measure == "all":
            args += ["--alpha", "%.9g" % alpha, "--beta", "1", "--lambda", "%.17g" % lam, "--eps-katz", "1e-6",
                     "--eps-ev", "1e-6"]
        import re
        runs, passes, pushed_x_m = [], [], []
        for _ in range(a.error_runs):
            r = subprocess.run([ref_bin, *args], capture_output=True, text=True, timeout=1800,
                               env=dict(os.environ, HOME=d))
            if r.returncode != 0:
                rep["reference_engine"] = {"error": (r.stderr or r.stdout)[-300:]}
                return rep
            mp = re.search(r"^passes (\d+)", r.stdout, re.M)
            passes.append(int(mp.group(1)) if mp else None)
            mx = re.search(r"edges pushed: ([0-9.]+) x", r.stdout)
            pushed_x_m.append(float(mx.group(1)) if mx else None)
            runs.append({k: error_vs_fp64(k, ref[k], np.fromfile(os.path.join(d, f"out.{k}.bin"), dtype=np.float32))
                         for k in kinds})
        rep["reference_engine"] = {"args": " ".join(args[1:]).replace(d, "<tmp>"), "passes": passes,
                                   "pushed_x_m": pushed_x_m, **median_errors(runs)}
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return rep


def run_ours(a, world, rank, local, dist):
    import torch

    import excent_b200 as X
    torch.cuda.set_device(local)
    scale, ef, seed, measure = CONFIGS[a.config]
    scale = a.scale or scale
    g = X.DeviceGraph(scale, ef, seed, device=local)
    n, m = g.n, g.m
    d_idx, d_adj, _ = g.device_ptrs()
    log(f"graph scale {scale}: n={n} m={m}")
    v1 = None
    if measure == "all":
        v1 = torch.empty(n, dtype=torch.float32, device="cuda")
        par = X.params_fp64(n, d_idx, d_adj, device=local, v1_out=v1)
        lam = par["lambda"]
        log(f"lambda1 {lam:.6f} after {par['sweeps']} sweeps")
        meas = X.measures("all", alpha=0.9 / lam, beta=1.0, lam=lam, eps_pr=1e-2, eps_katz=1e-6, eps_ev=1e-6,
                          ev_init_fp64=a.ev_init == "fp64")
    else:
        lam = None
        meas = X.measures("pr", eps_pr=1e-2)
    nm = meas.nm
    # pinned host copy of the graph for the end-to-end leg
    h_idx = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    h_adj = torch.empty(max(m, 1), dtype=torch.int32, pin_memory=True)
    g.download(h_idx, h_adj)
    idx_np = h_idx.numpy().view(np.uint64)
    v0, e = X.plan_chunks(idx_np, X.chunk_cap(m))
    eng = X.Engine(n, m, meas, v0, e, device=local)
    eng.upload_device(d_idx, d_adj)
    if v1 is not None and a.ev_project == "on":
        eng.ev_project(v1)
    # hub-target slots: fewer when each launch covers one chunk (a slot pays only with many adds per flush)
    sweeping = a.chunk_sweep == "on" or (a.chunk_sweep == "auto" and len(v0) > 1)
    hub_k = a.hub_targets if a.hub_targets >= 0 else min((2048 if sweeping else 16384) if nm == 1 else 4096, n)
    eng.set_hub_targets(hub_k)
    eng.set_hub_order(a.hub_order)
    eng.set_chunk_sweep({"auto": "auto", "on": True, "off": False}[a.chunk_sweep])
    eng.set_sweep_demand(a.sweep_demand)
    use_graph = not a.no_graph
    for _ in range(a.warmup):
        s = eng.solve(list_frac=a.list_frac, use_graph=use_graph)
        log(f"warmup solve: {s.passes} passes, {s.pushed} entries pushed")
    st = torch.cuda.ExternalStream(eng.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = eng.launches()
    clocks.start()
    ev0.record(st)
    pushed = 0
    passes = []
    for _ in range(a.steps):
        s = eng.solve(list_frac=a.list_frac, use_graph=use_graph)
        pushed += s.pushed
        passes.append(s.passes)
    ev1.record(st)
    torch.cuda.synchronize()
    ck = clocks.stop()
    launches = eng.launches() - l0
    t = ev0.elapsed_time(ev1) / 1e3
    if dist:
        t, pushed_all = reduce_over_ranks(t, pushed, dist, "cuda")
    else:
        pushed_all = float(pushed)
    value = pushed_all / t / 1e9
    log(f"timed: {a.steps} solves in {t:.3f}s, {value:.3f} GTEPS")

    # end to end through the C ABI: host buffers in, host results out
    outs = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(nm)]
    h2d = (n + 1) * 8 + m * 4
    d2h = n * 4 * nm
    e_pushed = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(st)
    w0 = time.perf_counter()
    for _ in range(a.steps):
        eng.upload_offsets(h_idx.data_ptr())
        eng.load_cache(0, m, h_adj.data_ptr())
        s = eng.solve(list_frac=a.list_frac, use_graph=use_graph)
        e_pushed += s.pushed
        for i in range(nm):
            eng.read(i, out=outs[i])
    ev1.record(st)
    torch.cuda.synchronize()
    te = ev0.elapsed_time(ev1) / 1e3
    te_wall = time.perf_counter() - w0
    if dist:
        te, e_pushed = reduce_over_ranks(te, e_pushed, dist, "cuda")

    log(f"e2e: {a.steps} solves in {te:.3f}s")
    # roofline of the dominant kernel (push + its hub tail), per-kernel events on a profiled solve
    eng.profile(True)
    eng.solve(list_frac=a.list_frac, use_graph=False)
    s, plog = eng.stats(with_log=True)
    prof, ppasses = eng.profile_read()
    eng.profile(False)
    b_alg, ep, pv = push_bytes(nm, plog)
    t_push = (prof["push"] + prof["hub"]) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = b_alg / t_push / 1e9 if t_push > 0 else 0.0
    snap_bytes = ppasses * (n * 4 * nm + n / 8)
    t_all = sum(prof.values()) / 1e3
    # the second roofline of the scatter: one reduction per entry to a random vertex of r,
    # whose array (67 MB for one measure) sits in L2; the ceiling is measured here
    red_peak = eng.scatter_peak()
    red_uniform = X.reduction_peak(n, vec4=nm > 1, device=local)
    red_achieved = ep / t_push if t_push > 0 else 0.0
    # DRAM traffic of the push kernels per solve, from an ncu capture of this workload (ncu cannot
    # run inside the timed process); other workloads: not captured
    traffic, traffic_note = None, "no ncu capture of this workload"
    if (a.config, scale) in TRAFFIC_CAPTURES:
        traffic, traffic_note = TRAFFIC_CAPTURES[(a.config, scale)]
    result = {
        "metric": "GTEPS (adjacency entries pushed per second, solve to eps)",
        "value": round(value, 4),
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": round(t / a.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded R-MAT, generated on the device)",
        "config": {"workload": f"{measure} on R-MAT scale {scale} EF {ef} seed {seed}", "cache": "fully HBM-cached",
                   "n": n, "m": m, "chunks": int(len(v0)), "measure": measure, "lambda1": lam,
                   "eps": [float(meas.eps[i]) for i in range(nm)], "passes_per_solve": passes[-1],
                   "pushed_per_solve": int(pushed / a.steps), "time_to_eps_ms": round(t / a.steps * 1e3, 3),
                   "l2_note": "inputs larger than L2 (edge cache %.2f GB)" % (m * 4 / 1e9),
                   "cuda_graph": use_graph, "parallelism": f"{world} independent replicas",
                   "ev_init": a.ev_init, "ev_project": a.ev_project if measure == "all" else None,
                   "hub_targets": hub_k, "list_frac": a.list_frac,
                   "hub_order": a.hub_order, "chunk_sweep": a.chunk_sweep, "sweep_demand": a.sweep_demand},
        "e2e": {"value": round(e_pushed / te / 1e9, 4), "unit": "GTEPS", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": round(te / a.steps * 1e3, 3),
                "wall_ms_per_step": round(te_wall / a.steps * 1e3, 3)},
        "roofline": {"bound": "hbm", "kernel": "k_push + k_segments (one logical push: the takes, the short lists, then the queued long-list segments)",
                     "achieved": round(achieved, 1), "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "traffic_note": traffic_note,
                     "alg_bytes_per_solve": int(b_alg), "push_ms_per_solve": round(t_push * 1e3, 3),
                     "pass_ms_per_solve": round(t_all * 1e3, 3),
                     "pass_achieved_gbs": round((b_alg + snap_bytes) / t_all / 1e9, 1) if t_all else None,
                     "kernel_ms": {k: round(v, 3) for k, v in prof.items()},
                     "l2_reduction": {"achieved": round(red_achieved / 1e9, 2),
                                      "peak": round(red_peak / 1e9, 2), "unit": "G reductions/s",
                                      "frac": round(red_achieved / red_peak, 4) if red_peak else None,
                                      "peak_source": "excent_engine_scatter_peak in this run: one %s per entry of "
                                                     "the edge cache, in cache order, to its target (no take, no "
                                                     "list bookkeeping)" % ("red.global.add.v4.f32" if nm > 1
                                                                            else "red.global.add.f32"),
                                      "uniform_random_peak": round(red_uniform / 1e9, 2),
                                      "achieved_note": "entries pushed (one reduction each, a shared-memory "
                                                       "atomic for hub targets) per second of push-kernel time"}},
        "clocks": ck,
        "gpu_launches": int(launches),
    }
    log(f"profiled solve: {prof}")
    if rank == 0 and world == 1 and a.errors == "on":
        result["error_vs_fp64"] = error_report(a, n, m, d_idx, d_adj, idx_np, h_adj.numpy()[:m], v0, e, eng, meas,
                                               measure, lam, local)
        log(f"error vs FP64: {json.dumps(result['error_vs_fp64'])}")
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(n, idx_np, h_adj.numpy()[:m], meas, measure, lam)
    if rank == 0 and world == 1 and a.ref_gpu:
        result["cli_vs_reference_gpu"] = cli_compare(a, idx_np, h_adj.numpy()[:m], measure, meas, lam, local)
    g.close()
    eng.close()
    return result


def ppr_queries(n, nq=256, seed=7, max_size=4096):
    """Seed sets: sizes floor(exp(U[0, ln 4096])) clamped to [1, 4096], vertices uniform without replacement."""
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.floor(np.exp(rng.uniform(0, np.log(max_size), nq))).astype(np.int64), 1, max_size)
    return [np.sort(rng.choice(n, int(k), replace=False)).astype(np.int32) for k in sizes]


def ppr_point(a, X, torch, g, n, m, di, da, qs, vals, d, eps, local, dist, seq_limit):
    """One accuracy point of the batched PPR benchmark: the queries batched (autotuned width)
    against one-at-a-time seeded solves of the plain engine (the first seq_limit queries, the
    time scaled to all of them when that is fewer), and the L1 error of the first four against
    the FP64 oracle on the device."""
    if a.batch_width:
        best, greedy, table = a.batch_width, a.greedy == "on", {}
    else:
        best, greedy, table = X.autotune_batch(n, m, di, da, qs, vals, eps, "ppr", d, device=local)
    log(f"eps {eps:.3g}: autotune per-query ms {table} -> B={best} greedy={greedy}")
    use_graph = not a.no_graph
    b = X.Batch(n, m, di, da, best, "ppr", d, device=local)
    b.set_greedy(greedy)
    if a.dense_groups >= 0:
        b.set_dense(a.dense_groups)
    st = torch.cuda.ExternalStream(b.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.seed(qs[:best], vals[:best], eps)   # warm-up (graph build)
    b.solve(use_graph=use_graph)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(st)
    tot_e = 0
    passes = []
    counters = {"pushed_vertices": 0, "lane_updates": 0, "rows_checked": 0, "hub_segments": 0}
    for i in range(0, len(qs), best):
        b.seed(qs[i:i + best], vals[i:i + best], eps)
        s = b.solve(use_graph=use_graph)
        tot_e += s["pushed_edges"]
        passes.append(s["passes"])
        for k in counters:
            counters[k] += s[k]
    ev1.record(st)
    torch.cuda.synchronize()
    t_batch = ev0.elapsed_time(ev1) / 1e3
    b.seed(qs[:best], vals[:best], eps)   # first batch again, for the comparison below (untimed)
    b.solve(use_graph=use_graph)
    xb = [b.read(j) for j in range(min(4, len(qs)))]
    log(f"batched: {len(qs)} queries in {t_batch:.3f}s, passes {passes}")
    # the same queries one at a time through the plain engine (seeded PageRank, full snapshot per pass)
    meas = X.measures("pr", eps_pr=eps)
    h_idx = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    g.download(h_idx, torch.empty(max(m, 1), dtype=torch.int32, pin_memory=True))
    v0, e = X.plan_chunks(h_idx.numpy().view(np.uint64), X.chunk_cap(m))
    eng = X.Engine(n, m, meas, v0, e, device=local)
    eng.upload_device(di, da)
    X.seed_engine(eng, qs[0], vals[0])
    X.resume(eng, use_graph=use_graph)
    se = torch.cuda.ExternalStream(eng.stream())
    nseq = min(len(qs), seq_limit)
    torch.cuda.synchronize()
    ev0.record(se)
    seq_e = 0
    xs = []
    for j, q in enumerate(qs[:nseq]):
        X.seed_engine(eng, q, vals[j])
        s = X.resume(eng, use_graph=use_graph)
        seq_e += s.pushed
        if j < 4:
            xs.append(eng.read(0))
    ev1.record(se)
    torch.cuda.synchronize()
    t_seq_run = ev0.elapsed_time(ev1) / 1e3
    t_seq = t_seq_run * len(qs) / nseq
    log(f"sequential: {nseq} queries in {t_seq_run:.3f}s")
    diff = [float(np.abs(xb[j].astype(np.float64) - xs[j]).sum()) for j in range(len(xs))]
    # the FP64 oracle of those queries on the device (Jacobi to 1e-10), L1 error relative to its mass
    l1b, l1s = [], []
    for j in range(len(xs)):
        ref, _ = X.ppr_fp64(n, di, da, qs[j], vals[j], d=d, tol=1e-10, device=local)
        mass = float(np.abs(ref).sum())
        l1b.append(float(np.abs(xb[j] - ref).sum()) / mass)
        l1s.append(float(np.abs(xs[j] - ref).sum()) / mass)
    if dist:
        tt = torch.tensor([t_batch, t_seq], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_batch, t_seq = float(tt[0]), float(tt[1])
    b.close()
    eng.close()
    return {"eps_times_seed_mass": eps / (1 - d), "batch_width": best, "greedy": greedy,
            "autotune_ms_per_query": {f"B{k[0]}{'_greedy' if k[1] else ''}": round(v, 4) for k, v in table.items()},
            "batched_seconds": round(t_batch, 4), "passes_per_batch": passes, "pushed_edges": int(tot_e), **counters,
            "sequential": {"seconds": round(t_seq, 3), "queries_run": nseq,
                           "timing": "measured" if nseq == len(qs) else
                                     f"{t_seq_run:.3f}s for the first {nseq} queries, scaled to {len(qs)}",
                           "pushed_edges": int(seq_e)},
            "speedup_vs_sequential": round(t_seq / t_batch, 2),
            "l1_batched_minus_sequential": diff,
            "l1_rel_vs_fp64_oracle": {"batched": l1b, "sequential": l1s, "queries": "the first 4"}}


def run_ppr(a, world, rank, local, dist):
    """256 personalized PageRank queries: batched (autotuned width) against one-at-a-time seeded solves,
    at eps 1e-4 x seed mass (the headline) and at the tighter --ppr-eps points."""
    import torch

    import excent_b200 as X
    torch.cuda.set_device(local)
    scale, ef, seed, _ = CONFIGS[a.config]
    scale = a.scale or scale
    g = X.DeviceGraph(scale, ef, seed, device=local)
    n, m = g.n, g.m
    di, da, _ = g.device_ptrs()
    d = 0.85
    nq_all = 256
    qs_all = ppr_queries(n, nq_all)
    lo, hi = X.shard(nq_all, world, rank)  # queries shard by rank, no exchange
    qs = qs_all[lo:hi]
    vals = [(1 - d) / len(q) for q in qs]
    log(f"graph scale {scale}: n={n} m={m}; {len(qs)} queries on this rank")
    points = [float(x) for x in a.ppr_eps.split(",")]
    res = [ppr_point(a, X, torch, g, n, m, di, da, qs, vals, d, p * (1 - d), local, dist,
                     256 if i == 0 else a.ppr_seq_limit) for i, p in enumerate(points)]
    head = res[0]
    g.close()
    return {
        "metric": "batched personalized PageRank solves/s (256 queries, eps %g x seed mass)" % points[0],
        "value": round(nq_all / head["batched_seconds"], 3), "unit": "solves/s", "n_gpus": world, "steps": 1,
        "warmup": 1, "ms_per_step": round(head["batched_seconds"] * 1e3, 3), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded R-MAT, generated on the device; query seeds numpy seed 7)",
        "config": {"workload": f"256-query PPR on R-MAT scale {scale} EF {ef} seed {seed}", "n": n, "m": m,
                   "queries_per_rank": len(qs)},
        "speedup_vs_sequential": head["speedup_vs_sequential"],
        "points": res,
    }


def run_adjoint(a, world, rank, local, dist):
    """Gradient of L = sum of x over 1000 random targets w.r.t. the raw edge weights and the teleport
    vector, on a weighted directed R-MAT graph; adjoint solve time against the forward solve, and the
    adjoint gradient against FP64 central differences on 64 random edges."""
    import ctypes as C

    import torch

    import excent_b200 as X
    from excent_b200._capi import call
    from excent_b200.autograd import WeightedGraph
    torch.cuda.set_device(local)
    scale, ef, seed, _ = CONFIGS[a.config]
    scale = a.scale or scale
    g = X.DeviceGraph(scale, ef, seed, symmetric=False, weights=True, device=local)
    n, m = g.n, g.m
    idx_h, adj_h, w_h = g.download()
    idx_t = torch.from_numpy(idx_h.view(np.int64)).cuda()
    adj_t = torch.from_numpy(adj_h[:m]).cuda()
    w_t = torch.from_numpy(w_h[:m]).cuda()
    G = WeightedGraph(n, idx_t, adj_t, w_t)
    rng = np.random.default_rng(seed)
    tg = torch.from_numpy(np.sort(rng.choice(n, 1000, replace=False))).cuda()
    c = torch.zeros(n, device="cuda")
    c[tg] = 1.0
    eps, d = 1e-7, 0.85
    s = C.c_void_p()
    call("excent_wgraph_stream", G.h, C.byref(s))
    st = torch.cuda.ExternalStream(s.value or 0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    G.forward("pr", d, None, eps)          # warm-up (graphs)
    G.vjp(c, eps)
    torch.cuda.synchronize()
    ev[0].record(st)
    x, fp, fe = G.forward("pr", d, None, eps)
    ev[1].record(st)
    gt, gw = G.vjp(c, eps)
    ev[2].record(st)
    torch.cuda.synchronize()
    t_f = ev[0].elapsed_time(ev[1]) / 1e3
    t_b = ev[1].elapsed_time(ev[2]) / 1e3
    log(f"forward {t_f:.3f}s ({fp} passes), adjoint {t_b:.3f}s")
    edges = rng.choice(m, 64, replace=False)
    h = 1e-3
    fd = []
    for e in edges:
        lp, lm = C.c_double(), C.c_double()
        call("excent_wgraph_loss_fp64", G.h, 0, d, None, c.data_ptr(), int(e), h, 1e-15, C.byref(lp))
        call("excent_wgraph_loss_fp64", G.h, 0, d, None, c.data_ptr(), int(e), -h, 1e-15, C.byref(lm))
        fd.append((lp.value - lm.value) / (2 * h))
    fd = np.array(fd)
    ad = gw.cpu().numpy()[edges].astype(np.float64)
    gw64 = np.zeros(m)
    gt64 = np.zeros(n)
    call("excent_wgraph_grad_fp64", G.h, 0, d, None, c.data_ptr(), 1e-15, gt64.ctypes.data, gw64.ctypes.data)
    rel_fd = float(np.linalg.norm(ad - fd) / np.linalg.norm(fd))
    rel_or_w = float(np.linalg.norm(gw.cpu().numpy().astype(np.float64) - gw64) / np.linalg.norm(gw64))
    rel_or_t = float(np.linalg.norm(gt.cpu().numpy().astype(np.float64) - gt64) / np.linalg.norm(gt64))
    G.forward("katz", 0.85, None, eps)
    gtk, _ = G.vjp(c, eps)
    gk64 = np.zeros(n)
    call("excent_wgraph_grad_fp64", G.h, 1, 0.85, None, c.data_ptr(), 1e-15, gk64.ctypes.data, None)
    rel_katz = float(np.linalg.norm(gtk.cpu().numpy().astype(np.float64) - gk64) / np.linalg.norm(gk64))
    log(f"grad vs FD rel {rel_fd:.2e}, vs FP64 oracle w {rel_or_w:.2e} t {rel_or_t:.2e} katz beta {rel_katz:.2e}")
    G.close()
    g.close()
    return {"metric": "adjoint (VJP) solve time vs the forward solve", "value": round(t_b * 1e3, 3), "unit": "ms",
            "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": round((t_f + t_b) * 1e3, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded weighted directed R-MAT, generated on the device)",
            "config": {"workload": f"adjoint of weighted PageRank on directed R-MAT scale {scale} EF {ef} seed {seed}",
                       "n": n, "m": m, "targets": 1000, "eps": eps, "forward_ms": round(t_f * 1e3, 3),
                       "forward_passes": fp, "adjoint_over_forward": round(t_b / t_f, 3)},
            "grad_rel_err_vs_fp64_central_fd_64_edges": rel_fd, "grad_w_rel_err_vs_fp64_oracle": rel_or_w,
            "grad_t_rel_err_vs_fp64_oracle": rel_or_t, "katz_beta_grad_rel_err_vs_fp64_oracle": rel_katz}


def cpu_sample(n, idx, adj, meas, measure, lam, max_edges, threads=None):
    """The oracle's CPU port of the engine, bounded to about max_edges pushed entries
    (threads: OpenMP threads, default every host core)."""
    import oracle as O
    kinds = ["pr", "katz", "ev"] if measure == "all" else [measure]
    kw = {}
    if measure == "all":
        kw = dict(alpha=float(meas.scale[1]), lam=lam, eps_katz=float(meas.eps[1]), eps_ev=float(meas.eps[2]))
    cv0 = np.ascontiguousarray(O.plan_chunks(idx, O.chunk_cap(len(adj)))[:, 0].astype(np.int32))
    t0 = time.perf_counter()
    _, _, passes, pushed = O.delta_push(n, idx, np.ascontiguousarray(adj), kinds, cv0=cv0, eps_pr=float(meas.eps[0]),
                                        max_edges=max_edges, threads=threads or os.cpu_count(), **kw)
    return pushed, passes, time.perf_counter() - t0


def cli_runs(binary, args, reps=2, log_name=None):
    """Run a CLI `reps` times; keep the run with the shortest pass time."""
    import re
    import subprocess
    best = None
    for _ in range(reps):
        r = subprocess.run([binary, *args], capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            return {"error": (r.stderr or r.stdout)[-300:]}
        out = r.stdout
        passes = int(re.search(r"^passes (\d+)", out, re.M).group(1))
        xe = float(re.search(r"edges pushed: ([0-9.]+) x", out).group(1))
        tp = float(re.search(r"time: .* passes ([0-9.]+)s", out).group(1))
        if best is None or tp < best["passes_s"]:
            best = {"passes": passes, "pushed_x_m": xe, "passes_s": tp}
            keep = out
    if log_name and LOG_DIR:
        with open(os.path.join(LOG_DIR, log_name), "w") as f:
            f.write(keep)
    return best


def cli_compare(a, idx, adj, measure, meas, lam, device):
    """The same EGR file and flags through this repo's CLI and through the reference CLI
    (src/excent.cu built from source by oracle/Makefile), both on this GPU. GTEPS =
    edges pushed / pass-loop time as each CLI prints them."""
    import shutil
    import tempfile

    import excent_b200 as X
    import excent_b200._capi as K
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "excent")
    if not os.path.exists(ref_bin):
        return {"unavailable": "reference CLI not built (oracle/Makefile)"}
    d = tempfile.mkdtemp(prefix="excent_bench_")
    try:
        path = os.path.join(d, "g.egr")
        X.write_egr(path, idx, adj)
        m = len(adj)
        args = [path, "--measure", measure, "--stream-ratio", "2", "--cache", "chunks", "--count-pushes"]
        if measure == "all":
            args += ["--alpha", "%.9g" % (0.9 / lam), "--beta", "1", "--lambda", "%.17g" % lam,
                     "--eps-katz", "1e-6", "--eps-ev", "1e-6", "--max-passes", str(a.ref_passes)]
        env_dev = {"CUDA_VISIBLE_DEVICES": os.environ.get("CUDA_VISIBLE_DEVICES", str(device))}
        os.environ.update(env_dev)
        res = {"args": " ".join(args[1:]), "file_gb": round(os.path.getsize(path) / 1e9, 3)}
        for name, binary, extra in (("reference", ref_bin, []), ("ours", K.CLI_PATH, []),
                                    ("ours_device_loop", K.CLI_PATH, ["--device-loop"])):
            r = cli_runs(binary, args + extra, log_name=f"cli_{measure}_{name}.log")
            if "passes_s" in r:
                r["gteps"] = round(r["pushed_x_m"] * m / r["passes_s"] / 1e9, 3)
            res[name] = r
            log(f"CLI {name}: {r}")
        if "gteps" in res["reference"] and "gteps" in res["ours"]:
            res["speedup_passes_time"] = round(res["reference"]["passes_s"] / res["ours"]["passes_s"], 3)
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def parse_cli(out):
    """Figures of one CLI run, from the stdout lines both CLIs print (src/excent.cu:756-804)."""
    import re
    f = {"passes": int(re.search(r"^passes (\d+)", out, re.M).group(1)),
         "pushed_x_m": float(re.search(r"edges pushed: ([0-9.]+) x", out).group(1)),
         "passes_s": float(re.search(r"time: .* passes ([0-9.]+)s", out).group(1))}
    mb = re.search(r"bytes shipped: stream ([0-9.]+) GB, gather ([0-9.]+) GB", out)
    f["stream_gb"], f["gather_gb"] = float(mb.group(1)), float(mb.group(2))
    mf = re.search(r"page faults in passes: major (\d+), minor (\d+)", out)
    f["major_faults"] = int(mf.group(1))
    f["gather_passes"] = len(re.findall(r"^pass +\d+:.*gather [1-9]", out, re.M))
    mt = re.search(r"fetch rule: tau = ([0-9.]+)", out)
    f["tau"] = float(mt.group(1)) if mt else None
    mw = re.search(r"gpu wait ([0-9.]+)s", out)
    f["gpu_wait_s"] = float(mw.group(1)) if mw else None
    mi = re.search(r"cpu io ([0-9.]+)s", out)
    f["cpu_io_s"] = float(mi.group(1)) if mi else None
    ms = re.search(r"setup ([0-9.]+)s", out)
    f["setup_s"] = float(ms.group(1)) if ms else None
    mh = re.search(r"GPU cache load ([0-9.]+)s, read ([0-9.]+)s, pinning ([0-9.-]+)s past the read", out)
    if mh:
        f["host_cache_s"] = {"gpu_cache_load": float(mh.group(1)), "read": float(mh.group(2)),
                             "pinning_past_the_read": float(mh.group(3))}
    return f


def evict(path):
    """Drop the file's pages from the host page cache (what the reference's evict_file does)."""
    fd = os.open(path, os.O_RDONLY)
    try:
        os.fsync(fd)
        os.posix_fadvise(fd, 0, 0, os.POSIX_FADV_DONTNEED)
    finally:
        os.close(fd)


def h2d_gbs(torch, nbytes=1 << 30, reps=5):
    """Pinned host -> device copy bandwidth on this box (the host-link denominator)."""
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        d.copy_(h, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    bw = nbytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9
    del h, d
    torch.cuda.empty_cache()
    return bw


def run_ooc(a, world, rank, local, dist):
    """Out-of-core PageRank (and eigenvector) through the CLI on an EGR file larger than the
    device memory left to it, page cache evicted before each run; this repo's CLI against the
    reference CLI on the same file, flags and device memory."""
    import shutil
    import subprocess
    import tempfile

    import torch

    import excent_b200 as X
    import excent_b200._capi as K
    torch.cuda.set_device(local)
    scale, ef, seed, _ = CONFIGS[a.config]
    scale = a.scale or scale
    n = 1 << scale
    est = 16 + 8 * (n + 1) + 4 * n * ef   # upper bound of the file size
    base = a.ooc_dir or tempfile.gettempdir()
    free_disk = shutil.disk_usage(base).free
    if free_disk < est * 1.05:
        return {"metric": "GTEPS (out of core)", "unavailable": f"needs {est / 1e9:.1f} GB of disk in {base}, "
                f"{free_disk / 1e9:.1f} GB free"}
    d = tempfile.mkdtemp(prefix="excent_ooc_", dir=base)
    try:
        path = os.path.join(d, f"rmat{scale}.egr")
        t0 = time.perf_counter()
        m, parts = X.rmat_write_egr(path, scale, ef, seed, device=local)
        t_gen = time.perf_counter() - t0
        log(f"wrote {path}: n={n} m={m} in {parts} partitions, {t_gen:.1f}s")
        torch.cuda.synchronize()
        link = h2d_gbs(torch)
        log(f"pinned H2D {link:.1f} GB/s")
        lam = None
        fp64 = {}
        measures = a.ooc_measures.split(",")
        if "ev" in measures or a.errors == "on":
            # lambda1 and the FP64 oracle solutions with the whole graph on the device (it fits in
            # HBM; the CLIs then run with the device memory held to the budget)
            mm = np.memmap(path, dtype=np.uint8, mode="r")
            off_idx, off_adj = 16, 16 + 8 * (n + 1)
            d_idx = torch.from_numpy(np.frombuffer(mm[off_idx:off_adj], dtype=np.int64).copy()).cuda()
            d_adj = torch.empty(m, dtype=torch.int32, device="cuda")
            step = 1 << 28
            for e0 in range(0, m, step):
                e1 = min(m, e0 + step)
                d_adj[e0:e1].copy_(torch.from_numpy(
                    np.frombuffer(mm[off_adj + 4 * e0:off_adj + 4 * e1], dtype=np.int32).copy()))
            if "ev" in measures:
                par = X.params_fp64(n, d_idx.data_ptr(), d_adj.data_ptr(), device=local)
                lam = par["lambda"]
                log(f"lambda1 {lam:.6f} after {par['sweeps']} FP64 sweeps")
            if a.errors == "on":
                fp64 = fp64_solutions(n, d_idx.data_ptr(), d_adj.data_ptr(), measures, None, local)
            del d_idx, d_adj, mm
            torch.cuda.empty_cache()
        free, total = torch.cuda.mem_get_info()
        keep = int(a.ooc_budget_gb * 1e9)
        ballast = None
        if free > keep:
            ballast = torch.empty(free - keep, dtype=torch.uint8, device="cuda")
        free2, _ = torch.cuda.mem_get_info()
        log(f"device memory left to the CLIs: {free2 / 1e9:.2f} GB")
        home = os.path.join(d, "home")
        os.makedirs(home, exist_ok=True)
        env = dict(os.environ, HOME=home)
        ref_bin = os.path.join(ROOT, "oracle", "_ref", "excent")
        runs = {}
        for measure in a.ooc_measures.split(","):
            args = [path, "--measure", measure, "--count-pushes"]
            if measure == "ev":
                args += ["--lambda", "%.17g" % lam, "--eps-ev", "1e-6", "--max-passes", str(a.ref_passes)]
            elif measure != "pr":
                return {"metric": "GTEPS (out of core)", "unavailable": f"measure {measure} is not part of this run"}
            arms = [("ours_pinned", K.CLI_PATH, ["--host-cache", "pinned", "--list-frac", str(a.list_frac),
                                                 "--hub-order", a.hub_order])]
            if a.ooc_pipeline == "on":
                arms.append(("ours", K.CLI_PATH, []))
            if a.ooc_ref == "on" and os.path.exists(ref_bin):
                arms.append(("reference", ref_bin, []))
            for name, binary, extra in arms:
                evict(path)
                dump = ["--dump", os.path.join(d, "out")] if measure in fp64 else []
                w0 = time.perf_counter()
                r = subprocess.run([binary, *args, *extra, *dump], capture_output=True, text=True, env=env,
                                   timeout=3600)
                wall = time.perf_counter() - w0
                if r.returncode != 0:
                    runs[f"{measure}/{name}"] = {"error": (r.stderr or r.stdout)[-400:]}
                    continue
                f = parse_cli(r.stdout)
                f["wall_s"] = round(wall, 2)
                b_link = (f["stream_gb"] + f["gather_gb"]) * 1e9 + f["gather_passes"] * n / 8
                f["link_bytes"] = int(b_link)
                f["link_bound_s"] = round(b_link / (link * 1e9), 3)
                f["frac_of_link_bound"] = round(f["link_bound_s"] / f["passes_s"], 4) if f["passes_s"] else None
                f["gteps"] = round(f["pushed_x_m"] * m / f["passes_s"] / 1e9, 4) if f["passes_s"] else None
                if dump:
                    out = os.path.join(d, f"out.{measure}.bin")
                    f["error_vs_fp64"] = error_vs_fp64(measure, fp64[measure], np.fromfile(out, dtype=np.float32))
                    os.remove(out)
                runs[f"{measure}/{name}"] = f
                log(f"{measure}/{name}: {f}")
                if LOG_DIR:
                    with open(os.path.join(LOG_DIR, f"ooc_{measure}_{name}.log"), "w") as fo:
                        fo.write(r.stdout)
        del ballast
        head = "ours_pinned" if a.ooc_mode == "pinned" else "ours"
        ours = runs.get(f"{a.ooc_measures.split(',')[0]}/{head}", {})
        refr = runs.get(f"{a.ooc_measures.split(',')[0]}/reference", {})
        if "passes_s" in ours and "link_bytes" in refr:
            # the link bound counted on the reference's own bytes shipped (src/excent.cu:699, :730)
            ours["link_bound_on_reference_bytes_s"] = round(refr["link_bytes"] / (link * 1e9), 3)
            ours["frac_of_reference_bytes_bound"] = round(refr["link_bytes"] / (link * 1e9) / ours["passes_s"], 4)
        if "passes_s" not in ours:
            return {"metric": "GTEPS (out of core)", "unavailable": f"CLI run failed: {ours}"}
        return {
            "metric": "GTEPS (adjacency entries pushed per second, out of core, solve to eps)",
            "value": ours["gteps"], "unit": "GTEPS", "n_gpus": world, "steps": 1, "warmup": 0,
            "ms_per_step": round(ours["passes_s"] * 1e3, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded R-MAT written as EGR on local disk)",
            "config": {"workload": f"{a.ooc_measures} out of core on R-MAT scale {scale} EF {ef} seed {seed}",
                       "lambda1": lam, "ev_max_passes": a.ref_passes if lam else None,
                       "headline_arm": head + (" (--host-cache pinned: lists read in place from pinned host memory)"
                                               if head == "ours_pinned" else " (host gather/stream pipeline)"),
                       "n": n, "m": m, "egr_gb": round(os.path.getsize(path) / 1e9, 2), "partitions": parts,
                       "device_gb_left": round(free2 / 1e9, 2), "generation_s": round(t_gen, 1),
                       "page_cache": "evicted before each CLI run", "l2_note": "inputs far larger than L2"},
            "e2e": {"value": ours["gteps"], "unit": "GTEPS", "note": "the CLI from file to dumps is the end to end path",
                    "h2d_bytes_per_step": ours["link_bytes"], "d2h_bytes_per_step": 4 * n},
            "roofline": {"bound": "host-link", "achieved": round(ours["link_bytes"] / ours["passes_s"] / 1e9, 2),
                         "peak": round(link, 2), "peak_source": "pinned H2D copy measured in this run", "unit": "GB/s",
                         "frac": ours["frac_of_link_bound"], "traffic": None},
            "runs": runs,
        }
    finally:
        shutil.rmtree(d, ignore_errors=True)


def one_core(n, idx, adj, meas, measure, lam):
    """The same port on one host core: its first pass (every vertex pending)."""
    p1, passes, t1 = cpu_sample(n, idx, adj, meas, measure, lam, max_edges=1, threads=1)
    return {"value": round(p1 / t1 / 1e9, 5), "unit": "GTEPS", "cores": 1,
            "sample": f"{passes} pass(es), {p1} entries pushed in {t1:.2f}s, one thread"}


def cpu_baseline(n, idx, adj, meas, measure, lam):
    pushed, passes, t = cpu_sample(n, idx, adj, meas, measure, lam, max_edges=len(adj))
    return {"value": round(pushed / t / 1e9, 5), "unit": "GTEPS", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first {passes} pass(es) of the same solve ({pushed} entries pushed in {t:.2f}s) by the "
                      "OpenMP CPU port of the reference engine (oracle/oracle.c)",
            "one_core": one_core(n, idx, adj, meas, measure, lam)}


def run_reference(a, world, rank):
    """CPU port of the reference engine on the host cores, bounded samples of the workload."""
    if rank != 0:
        return None
    import oracle as O
    scale, ef, seed, measure = CONFIGS[a.config]
    scale = a.scale or scale
    if measure not in ("pr", "all"):
        why = {"ppr": "the reference has no batched personalized PageRank",
               "adjoint": "the reference has no adjoint or gradient path",
               "ooc": "the CPU port does not run out of core; the out-of-core run times the reference CLI beside ours"}
        return {"impl": "reference", "unavailable": why[measure]}
    n, idx, adj = O.rmat_graph(scale, ef, seed, fast=True)
    lam = O.lambda1(n, idx, adj, 1e-10) if measure == "all" else None
    eps = [1e-2, 1e-6, 1e-6] if measure == "all" else [1e-2]

    class M:  # float32 constants as the engine rounds them
        pass
    meas = M()
    meas.eps = [float(np.float32(x)) for x in eps]
    meas.scale = [0.85, float(np.float32(0.9 / lam)) if lam else 0.0, float(np.float32(1.0 / lam)) if lam else 0.0]
    for _ in range(a.warmup):
        cpu_sample(n, idx, adj, meas, measure, lam, max_edges=len(adj) // 4)
    tot_p, tot_t = 0, 0.0
    for _ in range(a.steps):
        p, passes, t = cpu_sample(n, idx, adj, meas, measure, lam, max_edges=len(adj))
        tot_p += p
        tot_t += t
    v = tot_p / tot_t / 1e9
    return {"metric": "GTEPS (adjacency entries pushed per second, solve to eps)", "value": round(v, 5),
            "unit": "GTEPS", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(tot_t / a.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded R-MAT, oracle generator)",
            "impl": "reference",
            "config": {"workload": f"{measure} on R-MAT scale {scale} EF {ef} seed {seed}", "n": n, "m": len(adj)},
            "cpu_baseline": {"value": round(v, 5), "unit": "GTEPS", "cores": os.cpu_count(), "kind": "port",
                             "sample": "pass 0 of the solve (every vertex pending) per step; the reference has "
                                       "no CPU engine, so this is the OpenMP port in oracle/oracle.c",
                             "one_core": one_core(n, idx, adj, meas, measure, lam)},
            "e2e": {"value": round(v, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    global LOG_DIR
    a = parse()
    LOG_DIR = a.log_dir
    world, rank, local, dist = dist_setup(a.gpus)
    if a.impl == "reference":
        res = run_reference(a, world, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if res is not None:
            print(json.dumps(res))
        return
    kind = CONFIGS[a.config][3]
    runner = {"ppr": run_ppr, "adjoint": run_adjoint, "ooc": run_ooc}.get(kind, run_ours)
    res = runner(a, world, rank, local, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


def reduce_over_ranks(t, units, dist, device):
    """Job time = max over ranks; units = sum over ranks."""
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    uu = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    dist.all_reduce(uu)
    return float(tt.item()), float(uu.item())


if __name__ == "__main__":
    main()
