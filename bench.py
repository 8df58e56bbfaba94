#!/usr/bin/env python3
"""Throughput of the B200 traversal engine (GTEPS) on RMAT-24.

Workload (one "step"): on RMAT scale 24, edge factor 16, (a,b,c,d) =
(0.57,0.19,0.19,0.05), seed 2, directed, self-loops and duplicates removed,
uint32 ids, FP32 edge weights uniform in (0,1], 384 edge-balanced
destination partitions with Hilbert-ordered COO:
    BFS from vertex 100  +  PageRank (10 iterations, FP32)  +  SpMV (FP32 weights)
each run through the library's C ABI (gg_bfs / gg_pagerank / gg_spmv).

  value  = traversed edges of the step / device time of the three Compute
           loops (CUDA events on the library's stream), graph resident in HBM
  e2e    = same edges / host wall time of the K steps' C-ABI calls, including
           every step's H2D copy of the SpMV input vector from pinned memory
           (staged with gg_spmv_stage_input, so that it crosses while
           PageRank runs)
           and D2H copies of every result array of the reference's apps (BFS
           parents, PageRank ranks, SpMV y); the copies leave on the
           library's copy stream while the next application (and the next
           step) runs, and the clock stops when the last step's copies have
           arrived (--copies pipeline; --copies overlap makes every step wait
           for its own copies)
  roofline = the dense-pull kernel of the PageRank iterations: algorithmic
           bytes 8m + 16n per launch over its CUDA-event duration
  cpu_baseline = the reference's own OpenMP build (oracle/_ref, compiled from
           GraphGrind's sources) on the host cores, on the same graph written
           as Galois .gr, -c 384 -r 100 (2 rounds after 1 warm-up)
  batched  = (N=1, outside the timed step) the batched and differentiated
           forms against the plain form on the same GPU: k=64 personalised
           PageRank (RMAT-22 seed 5, 20 iterations) vs 64 single-column runs;
           64-source BFS and BC vs 64 single-source runs; 1,024 RMAT graphs
           (scales 10-16, edge factor 8-32, seeds 1000-2023, BFS from 0) in one
           persistent launch vs plain per-graph BFS on a sample; weighted
           PageRank adjoint (RMAT-22 seed 6, 30 iterations, checkpoints every 5)
           backward vs forward time
  other_apps = (N=1, outside the timed step) Components, PageRankDelta and
           BellmanFord (uint32 weights in [1,100]) on the same RMAT-24 graph
  stress   = (N=1, outside the timed step) BFS from 100 and Components on the
           4096^2 grid with 0.1 % long-range edges (seed 3, high diameter,
           sparse frontiers) and on Erdos-Renyi n=2^24, m=2^28 (seed 4, dense)

--impl reference times the same step with the reference's own build: the
graph is generated by the oracle's restatement of the library's generator (so
that process loads no library of the product), written as .gr, and each of
BFS, PageRank and SPMV runs W + K rounds through the reference's own driver
("Running : t", Compute only); a one-thread round of each is reported beside.

Multi-GPU: the path does not shard across GPUs in this build (one GPU per
graph); --gpus N runs N independent replicas under torchrun and reports the
aggregate ("scaling": "weak").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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

METRIC = "GTEPS"
UNIT = "GTEPS"
WORKLOAD = ("RMAT-24 directed (n=2^24, edge factor 16, a/b/c/d=.57/.19/.19/.05, seed 2, dedup, FP32 weights U(0,1]), "
            "P=384 edge-balanced Hilbert COO; step = BFS from 100 + PageRank 10 iterations + SpMV")


def workload(scale: int, partitions: int, start: int) -> str:
    """The workload line for the configuration actually run."""
    if (scale, partitions, start) == (24, 384, 100):
        return WORKLOAD
    return (f"RMAT-{scale} directed (n=2^{scale}, edge factor 16, a/b/c/d=.57/.19/.19/.05, seed 2, dedup, FP32 "
            f"weights U(0,1]), P={partitions} edge-balanced Hilbert COO; step = BFS from {start} + PageRank 10 "
            "iterations + SpMV")


HBM_FALLBACK_GBS = 6650.0
# DRAM bytes per PageRank-pull launch of the default workload (the merged-run
# COO kernel with the vertex step at its commits), from one ncu capture
# (profiles/dram_k_pull_coo_w_pagerank_rmat24.md)
TRAFFIC_RMAT24_PR_PULL = {(6, 1): 2110578176, (7, 1): 1982974208}  # by (COO kernel, vertex order)
TRAFFIC_TILE_EDGES = 1 << 18


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", gpu_index, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once samples are flowing
            t0 = time.time()
            while time.time() - t0 < 5 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception as e:  # no nvidia-smi: report without clocks
            log("clock sampler unavailable:", e)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, power, reasons = [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
                power.append(float(p[3]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s, w in zip(sm, power) if w > 0.3 * max(power)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "samples": len(sm),
                "power_w_max": max(power), "reasons": sorted(reasons)}


def peak_hbm():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# ------------------------------------------------------------- the workload
def make_graph(gg, scale: int, seed: int, weights: int):
    hg = gg.HostGraph.rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed, symmetric=False)
    if weights == gg.W_FLOAT32:
        hg.add_weights(gg.W_FLOAT32, seed=seed + 100)
    elif weights == gg.W_INT32:
        hg.add_weights(gg.W_INT32, seed=seed + 100, lo=1, hi=100)
    return hg


# ------------------------------------------------ the workloads' other inputs
# (the full-size parity tests import these, so that they check the results of
# exactly the inputs measured here)
def spmv_input(n: int) -> np.ndarray:
    """x of the step's SpMV: uniform [0, 1) FP32."""
    return np.random.default_rng(7).random(n, dtype=np.float32)


def ppr_seeds(n: int) -> np.ndarray:
    """The 64 one-hot teleport vertices of the k=64 personalised PageRank."""
    return np.random.default_rng(5).integers(0, n, 64).astype(np.uint32)


def multi_sources(n: int) -> np.ndarray:
    """The 64 sources of the multi-source BFS / BC."""
    return np.random.default_rng(105).integers(0, n, 64).astype(np.uint32)


def many_graph_shapes(count: int = 1024):
    """(scale, edge factor) of each graph of the many-graph BFS."""
    rng = np.random.default_rng(11)
    return rng.integers(10, 17, count), rng.integers(8, 33, count)


def adjoint_inputs(n: int, m: int):
    """Weighted PageRank adjoint: edge weights U(0,1] (normalised per source
    inside the function), teleport 1/n, loss weights N(0,1)."""
    rng = np.random.default_rng(6)
    w = rng.uniform(0, 1, m).astype(np.float32)
    w[w == 0] = 0.5
    c = rng.standard_normal(n).astype(np.float32)
    return w, np.full(n, 1.0 / n, np.float32), c


def aggregate_ranks(dist, dev_ms, wall_s, edges, launches, device="cuda"):
    """Whole-job figures of N replicas: the slowest rank's device and wall
    times (max over ranks), the edges and kernel launches of all ranks (sum)."""
    if not dist:
        return dev_ms, wall_s, float(edges), int(launches)
    import torch
    t = torch.tensor([dev_ms, wall_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([edges, launches], dtype=torch.float64, device=device)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(e[0]), int(e[1])


def run_ours(args, rank: int, world: int, local_rank: int, dist):
    import graphgrind_b200 as gg

    t0 = time.time()
    hg = make_graph(gg, args.scale, 2, gg.W_FLOAT32)
    log(f"[rank {rank}] generated RMAT-{args.scale}: n={hg.n} m={hg.m} in {time.time() - t0:.1f}s")
    t0 = time.time()
    g = gg.Graph(hg, partitions=args.partitions, tile_edges=args.tile_edges, vertex_order=args.vertex_order,
                 order=gg.ORDER_HILBERT if args.order == "hilbert" else gg.ORDER_CSR,
                 coo_tile_vertices=args.coo_tile_vertices)
    g.set_dense_policy(args.dense_policy)
    g.set_tuning(gg.TUNE_PR_GRAPH, 1 if args.pr_loop == "graph" else 0)
    info = g.info()
    log(f"[rank {rank}] device graph built in {time.time() - t0:.1f}s: {info.device_bytes / 2**30:.2f} GiB, "
        f"{info.num_coo_tiles} COO tiles, {info.num_csc_tiles} CSC tiles")
    n, m = hg.n, hg.m
    x = gg.PinnedArray(n, np.float32)
    x.array[:] = spmv_input(n)
    par = gg.PinnedArray(n, np.int32)
    ranks, y = gg.PinnedArray(n, np.float32), gg.PinnedArray(n, np.float32)

    # runtime knobs per application, chosen by the library's autotuner on this graph
    knobs = {}
    tune_s = 0.0
    if not args.no_autotune:
        t0 = time.time()
        for name, app in (("bfs", gg.APP_BFS), ("pagerank", gg.APP_PAGERANK), ("spmv", gg.APP_SPMV)):
            best = g.autotune(app, start=args.start)[0]
            knobs[name] = {k: best[k] for k in ("dense_policy", "coo_kernel", "sparse_div")}
        tune_s = time.time() - t0
        log(f"[rank {rank}] autotuned in {tune_s:.1f}s: {knobs}")

    def use(name):
        if name in knobs:
            kb = knobs[name]
            g.set_tuning(gg.TUNE_DENSE_POLICY, kb["dense_policy"])
            g.set_tuning(gg.TUNE_COO_KERNEL, kb["coo_kernel"])
            g.set_tuning(gg.TUNE_SPARSE_DIV, kb["sparse_div"])

    # results leave for the pinned host arrays on the library's copy stream
    # while the next application runs; the step ends when all have arrived
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 0 if args.copies == "wait" else 1)

    staged = args.copies != "wait" and args.spmv_input == "staged"

    def step():
        use("bfs")
        _, _, b = g.bfs(args.start, out=(par.array, None))  # app/BFS.C's result is Parents
        if staged:  # SpMV's input crosses PCIe while PageRank runs
            g.spmv_stage_input(x.array)
        use("pagerank")
        _, p = g.pagerank(10, out=ranks.array)
        use("spmv")
        if staged:
            _, s = g.spmv_staged(out=y.array)
        else:
            _, s = g.spmv(x.array, out=y.array)
        if args.copies != "pipeline":
            g.synchronize()
        return b, p, s

    for _ in range(args.warmup):
        step()
    g.synchronize()
    if dist:
        dist.barrier()
    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank] if \
        os.environ.get("CUDA_VISIBLE_DEVICES") else str(local_rank)
    clocks = ClockSampler(gpu_index)
    dev_ms, wall_s, edges, launches = 0.0, 0.0, 0, 0
    per_app = {"bfs": [0, 0.0], "pagerank": [0, 0.0], "spmv": [0, 0.0]}
    pr_prof = {"launches": 0, "ms": 0.0}
    pr_kind = None
    # pipeline: a step's result copies overlap the next step, and the wall
    # clock stops once the last step's copies have arrived
    w0 = time.perf_counter()
    for _ in range(args.steps):
        b, p, s = step()
        for name, r in (("bfs", b), ("pagerank", p), ("spmv", s)):
            per_app[name][0] += r.edges_traversed
            per_app[name][1] += r.ms
            dev_ms += r.ms
            edges += r.edges_traversed
            launches += r.kernels
    g.synchronize()
    wall_s = time.perf_counter() - w0
    # per-kernel-class profile of one more step, outside the timed region
    # (profiling records an event pair per edgeMap, so PageRank takes its host
    # loop there instead of the captured graph)
    g.set_profiling(True)
    g.profile()  # reset
    step()
    prof = g.profile()
    # PageRank-only profile for the dense-pull roofline (separate, identical calls)
    use("pagerank")
    for _ in range(2):
        g.pagerank(10, out=ranks.array)
    prof_pr = g.profile()
    # SpMV-only profile for its own roofline line
    use("spmv")
    for _ in range(2):
        g.spmv(x.array, out=y.array)
    prof_sp = g.profile()
    g.set_profiling(False)
    g.synchronize()
    clk = clocks.stop()
    for k in ("csc_pull", "coo_pull"):
        if prof_pr[k]["launches"] >= pr_prof["launches"]:
            pr_kind, pr_prof = k, prof_pr[k]
    dev_ms, wall_s, edges_all, launches_all = aggregate_ranks(dist, dev_ms, wall_s, edges, launches)
    value = edges_all / (dev_ms / 1e3) / 1e9
    e2e = edges_all / wall_s / 1e9
    peak, peak_kind = peak_hbm()
    pull_ms = pr_prof["ms"] / max(pr_prof["launches"], 1)
    # the per-warp COO kernels run PageRank's vertex step at their commits:
    # 8 B per edge (index, gathered contribution) and 24 B per vertex (offset,
    # accumulator and previous rank read; rank, reset and next contribution written)
    pr_coo_kernel = knobs["pagerank"]["coo_kernel"] if "pagerank" in knobs else g.get_tuning(gg.TUNE_COO_KERNEL)
    pr_fused = pr_kind == "coo_pull" and pr_coo_kernel > 0
    pr_bytes = 8 * m + (24 if pr_fused else 16) * n
    algo_bytes = pr_bytes
    coo_names = {0: "k_pull (CTA ring)", 1: "k_pull_coo_w", 2: "k_pull_coo_w (2-stage ring)",
                 3: "k_pull_coo_w (3-stage ring)", 4: "k_pull_coo_w (lane-contiguous)", 5: "k_pull_coo_w (prefetch)",
                 6: "k_pull_coo_w (merged runs)", 7: "k_pull_coo_w (merged runs, cache hints)"}
    kernel_name = coo_names.get(pr_coo_kernel, "k_pull_coo_w") if pr_kind == "coo_pull" else "k_pull_seg"
    if pr_fused:
        kernel_name += " with the vertex step"
    # per-application dense-pull rooflines, algorithmic bytes: PageRank as
    # above (8m+16n without the vertex step), SpMV 12m+12n, plus 4 B per
    # vertex on a renumbered graph, whose commits read the given id of
    # every destination and write its sum there
    spmv_bytes = 12 * m + (16 if args.vertex_order else 12) * n
    roofline_by_app = {}
    for app, pf, bytes_ in (("pagerank", prof_pr, pr_bytes), ("spmv", prof_sp, spmv_bytes)):
        kind = max(("coo_pull", "csc_pull"), key=lambda k: pf[k]["launches"])
        if pf[kind]["launches"]:
            lm = pf[kind]["ms"] / pf[kind]["launches"]
            ach = bytes_ / (lm / 1e3) / 1e9
            roofline_by_app[app] = {"kernel": kind, "launch_ms": round(lm, 4), "algorithmic_bytes": bytes_,
                                    "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                                    "frac": round(ach / peak, 4)}
    # BFS as a whole (device loop, pulls, result copy): 4 B per traversed edge
    # plus 12 B per reached vertex (parent and level written, offset read)
    reached = int(np.count_nonzero(par.array >= 0))
    bfs_ms = per_app["bfs"][1] / args.steps
    if bfs_ms > 0:
        bfs_bytes = 4 * (per_app["bfs"][0] // args.steps) + 12 * reached
        ach = bfs_bytes / (bfs_ms / 1e3) / 1e9
        roofline_by_app["bfs"] = {"kernel": "whole application", "ms": round(bfs_ms, 4), "reached": reached,
                                  "algorithmic_bytes": int(bfs_bytes), "achieved": round(ach, 1), "peak": peak,
                                  "unit": "GB/s", "frac": round(ach / peak, 4)}
    traffic, traffic_src = args.traffic, "--traffic" if args.traffic else None
    if traffic is None and args.scale == 24 and args.partitions == 384 and args.dense_policy == 0 and \
            args.tile_edges == TRAFFIC_TILE_EDGES and pr_kind == "coo_pull" and \
            (pr_coo_kernel, args.vertex_order) in TRAFFIC_RMAT24_PR_PULL:
        traffic = TRAFFIC_RMAT24_PR_PULL[(pr_coo_kernel, args.vertex_order)]
        traffic_src = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/dram_k_pull_coo_w_pagerank_rmat24.md"
    achieved = algo_bytes / (pull_ms / 1e3) / 1e9 if pull_ms > 0 else None
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dev_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (PageRank/SpMV), u32 (BFS ids)",
        "data": "synthetic: seeded RMAT generated on the host (no dataset)",
        "config": common_config(args, n, m),
        "parallelism": "replicas" if world > 1 else "single GPU",
        "engine": {"dense_policy": ["reference rule", "csc pull", "coo pull"][args.dense_policy],
                   "tile_edges": args.tile_edges, "coo_order": args.order,
                   "coo_tile_vertices": args.coo_tile_vertices or 4096,
                   "pagerank_loop": {"graph": "iterations replayed as one CUDA graph",
                                     "host": "one host round trip per iteration"}[args.pr_loop],
                   "result_copies": {"pipeline": "to pinned host arrays on a copy stream, overlapping the next "
                                                 "application and the next step; the timed region ends after the "
                                                 "last step's copies (gg_graph_synchronize)",
                                     "overlap": "to pinned host arrays on a copy stream, overlapping the next "
                                                "application; the step waits for all (gg_graph_synchronize)",
                                     "wait": "each call returns after its copy"}[args.copies],
                   "spmv_input": "uploaded while PageRank runs (gg_spmv_stage_input)" if staged else
                                 "uploaded by the gg_spmv call",
                   "vertex_order": ["given ids", "hottest sources first inside each partition (results in the "
                                    "given ids)"][args.vertex_order],
                   "autotuned_knobs": knobs or None, "autotune_seconds": round(tune_s, 2)},
        "apps": {k: {"edges": int(v[0]), "ms": round(v[1] / args.steps, 4),
                     "gteps": round(v[0] / (v[1] / 1e3) / 1e9, 4) if v[1] else None} for k, v in per_app.items()},
        "roofline": {"bound": "hbm", "kernel": f"{kernel_name} (PageRank dense pull)",
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": algo_bytes, "launch_ms": round(pull_ms, 4),
                     "launches": pr_prof["launches"], "traffic": traffic,
                     "traffic_source": traffic_src,
                     # the same launch counted at the pull's 8m + 16n (its
                     # vertex step's 8 B per vertex left out)
                     "frac_pull_bytes_only": round((8 * m + 16 * n) / (pull_ms / 1e3) / 1e9 / peak, 4)
                     if pull_ms > 0 else None},
        "roofline_by_app": roofline_by_app,
        "kernel_profile": {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in prof.items()},
        "e2e": {"value": round(e2e, 4), "unit": UNIT, "h2d_bytes_per_step": 4 * n + 4,
                "d2h_bytes_per_step": 12 * n},
        "gpu_launches": launches_all,
        "clocks": clk,
    }
    if world == 1 and not args.no_stress:
        out["other_apps"] = run_other_apps(gg, hg, g, args)
    if world == 1 and not args.no_cpu_baseline:
        g.close()
        per_step = {"BFS": per_app["bfs"][0] // args.steps, "PR": per_app["pagerank"][0] // args.steps,
                    "SPMV": per_app["spmv"][0] // args.steps}
        out["cpu_baseline"] = cpu_baseline_for_ours(args, hg, per_step)
    return out


def run_other_apps(gg, hg, g, args):
    """The rest of the RMAT-24 application list (Components, PageRankDelta with
    eps 1e-7, BellmanFord from the start vertex on uint32 weights in [1,100]),
    outside the timed step, each the best of 3 device times; unless
    --no-autotune, each with the runtime knobs the library's autotuner picks
    for it on its graph (recorded under "knobs")."""
    out = {}

    def tuned(graph, app):
        if args.no_autotune:
            return None
        best = graph.autotune(app, start=args.start)[0]
        kb = {k: best[k] for k in ("dense_policy", "coo_kernel", "sparse_div")}
        graph.set_tuning(gg.TUNE_DENSE_POLICY, kb["dense_policy"])
        graph.set_tuning(gg.TUNE_COO_KERNEL, kb["coo_kernel"])
        graph.set_tuning(gg.TUNE_SPARSE_DIV, kb["sparse_div"])
        return kb

    def measure(name, fn, kb):
        fn()
        runs = [fn() for _ in range(3)]
        r = min(runs, key=lambda x: x.ms)
        out[name] = {"ms": round(r.ms, 3), "rounds": r.rounds, "gteps": round(r.edges_traversed / r.ms / 1e6, 2)}
        if kb is not None:
            out[name]["knobs"] = kb

    for name, app, fn in (("components", gg.APP_COMPONENTS, lambda: g.components()[1]),
                          ("pagerank_delta", gg.APP_PAGERANK_DELTA, lambda: g.pagerank_delta()[1])):
        measure(name, fn, tuned(g, app))
    hw = make_graph(gg, args.scale, 2, gg.W_INT32)
    gw = gg.Graph(hw, partitions=args.partitions, tile_edges=args.tile_edges, vertex_order=args.vertex_order,
                  order=gg.ORDER_HILBERT if args.order == "hilbert" else gg.ORDER_CSR,
                  coo_tile_vertices=args.coo_tile_vertices)
    measure("bellman_ford", lambda: gw.bellman_ford(args.start)[1], tuned(gw, gg.APP_BELLMAN_FORD))
    gw.close()
    return out


# ------------------------------------------------ batched and adjoint forms
def _best(f, reps):
    return min(f() for _ in range(reps))


def run_batched(gg):
    """Batched / differentiated forms vs the plain form, each on its own graph."""
    out = {}
    rng = np.random.default_rng(11)
    t0 = time.time()
    hg = gg.HostGraph.rmat(22, 16, 0.57, 0.19, 0.19, seed=5, symmetric=False)
    g = gg.Graph(hg, partitions=96)
    m = hg.m
    seeds = ppr_seeds(hg.n)
    o64 = np.empty((hg.n, 64), np.float32)
    o1 = np.empty((hg.n, 1), np.float32)
    g.ppr_k(64, 20, 0.85, seeds=seeds, out=o64)
    k64 = _best(lambda: g.ppr_k(64, 20, 0.85, seeds=seeds, out=o64)[1].ms, 3)
    plain, diffs = 0.0, []
    g.ppr_k(1, 20, 0.85, seeds=seeds[:1], out=o1)
    for j in range(64):
        plain += g.ppr_k(1, 20, 0.85, seeds=seeds[j:j + 1], out=o1)[1].ms
        if j < 4:
            diffs.append(float(np.abs(o64[:, j] - o1[:, 0]).sum() / np.abs(o1[:, 0]).sum()))
    out["ppr_k64"] = {"workload": f"RMAT-22 seed 5 directed (m={m}), 64 one-hot teleports, 20 iterations",
                      "batched_ms": round(k64, 3), "batched_gteps": round(64 * 20 * m / k64 / 1e6, 2),
                      "plain_64x_ms": round(plain, 3), "plain_gteps": round(64 * 20 * m / plain / 1e6, 2),
                      "speedup": round(plain / k64, 2), "max_rel_l1_vs_plain_cols0_3": max(diffs)}
    src = multi_sources(hg.n)
    lev = np.empty((hg.n, 64), np.int32)
    g.msbfs(src, out=lev)
    r = g.msbfs(src, out=lev)[1]
    ms_bfs = _best(lambda: g.msbfs(src, out=lev)[1].ms, 3)
    g.bfs(int(src[0]))  # warm-up (the first BFS of a graph builds its bottom-up in-lists)
    plain = sum(g.bfs(int(s))[2].ms for s in src)
    out["msbfs_k64"] = {"workload": "RMAT-22 seed 5 directed, 64 uniform sources", "batched_ms": round(ms_bfs, 3),
                        "batched_gteps": round(r.edges_traversed / ms_bfs / 1e6, 2), "plain_64x_ms": round(plain, 3),
                        "speedup": round(plain / ms_bfs, 2)}
    dep, npth = np.empty((hg.n, 64), np.float32), np.empty((hg.n, 64), np.float32)
    rb = g.msbc(src, dep_out=dep, paths_out=npth)[2]
    ms_bc = _best(lambda: g.msbc(src, dep_out=dep, paths_out=npth)[2].ms, 2)
    plain = sum(g.bc(int(s))[2].ms for s in src)
    out["msbc_k64"] = {"workload": "RMAT-22 seed 5 directed, 64 uniform sources", "batched_ms": round(ms_bc, 3),
                       "batched_gteps": round(rb.edges_traversed / ms_bc / 1e6, 2), "plain_64x_ms": round(plain, 3),
                       "speedup": round(plain / ms_bc, 2)}
    g.close()
    # 1,024 independent graphs in one persistent launch
    count = 1024
    scales, efs = many_graph_shapes(count)
    hgs = [gg.HostGraph.rmat(int(sc), int(ef), 0.57, 0.19, 0.19, seed=1000 + i, symmetric=False)
           for i, (sc, ef) in enumerate(zip(scales, efs))]
    b = gg.GraphBatch(hgs)
    zeros = np.zeros(count, np.uint32)
    levs = np.empty(b.total_vertices, np.int32)
    rr = b.bfs(zeros, out=levs)[1]
    many = _best(lambda: b.bfs(zeros, out=levs)[1].ms, 5)
    sample = rng.choice(count, 32, replace=False)
    p_ms, p_edges = 0.0, 0
    for i in sample:
        gi = gg.Graph(hgs[i], partitions=1)
        gi.bfs(0)
        r1 = gi.bfs(0)[2]
        p_ms += r1.ms
        p_edges += r1.edges_traversed
        gi.close()
    b.close()
    plain_gteps = p_edges / p_ms / 1e6
    out["many_graphs_bfs"] = {
        "workload": f"{count} RMAT graphs, scales U{{10..16}}, edge factor U{{8..32}}, seeds 1000-{999 + count}, "
                    f"directed, BFS from 0; {b.total_vertices} vertices, {b.total_edges} edges",
        "batched_ms": round(many, 3), "batched_gteps": round(rr.edges_traversed / many / 1e6, 2),
        "includes": "source upload, persistent traversal, level download (one CUDA-graph replay)",
        "plain_gteps_sample32": round(plain_gteps, 3),
        "speedup_vs_plain_gteps": round(rr.edges_traversed / many / 1e6 / plain_gteps, 2)}
    # weighted PageRank adjoint
    hw = gg.HostGraph.rmat(22, 16, 0.57, 0.19, 0.19, seed=6, symmetric=False)
    gw = gg.Graph(hw, partitions=96)
    w, tele, c = adjoint_inputs(hw.n, hw.m)
    wpr = gg.WeightedPageRank(gw, 30, 0.85, 5, True)
    wpr.forward(w, tele)
    wpr.backward(c)
    fwd = _best(lambda: wpr.forward(w, tele)[1].ms, 3)
    bwd = _best(lambda: wpr.backward(c)[3].ms, 3)
    wpr.close()
    gw.close()
    out["adjoint_weighted_pagerank"] = {
        "workload": f"RMAT-22 seed 6 directed (m={hw.m}), weights U(0,1] normalised per source inside the function, "
                    "damping 0.85, 30 iterations, loss weights N(0,1), checkpoints every 5",
        "forward_ms": round(fwd, 3), "backward_ms": round(bwd, 3), "backward_over_forward": round(bwd / fwd, 3),
        "forward_gteps": round(30 * hw.m / fwd / 1e6, 2)}
    out["seconds"] = round(time.time() - t0, 1)
    return out


def _accepted_partitions(gg, hg, preferred):
    """The largest P <= preferred that the reference partitioner accepts."""
    outd = hg.degrees()
    ind = outd if hg.symmetric else hg.transpose().degrees()
    for P in range(preferred, 0, -1):
        try:
            gg.partition_sizes(ind, outd, hg.m, P)
            return P
        except gg.GGError:
            continue
    return 1


def run_stress(gg):
    """Sparse-frontier / high-diameter stress against the dense-pull case: BFS
    and Components on the 4096^2 grid with 0.1 % long-range edges (seed 3) and
    on Erdos-Renyi n = 2^24, m = 2^28 (seed 4, directed)."""
    out = {}
    t0 = time.time()
    for name, make in (("grid4096", lambda: gg.HostGraph.grid(4096, 0.001, seed=3)),
                       ("er24", lambda: gg.HostGraph.er(1 << 24, 1 << 28, seed=4, symmetric=False))):
        hg = make()
        P = _accepted_partitions(gg, hg, 384)
        g = gg.Graph(hg, partitions=P, tile_edges=1 << 17)
        par = np.empty(hg.n, np.int32)
        ids = np.empty(hg.n, np.int32)
        g.bfs(100, out=(par, None))
        rb = g.bfs(100, out=(par, None))[2]
        bfs_ms = _best(lambda: g.bfs(100, out=(par, None))[2].ms, 3)
        g.components()
        rc = g.components()[1]
        cc_ms = _best(lambda: g.components()[1].ms, 2)
        out[name] = {"n": hg.n, "m": hg.m, "partitions": P,
                     "bfs": {"ms": round(bfs_ms, 3), "levels": rb.rounds,
                             "gteps": round(rb.edges_traversed / bfs_ms / 1e6, 2)},
                     "components": {"algorithm": "label propagation (app/Components.C)", "ms": round(cc_ms, 3),
                                    "rounds": rc.rounds, "gteps": round(rc.edges_traversed / cc_ms / 1e6, 2)}}
        if hg.symmetric:  # the same labels by union-find (GG_TUNE_CC_ALGO 1)
            g.set_tuning(gg.TUNE_CC_ALGO, 1)
            g.components()
            uf_ms = _best(lambda: g.components()[1].ms, 3)
            g.set_tuning(gg.TUNE_CC_ALGO, 0)
            out[name]["components_union_find"] = {"ms": round(uf_ms, 3),
                                                  "speedup_vs_label_propagation": round(cc_ms / uf_ms, 1)}
        g.close()
        del hg
    out["seconds"] = round(time.time() - t0, 1)
    return out


# ------------------------------------------------------- the reference (CPU)
REF_APPS = ("BFS", "PR", "SPMV")
REF_SPMV_WEIGHTS = ("SpMV reads uint32 weights U[1,100] (hash seed 102) where the GPU reads FP32 U(0,1]: the "
                    "reference takes integer weights only (graphgrind/graph-numa.h:78-89)")


def common_config(args, n: int, m: int) -> dict:
    """The workload block both arms print: same graph, partitions and step."""
    return {"workload": workload(args.scale, args.partitions, args.start), "n": n, "m": m,
            "partitions": args.partitions, "start": args.start, "pagerank_iterations": 10,
            "l2": "inputs larger than L2 (graph arrays > 3 GB vs 126 MB L2)"}


def reference_inputs(workdir: str, scale: int, start: int):
    """The step's graph and its edge counts from the oracle alone (no library
    of the product is loaded): R-MAT `scale`, seed 2, directed, written as
    Galois .gr (+ _t) unweighted for BFS/PageRank and with uint32 weights for
    SpMV; traversed edges per application as the library counts them
    (graphgrind/ligra-numa.h:944-945)."""
    import oracle

    r = oracle.RmatGraph(scale, 16, 0.57, 0.19, 0.19, seed=2, symmetric=False)
    pu, pw = os.path.join(workdir, "g.gr"), os.path.join(workdir, "gw.gr")
    r.write_gr(pu)
    og = oracle.Graph(r.offsets, r.indices)
    _, _, bst = og.bfs(start)
    pr_edges, _ = og.pagerank_edges(10)
    del og
    r.add_weights(False, seed=102, lo=1, hi=100)
    r.write_gr(pw)
    return r.n, r.m, {"BFS": bst.edges_traversed, "PR": pr_edges, "SPMV": r.m}, {"BFS": pu, "PR": pu, "SPMV": pw}


def time_reference(paths: dict, partitions: int, start: int, rounds: int, threads=None) -> dict:
    """The reference's own driver (parallel_main, graphgrind/ligra-numa.h:1095)
    on each file: its 'Running : t' seconds per round (Compute only, graph
    load and partition build excluded, :1150-1161)."""
    import oracle

    for app in REF_APPS:
        if not oracle.ref_available(app):
            raise RuntimeError(f"reference binary {oracle.ref_binary(app)} not built")
    flags = ["-b", "-c", str(partitions), "-r", str(start)]
    return {app: oracle.time_ref(app, paths[app], flags, rounds=rounds, threads=threads, timeout=1800)
            for app in REF_APPS}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def _per_round(edges: dict, times: dict, first: int):
    secs = [sum(times[a][r] for a in REF_APPS) for r in range(first, len(times[REF_APPS[0]]))]
    return secs, sum(edges.values()) * len(secs) / sum(secs) / 1e9


def run_reference_arm(args):
    """bench.py --impl reference: GraphGrind's own OpenMP build (oracle/_ref,
    compiled from the reference's sources) on this host's cores, on the same
    graph file, partitions and step as the GPU arm; W warm-up rounds, then K
    timed rounds of each application.  This process loads only the oracle."""
    cores = os.cpu_count() or 1
    try:
        with tempfile.TemporaryDirectory() as d:
            n, m, edges, paths = reference_inputs(d, args.scale, args.start)
            times = time_reference(paths, args.partitions, args.start, args.warmup + args.steps)
            one = None
            if not args.no_one_thread:
                t1 = time_reference(paths, args.partitions, args.start, 1, threads=1)
                one = {"value": round(_per_round(edges, t1, 0)[1], 4), "unit": UNIT, "cores": 1,
                       "sample": "one round of each application, OMP_NUM_THREADS=1",
                       "seconds": {a: round(t1[a][0], 4) for a in REF_APPS}}
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference build/run failed: {e}"[:300]}))
        return
    secs, value = _per_round(edges, times, args.warmup)
    sample = (f"the GPU arm's graph (R-MAT-{args.scale} seed 2, directed) as Galois .gr, -b -c {args.partitions} "
              f"-r {args.start}; {args.steps} timed rounds after {args.warmup} warm-up; {REF_SPMV_WEIGHTS}")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(secs) / len(secs), 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 (PageRank/SpMV), int64 (BFS ids)", "data": "synthetic: seeded RMAT (no dataset)",
           "config": common_config(args, n, m), "parallelism": f"host cores (OpenMP, {cores} threads)",
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                            "cpu": cpu_model(), "sample": sample},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "one_thread": one,
           "reference_detail": {"edges_per_step": sum(edges.values()), "edges": edges,
                                "seconds_per_round": {a: [round(t, 5) for t in times[a]] for a in REF_APPS}}}
    print(json.dumps(out))


def cpu_baseline_for_ours(args, hg, edges: dict):
    """The reference's own build on the GPU arm's graph (written from the same
    host CSR), 3 rounds of each application, the first dropped."""
    import graphgrind_b200 as gg

    cores = os.cpu_count() or 1
    sample = (f"the same graph as Galois .gr, reference OpenMP build, -b -c {args.partitions} -r {args.start}; "
              f"mean of 2 rounds after 1 warm-up; {REF_SPMV_WEIGHTS}")
    try:
        with tempfile.TemporaryDirectory() as d:
            pu, pw = os.path.join(d, "g.gr"), os.path.join(d, "gw.gr")
            gu = gg.HostGraph.from_csr(hg.offsets, hg.indices, None, symmetric=False)
            gu.write_gr(pu)
            gu.add_weights(gg.W_INT32, seed=102, lo=1, hi=100)
            gu.write_gr(pw)
            del gu
            times = time_reference({"BFS": pu, "PR": pu, "SPMV": pw}, args.partitions, args.start, 3)
        _, value = _per_round(edges, times, 1)
        return {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "reference", "cpu": cpu_model(),
                "sample": sample}
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample,
                "error": str(e)[:200]}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--partitions", type=int, default=384)
    ap.add_argument("--start", type=int, default=100)
    ap.add_argument("--dense-policy", type=int, default=0, help="0 reference rule, 1 CSC pull, 2 COO pull")
    ap.add_argument("--no-one-thread", action="store_true",
                    help="reference arm: skip the one-thread round of each application")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched / adjoint comparisons")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default runtime knobs")
    ap.add_argument("--no-stress", action="store_true",
                    help="skip the other RMAT-24 apps and the grid / Erdos-Renyi BFS and Components lines")
    ap.add_argument("--coo-tile-vertices", type=int, default=0,
                    help="max destinations per COO tile (0: 4096, the CSC tile width)")
    ap.add_argument("--order", choices=["hilbert", "csr"], default="hilbert",
                    help="COO order inside partitions: Hilbert (EDGES_HILBERT=1) or source-major (CSRDestSort)")
    ap.add_argument("--vertex-order", type=int, default=1, choices=[0, 1],
                    help="device numbering: 0 the given ids, 1 hottest sources first inside each partition")
    ap.add_argument("--tile-edges", type=int, default=1 << 18,
                    help="target edges per CTA tile (gg_autotune_build's choice for this workload)")
    ap.add_argument("--copies", choices=["pipeline", "overlap", "wait"], default="pipeline",
                    help="result copies to the host overlap the next application and the next step, the clock "
                         "stopping after the last step's copies (pipeline); overlap the next application, each "
                         "step waiting for its copies (overlap) (both GG_TUNE_ASYNC_RESULTS 1); or finish inside "
                         "each call (wait)")
    ap.add_argument("--spmv-input", choices=["staged", "call"], default="staged",
                    help="SpMV's input uploaded while PageRank runs (gg_spmv_stage_input + gg_spmv_staged) or "
                         "by the gg_spmv call itself")
    ap.add_argument("--pr-loop", choices=["graph", "host"], default="graph",
                    help="PageRank iterations as one CUDA graph (GG_TUNE_PR_GRAPH 1) or host-driven")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per dense-pull launch from an ncu capture (reported as roofline.traffic)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    out = run_ours(args, rank, world, local_rank, dist)
    if rank == 0:
        if world == 1 and not args.no_batched:
            import graphgrind_b200 as gg
            try:
                out["batched"] = run_batched(gg)
            except Exception as e:  # reported, the headline line still prints
                out["batched"] = {"error": str(e)[:300]}
        if world == 1 and not args.no_stress:
            import graphgrind_b200 as gg
            try:
                out["stress"] = run_stress(gg)
            except Exception as e:
                out["stress"] = {"error": str(e)[:300]}
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
