#!/usr/bin/env python
"""Benchmark of the tribit_b200 exact triangle counter on B200.

Metric (edges/s = m / count time): the exact count of an RMAT scale-24 graph
(edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05, seeded, duplicates and
self-loops removed, ~16.7M vertices, ~250M undirected edges), with synthetic
data of that shape generated on the host. A step is one launch of the counting
kernels over the prepared (oriented, bit-packed) graph already resident in
HBM; preprocessing is timed separately, as the reference reports it. `e2e` is
the same metric through the public C-ABI call tribit_count_edges on pinned
host entries: H2D copy, preprocessing, counting and the D2H result inside,
the mean wall time of --e2e-steps calls (5; each call's time in step_ms;
Python's garbage collector run before the calls and held off during them).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload rmat24|rmat22|rmat20|chung_lu|planted]
                  [--dispatch auto|plain|learned|bitmap|merge|mma] [--no-batch]

config.batch reports the batched workload: 4,096 graphs (n log-uniform in
[64, 65536], Erdos-Renyi or Chung-Lu by seed) counted by one persistent
launch replayed from a CUDA graph (graphs/s), against one count per graph.

Multi-GPU: the counter has no cross-GPU exchange, so N GPUs run N independent
replicas (seed + rank), one process each under torchrun; value is the sum of
edges over the max-over-ranks time ("scaling": "weak").

--impl reference times the reference's algorithm on the host cores: the
reference has no CPU implementation, so this is the CPU merge-intersection
oracle (a port), timed on a strided sample of 32-row blocks and extrapolated.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges/s (m / count time) on RMAT-24, learned vs plain dispatch, exact; graphs/s"

WORKLOADS = {
    "rmat24": {"gen": "rmat", "scale": 24, "edge_factor": 16, "seed": 24},
    "rmat22": {"gen": "rmat", "scale": 22, "edge_factor": 16, "seed": 22},
    "rmat20": {"gen": "rmat", "scale": 20, "edge_factor": 16, "seed": 20},
    "chung_lu": {"gen": "chung_lu", "n": 7115, "n_entries": 115300, "beta": 2.0, "max_degree": 1000.0, "seed": 1},
    "planted": {"gen": "planted", "communities": 20000, "size": 100, "p_in": 0.3, "inter": 2, "seed": 3},
    # Dense-tile stress: disjoint cliques on consecutive ids; every vertex has
    # the same degree, so the degree order keeps each clique contiguous and
    # every row block fits one bit tile.
    "cliques": {"gen": "cliques", "count": 512, "size": 512, "seed": 0},
}


def make_graph(tb, spec, rank):
    s = dict(spec)
    seed = s["seed"] + 1000 * rank
    if s["gen"] == "rmat":
        return 1 << s["scale"], tb.gen_rmat(s["scale"], s["edge_factor"], 0.57, 0.19, 0.19, seed)
    if s["gen"] == "chung_lu":
        return s["n"], tb.gen_chung_lu(s["n"], s["n_entries"], s["beta"], s["max_degree"], seed)
    if s["gen"] == "planted":
        return s["communities"] * s["size"], tb.gen_planted(s["communities"], s["size"], s["p_in"], s["inter"], seed)
    if s["gen"] == "cliques":
        import numpy as np
        k, c = s["size"], s["count"]
        i, j = np.triu_indices(k, 1)
        base = (np.arange(c, dtype=np.uint64) * np.uint64(k))[:, None]
        lo = (base + i.astype(np.uint64)[None, :]).ravel()
        hi = (base + j.astype(np.uint64)[None, :]).ravel()
        return c * k, (lo << np.uint64(32)) | hi
    raise ValueError(s["gen"])


def reduce_replicas(dist, edges, seconds, device):
    """Replicas only (no data-path collective): each rank counts its own graph.
    Returns (edges summed over ranks, time maxed over ranks); with dist None,
    this rank's own. The two reductions are the only collectives of the bench."""
    if dist is None:
        return edges, seconds
    import torch
    e = torch.tensor([edges], device=device, dtype=torch.float64)
    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return int(e.item()), float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profiled_traffic(workload, dispatch):
    """Per-launch DRAM bytes of the counting kernels from the committed ncu summary
    (lines: workload, bytes, dispatch)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == workload and parts[2] == dispatch:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class gc_held:
    """Python's garbage collector run once before a timed loop and held off
    during it: the library calls allocate almost no Python objects, so a
    collection inside one would time the interpreter's heap, not the call."""

    def __enter__(self):
        gc.collect()
        gc.disable()
        return self

    def __exit__(self, *exc):
        gc.enable()


def wall_call(fn):
    """(fn(), its wall time in s)."""
    t0 = time.perf_counter()
    out = fn()
    return out, time.perf_counter() - t0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"tribit_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(entries, n, m, target_s=15.0, steps=1):
    """Oracle merge-intersection count on a strided sample of 32-row blocks of
    the degree-ordered CSR, on all host threads; returns per-step results."""
    import oracle
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    g = oracle.CSR(entries, n, order=1)
    stride = 1024
    # Grow the sample until one step costs about target_s of CPU wall time.
    _, s = g.count_sample(threads, stride, 0)
    while s < target_s / 8 and stride > 1:
        stride //= 4 if s < target_s / 64 else 2
        stride = max(stride, 1)
        _, s = g.count_sample(threads, stride, 0)
    out = []
    for k in range(steps):
        t, s = g.count_sample(threads, stride, k % stride)
        full_s = s * stride
        out.append({"value": m / full_s, "seconds": s, "stride": stride, "offset": k % stride, "sample_triangles": t})
    work = g.work()
    g.close()
    return out, threads, work


def batch_measurement(tb, np, torch, local, dispatch, model_path, num_graphs=4096, seed=4096, steps=5,
                      per_graph_sample=256):
    """The batched workload: num_graphs graphs (n log-uniform in [64, 65536],
    Erdos-Renyi or Chung-Lu by seed) counted in one persistent launch replayed
    from a CUDA graph, against counting graphs one at a time."""
    e, off, nn = tb.gen_batch(num_graphs, seed=seed)
    pinned = torch.empty(e.size, dtype=torch.int64, pin_memory=True)
    pinned.numpy()[:] = e.view(np.int64)
    host = pinned.numpy().view(np.uint64)
    c = tb.Counter(device=local, dispatch=dispatch)
    if dispatch == "learned":
        c.load_model(model_path)
    counts, r = c.count_batch(host, off, nn)  # sizes the arena, prepares the batch
    with gc_held():
        (counts, r), e2e_s = wall_call(lambda: c.count_batch(host, off, nn))
    tune = c.autotune(reps=2)
    c.capture_count()
    s = torch.cuda.Stream(device=local)
    c.set_stream(s.cuda_stream)

    def replay_ms():
        out = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            c.launch_count()
            b.record(s)
            b.synchronize()
            out.append(a.elapsed_time(b))
        assert np.array_equal(c.batch_counts(num_graphs), counts), "graph replay changed the per-graph counts"
        return statistics.median(out)

    ms = replay_ms()
    # The other launch model at the same tuning: the row pieces and hub pass
    # in one persistent kernel over the device work queue, or one per variant.
    tuned_model = tb.LAUNCH_MODELS[tune.launch_model]
    other = "queue" if tuned_model == "kernels" else "kernels"
    c.set_tuning(tune.ctas_per_sm, tune.piece_width, tune.tile_min_nnz, launch_model=other)
    c.capture_count()
    by_model = {tuned_model: ms, other: replay_ms()}
    c.close()
    # One graph at a time (a strided sample), same library, same stream model.
    d = torch.from_numpy(e.view(np.int64)).to(f"cuda:{local}")
    c1 = tb.Counter(device=local, dispatch=dispatch)
    if dispatch == "learned":
        c1.load_model(model_path)
    # The batch's tuned settings, each graph's launch model chosen by its size
    # (small graphs: the queue kernel).
    c1.set_tuning(tune.ctas_per_sm, tune.piece_width, tune.tile_min_nnz, launch_model="auto")
    idx = np.linspace(0, num_graphs - 1, per_graph_sample).astype(int)
    k_ms, e2e_one = 0.0, 0.0
    with gc_held():
        for g in idx:
            lo, hi = int(off[g]), int(off[g + 1])
            c1.count_edges_device(d[lo:].data_ptr(), hi - lo, int(nn[g]))  # sizes the arena
            rg, dt = wall_call(lambda: c1.count_edges_device(d[lo:].data_ptr(), hi - lo, int(nn[g])))
            e2e_one += dt
            k_ms += rg.kernel_ms
            assert rg.triangles == int(counts[g]), f"graph {g}: batch {counts[g]} vs single {rg.triangles}"
    c1.close()
    scale = num_graphs / per_graph_sample
    batched_ms = ms
    return {
        "graphs": num_graphs, "entries": int(e.size), "edges": int(r.edges), "triangles": int(counts.sum()),
        "batched_count_ms": batched_ms, "graphs_per_s_batched": num_graphs / (batched_ms / 1e3),
        "graphs_per_s_per_graph_launches": num_graphs / (k_ms * scale / 1e3),
        "e2e_graphs_per_s_batched": num_graphs / e2e_s,
        "e2e_graphs_per_s_per_graph": num_graphs / (e2e_one * scale),
        "per_graph_sample": per_graph_sample, "tuning": tune.as_dict(), "cuda_graph": True,
        "batched_count_ms_by_launch_model": by_model,
        "row_blocks_by_variant": dict(zip(tb.VARIANTS, r.row_blocks_by_variant)),
    }


REF_FIELDS = {
    "blocks_of_threads": r"Blocks of threads\s*:\s*(\d+)",
    "preprocessing_ms": r"Preprocessing \(ms\)\s*:\s*([\d.]+)",
    "kernel_ms": r"Kernel \(ms\)\s*:\s*([\d.]+)",
    "triangles": r"Triangles\s*:\s*(\d+)",
}


def reference_graph(spec):
    """The workload's graph for the reference arm: R-MAT from the oracle's own
    generator (word for word the product's), so this arm never loads the
    product library; the other workloads come from the product's generators."""
    if spec["gen"] == "rmat":
        import oracle
        return 1 << spec["scale"], oracle.gen_rmat(spec["scale"], spec["edge_factor"], 0.57, 0.19, 0.19, spec["seed"])
    import tribit_b200 as tb
    return make_graph(tb, spec, 0)


def reference_binary(name, timeout=900):
    """The reference's own GPU counter (sixt99/TriBIT src/single_gpu/tribit.cu,
    built unchanged for sm_100a into oracle/_ref/tribit_ref) on the workload
    `name` written as a Matrix Market file: its printed summary, parsed with
    the regexes of its harness (artifact/sc26/run_benchmarks/run_single_gpu.py:78-83)."""
    import re
    import oracle
    exe = os.path.join(ROOT, "oracle", "_ref", "tribit_ref")
    if not os.path.exists(exe):
        return {"workload": name, "unavailable": "oracle/_ref/tribit_ref is not built"}
    n, e = reference_graph(WORKLOADS[name])
    edges = int(len(oracle.fold_dedup(e.copy())))
    path = os.path.join("/tmp", f"tribit_ref_{os.getpid()}_{name}.mtx")
    rec = {"workload": name, "edges": edges}
    try:
        oracle.write_mtx(path, n, e)
        t0 = time.time()
        r = subprocess.run([exe, "-i", path], capture_output=True, text=True, timeout=timeout)
        rec["wall_s"] = round(time.time() - t0, 1)
        rec["status"] = "ok" if r.returncode == 0 else f"exit {r.returncode}"
        for k, rx in REF_FIELDS.items():
            mt = re.search(rx, r.stdout)
            if mt:
                rec[k] = float(mt.group(1)) if k.endswith("_ms") else int(mt.group(1))
        if r.returncode != 0:
            rec["stderr_tail"] = r.stderr.strip().splitlines()[-2:]
        if rec.get("kernel_ms"):
            rec["edges_per_s"] = edges / (rec["kernel_ms"] / 1e3)
    except subprocess.TimeoutExpired:
        rec["status"] = f"timeout after {timeout} s"
    finally:
        if os.path.exists(path):
            os.remove(path)
    return rec


def run_reference(args, spec, rank, world):
    if rank != 0:
        return
    import oracle
    n, e = reference_graph(spec)
    edges = int(len(oracle.fold_dedup(e.copy())))
    steps, threads, _ = cpu_baseline(e, n, edges, steps=args.warmup + args.steps)
    timed = steps[args.warmup:]
    value = statistics.mean(x["value"] for x in timed)
    per_step_s = edges / value
    line = {
        "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, **spec, "n": n, "entries": int(len(e)), "edges": edges},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": threads, "kind": "port",
                         "sample": f"32-row blocks b % {timed[0]['stride']} == offset (offset per step), "
                                   f"~{timed[0]['seconds']:.1f} s each, time x stride"},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.ref_binary != "none":
        # The reference GPU binary cannot count the headline graph (RMAT-24: its
        # grid exceeds INT_MAX CTAs, tribit.cu:772-773); its Kernel (ms) on the
        # largest workload it runs is recorded beside the CPU port.
        line["reference_gpu_binary"] = reference_binary(args.ref_binary)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat24", choices=sorted(WORKLOADS))
    ap.add_argument("--dispatch", default="auto")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 4,096-graph batch measurement")
    ap.add_argument("--stream-budgets", default="0.5,0.3",
                    help="device budgets (fractions of the one-piece need, each optionally ':rows' or ':pairs' "
                         "to force a tier) for the out-of-HBM end-to-end measurement; empty to skip")
    ap.add_argument("--stream-pageable", action="store_true",
                    help="the out-of-HBM measurement reads pageable host entries instead of pinned ones")
    ap.add_argument("--tile-engine", default="tcgen05", choices=["mma_sync", "tcgen05"],
                    help="arithmetic of the bit-tile variant")
    ap.add_argument("--ref-binary", default="rmat22", choices=["none"] + sorted(WORKLOADS),
                    help="--impl reference: also run the reference GPU binary on this workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    spec = WORKLOADS[args.workload]

    if args.impl == "reference":
        run_reference(args, spec, rank, world)
        return

    import numpy as np
    import torch
    import tribit_b200 as tb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    t0 = time.time()
    n, entries = make_graph(tb, spec, rank)
    gen_s = time.time() - t0

    dispatch = args.dispatch
    model_path = os.path.join(ROOT, "tribit_b200", "models", "dispatch_mlp.bin")
    if dispatch == "auto":
        dispatch = "learned" if os.path.exists(model_path) else "plain"

    # Inputs resident in HBM for the device-timed value.
    d_entries = torch.from_numpy(entries.view(np.int64)).to(f"cuda:{local}")
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > 126 MB L2

    def timed_counter(mode):
        c = tb.Counter(device=local, dispatch=mode)
        c.set_tile_engine(args.tile_engine)
        if mode == "learned":
            c.load_model(model_path)
        c.set_stream(stream.cuda_stream)
        # The first call loads the kernels and sizes the arena; the second is timed.
        c.prepare_device(d_entries.data_ptr(), d_entries.numel(), n)
        prep = c.prepare_device(d_entries.data_ptr(), d_entries.numel(), n)
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                flush.fill_(1)
                c.launch_count()
            torch.cuda.synchronize()
            first = c.read_count()
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
            stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
            for k in range(args.steps):
                flush.fill_(k & 0xff)
                starts[k].record(stream)
                c.launch_count()
                stops[k].record(stream)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
        last = c.read_count()
        assert last.triangles == first.triangles, "count changed between launches"
        ms = [a.elapsed_time(b) for a, b in zip(starts, stops)]
        return c, prep, last, ms

    results = {}
    # The learned dispatcher is compared on the same GPU with the plain
    # fixed-threshold rule (tiles / merge / bitmap) and with all-merge.
    modes = [dispatch] + (["plain", "merge"] if dispatch == "learned" else [])
    with ClockSampler(local) as clocks:
        for mode in modes:
            c, prep, res, ms = timed_counter(mode)
            results[mode] = (prep, res, ms)
            c.close()
    clk = clocks.summary()
    prep, res, ms = results[dispatch]
    m = res.edges
    device = f"cuda:{local}"
    # Whole job: every replica's edges over the slowest replica's time.
    job_edges, total_ms = reduce_replicas(dist, m, sum(ms), device)
    ms_per_step = total_ms / args.steps
    value = job_edges / (ms_per_step / 1e3)
    per_mode = {}
    for k, v in results.items():
        e_k, t_k = reduce_replicas(dist, v[1].edges, sum(v[2]), device)
        per_mode[k] = e_k / (t_k / len(v[2]) / 1e3)

    # End to end through the public C-ABI call with pinned host entries.
    pinned = torch.empty(entries.size, dtype=torch.int64, pin_memory=True)
    pinned.numpy()[:] = entries.view(np.int64)
    host = pinned.numpy().view(np.uint64)

    def e2e_run(mode):
        c = tb.Counter(device=local, dispatch=mode)
        if mode == "learned":
            c.load_model(model_path)
        c.count_edges(host, n)  # sizes the arena
        secs, last = [], None
        with gc_held():
            for _ in range(args.e2e_steps):
                torch.cuda.synchronize()
                last, dt = wall_call(lambda: c.count_edges(host, n))
                secs.append(dt)
        c.close()
        assert last.triangles == res.triangles
        return reduce_replicas(dist, m, statistics.mean(secs), device)[1], last, secs

    e2e_t, e2e_res, e2e_secs = e2e_run(dispatch)
    e2e_by_mode = {dispatch: job_edges / e2e_t}
    if dispatch == "learned":
        t_plain, _, _ = e2e_run("plain")
        e2e_by_mode["plain"] = job_edges / t_plain

    def streamed_run(item):
        # The same call with a device budget below what a one-piece count
        # needs: the graph is counted in rank ranges (out-of-HBM path).
        frac, _, tier = item.partition(":")
        frac = float(frac)
        src = entries if args.stream_pageable else host
        c = tb.Counter(device=local, dispatch=dispatch)
        if dispatch == "learned":
            c.load_model(model_path)
        need = c.device_bytes(entries.size, n)
        c.set_device_budget(int(need * frac))
        c.set_stream_options(tier or "auto", 0)
        c.count_edges(src, n)
        secs, last = [], None
        with gc_held():
            for _ in range(2):
                torch.cuda.synchronize()
                last, dt = wall_call(lambda: c.count_edges(src, n))
                secs.append(dt)
        c.close()
        assert last.triangles == res.triangles
        t = reduce_replicas(dist, m, statistics.mean(secs), device)[1]
        return {"budget_frac": frac, "forced_tier": tier or None, "pinned": not args.stream_pageable,
                "budget_gb": round(need * frac / 1e9, 3), "one_piece_gb": round(need / 1e9, 3),
                "tier": ("one piece", "rows", "pairs")[last.stream_tier], "ranges": last.stream_ranges,
                "tasks": last.stream_tasks, "value": job_edges / t, "ms_per_step": t * 1e3,
                # host wall times of the call's uploads and of the rest before counting
                "h2d_ms": last.h2d_ms, "preprocess_ms": last.preprocess_ms,
                "count_ms": last.kernel_ms, "hub_edges": last.hub_edges}

    streamed = [streamed_run(f.strip()) for f in args.stream_budgets.split(",") if f.strip()]

    peak, peak_kind = measured_peaks()
    b_alg = 4 * (n + 1) + 4 * m
    achieved = b_alg / (ms_per_step / 1e3) / 1e9
    traffic = profiled_traffic(args.workload, dispatch)

    batch = None
    if not args.no_batch:
        # The batch under each dispatcher; the faster one is reported.
        runs = {d: batch_measurement(tb, np, torch, local, d, model_path, seed=4096 + rank)
                for d in ([dispatch, "plain"] if dispatch == "learned" else [dispatch])}
        best = min(runs, key=lambda d: runs[d]["batched_count_ms"])
        batch = dict(runs[best], dispatch=best,
                     batched_count_ms_by_dispatch={d: r["batched_count_ms"] for d, r in runs.items()})

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        steps, threads, work = cpu_baseline(entries, n, m, steps=1)
        x = steps[0]
        cpu = {"value": x["value"], "unit": "edges/s", "cores": threads, "kind": "port",
               "sample": f"oracle merge count of 32-row blocks b % {x['stride']} == 0 of the degree-ordered CSR "
                         f"({x['seconds']:.1f} s), time x {x['stride']}",
               # element reads of a sorted-merge count on the degree-ordered CSR, and per second of the GPU count
               "work_elements": work, "work_elements_per_s_gpu": work / (ms_per_step / 1e3)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": args.workload, **spec, "n": n, "entries": int(entries.size), "edges": m,
                       "triangles": res.triangles, "dispatch": dispatch, "tile_engine": args.tile_engine,
                       "parallelism": f"replicas{world}",
                       "l2": "256 MiB buffer written between timed steps; inputs > L2",
                       "preprocess_ms": prep.preprocess_ms, "gen_s": round(gen_s, 2),
                       "row_blocks_by_variant": dict(zip(tb.VARIANTS, res.row_blocks_by_variant)),
                       "per_mode_edges_per_s": per_mode,
                       "batch": batch},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes": b_alg,
                         # measured DRAM bytes of a launch (ncu, committed) over this run's launch time
                         "traffic_gbs": traffic / (ms_per_step / 1e3) / 1e9 if traffic else None,
                         "traffic_frac": traffic / (ms_per_step / 1e3) / 1e9 / peak if traffic else None},
            "cpu_baseline": cpu,
            "e2e": {"value": job_edges / e2e_t, "unit": "edges/s", "h2d_bytes_per_step": int(entries.size) * 8,
                    "d2h_bytes_per_step": 108, "ms_per_step": e2e_t * 1e3,
                    # wall time of each call on this rank (ms_per_step: their mean, slowest rank)
                    "step_ms": [round(t * 1e3, 2) for t in e2e_secs],
                    # device-timed parts of the last call (the degree pass overlaps the upload)
                    "parts_ms": {"h2d": e2e_res.h2d_ms, "preprocess": e2e_res.preprocess_ms,
                                 "count": e2e_res.kernel_ms},
                    "per_mode_edges_per_s": e2e_by_mode,
                    "streamed": streamed},
            "clocks": clk,
            "gpu_launches": args.steps * res.count_kernels,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
