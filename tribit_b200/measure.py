"""Counting time and preprocessing time of one seeded workload, device-timed.

The graph is generated on the host, copied to the device once, and prepared
three times from device memory (median preprocessing time); then
`steps + 3` counting launches run on one stream, each after a 256 MiB buffer
write that flushes the L2, timed with CUDA events on that stream; the first
three are warm-up. Prints one JSON line: the median and minimum counting time,
the preprocessing time, the count and the dispatcher's row blocks per variant.
`--gen batch` is the benchmark's 4,096-graph batch, prepared from host memory
by tribit_count_batch (tiles off, 7 CTAs an SM, 128-neighbour pieces).

  python -m tribit_b200.measure --scale 24 --seed 24 [--dispatch learned]
      [--model PATH] [--gen rmat|planted|er|er_small|c1|batch] [--launch-model kernels|queue|auto]
      [--steps 10] [--tag NAME]

This is the launch-timing loop the profiles under `profiles/` cite; `bench.py`
is the benchmark.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics

import numpy as np

import tribit_b200 as tb

HERE = os.path.dirname(os.path.abspath(__file__))


def workload(gen: str, scale: int, seed: int):
    """(num_nodes, entries) of a named seeded workload."""
    if gen == "planted":
        return 2_000_000, tb.gen_planted(20000, 100, 0.3, 2, seed=3)
    if gen == "er":
        return 1 << 20, tb.gen_er(1 << 20, 16 << 20, seed=5)
    if gen == "er_small":
        return 1 << 16, tb.gen_er(1 << 16, 1 << 20, seed=6)
    if gen == "c1":
        return 7115, tb.gen_chung_lu(7115, 115300, 2.0, 1000.0, seed=1)
    if gen == "rmat":
        return 1 << scale, tb.gen_rmat(scale, 16, seed=seed)
    raise ValueError(f"unknown workload {gen}")


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--seed", type=int, default=24)
    ap.add_argument("--dispatch", default="learned", choices=sorted(tb.DISPATCH))
    ap.add_argument("--model", default=os.path.join(HERE, "models", "dispatch_mlp.bin"))
    ap.add_argument("--gen", default="rmat", choices=["rmat", "planted", "er", "er_small", "c1", "batch"])
    ap.add_argument("--launch-model", default="auto", choices=list(tb.LAUNCH_MODELS))
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--tag", default="")
    a = ap.parse_args()

    batch = a.gen == "batch"
    if batch:  # the 4,096-graph batch of the benchmark, tiles off, 7 CTAs an SM, 128-neighbour pieces
        e, off, nn = tb.gen_batch(4096, seed=4096)
    else:
        n, e = workload(a.gen, a.scale, a.seed)
        d = torch.from_numpy(e.view(np.int64)).cuda()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    with tb.Counter(dispatch=a.dispatch) as c:
        if a.dispatch == "learned":
            c.load_model(a.model)
        c.set_stream(s.cuda_stream)
        if batch:
            c.set_tuning(7, 128, 1e30, launch_model=a.launch_model)
            c.count_batch(e, off, nn)
            prep = [c.count_batch(e, off, nn)[1].preprocess_ms for _ in range(3)]
        else:
            c.set_tuning(0, 64, 64.0, launch_model=a.launch_model)
            c.prepare_device(d.data_ptr(), d.numel(), n)
            prep = [c.prepare_device(d.data_ptr(), d.numel(), n).preprocess_ms for _ in range(3)]
        ms = []
        with torch.cuda.stream(s):
            for k in range(a.steps + 3):
                flush.fill_(k & 0xff)
                x, y = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                x.record(s)
                c.launch_count()
                y.record(s)
                y.synchronize()
                ms.append(x.elapsed_time(y))
        r = c.read_count()
    print(json.dumps({"tag": a.tag, "gen": a.gen, "scale": a.scale, "dispatch": a.dispatch,
                      "launch_model": a.launch_model, "count_ms": round(statistics.median(ms[3:]), 3),
                      "count_min_ms": round(min(ms[3:]), 3), "prep_ms": round(statistics.median(prep), 2),
                      "triangles": r.triangles, "blocks": list(r.row_blocks_by_variant),
                      "hub_edges": r.hub_edges}), flush=True)


if __name__ == "__main__":
    main()
