"""Trains the learned dispatcher from timings the counter records itself.

For each training graph (generated here, with seeds disjoint from the
benchmark's) the counter prepares the graph on the GPU, reads the 16
features of every 32-row block (tribit_block_features), then counts the whole
graph once per variant with every row block forced onto that variant,
recording the SM cycles each row block took and the device time of the
variant's kernels (tribit_block_times); cycles scaled to that time give each
row block's cost under each variant. The MLP (16 -> 64 -> 64 -> 3) is trained
on the GPU by the library's own forward, backward and Adam kernels
(tribit_model_train) to predict log2(1 + cost in ns) of each variant, and is
evaluated on a held-out graph: total cost of the plain dispatcher's choice,
of the MLP's choice and of the per-block best (regret = chosen - best), plus
the measured counting time under each dispatcher.

  python -m tribit_b200.train_dispatch [--out tribit_b200/models/dispatch_mlp.bin] [--quick]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import tribit_b200 as tb

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "models", "dispatch_mlp.bin")


def training_graphs(quick: bool):
    """(name, make) pairs; make() returns ("graph", n, entries) or ("batch",
    entries, offsets, num_nodes) -- batches are prepared as the batched
    workload is, graph by graph (tribit_count_batch)."""
    def rmat(scale, seed):
        return lambda: ("graph", 1 << scale, tb.gen_rmat(scale, 16, seed=seed))

    def planted(c, seed):
        return lambda: ("graph", c * 100, tb.gen_planted(c, 100, 0.3, 2, seed=seed))

    def batch(g, seed):
        return lambda: ("batch", *tb.gen_batch(g, seed=seed))

    def cliques(count, size):
        # Dense tiles: disjoint cliques on consecutive ids (the planted graph's
        # random ids leave no tile dense).
        def make():
            i, j = np.triu_indices(size, 1)
            base = (np.arange(count, dtype=np.uint64) * np.uint64(size))[:, None]
            lo = (base + i.astype(np.uint64)[None, :]).ravel()
            hi = (base + j.astype(np.uint64)[None, :]).ravel()
            return "graph", count * size, (lo << np.uint64(32)) | hi
        return make

    if quick:
        return [("rmat18_s118", rmat(18, 118)), ("planted_s103", planted(4000, 103)), ("batch_s101", batch(64, 101)),
                ("cliques_32x256", cliques(32, 256))]
    # RMAT at several scales: which variant wins a block shifts with the graph's size.
    return [("rmat23_s123", rmat(23, 123)), ("rmat22_s122", rmat(22, 122)), ("rmat21_s121", rmat(21, 121)),
            ("rmat20_s120", rmat(20, 120)),
            ("rmat19_s119", rmat(19, 119)), ("rmat18_s118", rmat(18, 118)), ("planted_s103", planted(20000, 103)),
            ("batch_s101", batch(1024, 101)), ("cliques_96x384", cliques(96, 384))]


def holdout_graphs(quick: bool):
    if quick:
        return [("rmat17_s7", ("graph", 1 << 17, tb.gen_rmat(17, 16, seed=7)))]
    return [("rmat22_s7", ("graph", 1 << 22, tb.gen_rmat(22, 16, seed=7))),
            ("rmat18_s181", ("graph", 1 << 18, tb.gen_rmat(18, 16, seed=181)))]


def collect(item, repeats: int = 2):
    """Features and per-row-block cost (ns) of each variant.

    A row block's SM cycles measure how long its warp worked, not what it cost
    the machine: a variant whose kernel keeps fewer warps resident per SM
    finishes fewer blocks per second at the same cycles per block. So each
    variant's cycles are scaled to its measured device time: cost of block b
    = cycles_b / sum of cycles * time of the variant kernels."""
    import torch
    with tb.Counter(dispatch="plain") as c:
        if item[0] == "batch":
            c.count_batch(*item[1:])
        else:
            _, n, e = item
            d = torch.from_numpy(e.view(np.int64)).cuda()
            c.prepare_device(d.data_ptr(), d.numel(), n)
        x = c.block_features()
        costs, tri = [], set()
        for v in tb.VARIANTS:
            best = None
            for _ in range(repeats):
                cyc, count, ms = c.block_times(v)
                tri.add(count)
                cost = cyc / max(float(cyc.sum()), 1.0) * ms * 1e6
                best = cost if best is None or cost.sum() < best.sum() else best
            costs.append(best)
        assert len(tri) == 1, "variants disagree on the count"
    t = np.stack(costs, 1)
    keep = t.max(1) > 0
    return x[keep], t[keep], x, t


def plain_choice(item):
    """The plain dispatcher's choice of every row block (tribit_block_variants)."""
    import torch
    _, n, e = item
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter(dispatch="plain") as c:
        c.prepare_device(d.data_ptr(), d.numel(), n)
        return c.block_variants().astype(np.int64)


def learned_choice(pred, x):
    """The learned dispatcher's rule (k_dispatch): the variant of least predicted
    cost, bit tiles only for blocks that fit one tile (span of 1..64 blocks)."""
    span = np.exp2(x[:, 13]) - 1
    p = pred.copy()
    p[~((span > 0.5) & (span <= 64.5)), tb.VARIANTS.index("mma")] = np.inf
    return p.argmin(1)


def timed_count(n, e, dispatch, model, steps=5):
    import torch
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter(dispatch=dispatch) as c:
        if dispatch == "learned":
            c.load_model(model)
        s = torch.cuda.Stream()
        c.set_stream(s.cuda_stream)
        c.prepare_device(d.data_ptr(), d.numel(), n)
        ms = []
        with torch.cuda.stream(s):
            c.launch_count()
            for _ in range(steps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                c.launch_count()
                b.record(s)
                b.synchronize()
                ms.append(a.elapsed_time(b))
        r = c.read_count()
    return float(np.median(ms)), r.triangles, dict(zip(tb.VARIANTS, r.row_blocks_by_variant))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()

    xs, ys = [], []
    for name, make in training_graphs(args.quick):
        t0 = time.time()
        x, t, _, _ = collect(make())
        xs.append(x)
        ys.append(np.log2(1.0 + t))
        print(json.dumps({"graph": name, "row_blocks": int(x.shape[0]), "seconds": round(time.time() - t0, 1),
                          "ms_per_variant": dict(zip(tb.VARIANTS, [float(v) / 1e6 for v in t.sum(0)]))}), flush=True)
    X = np.concatenate(xs).astype(np.float32)
    Y = np.concatenate(ys).astype(np.float32)
    norm = np.concatenate([X.mean(0), X.std(0) + 1e-3, Y.mean(0), Y.std(0) + 1e-3]).astype(np.float32)

    with tb.Counter() as c:
        c.model_init(norm, seed=args.seed)
        loss = c.model_train(X, Y, epochs=args.epochs, batch=4096, lr=args.lr, seed=args.seed)
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        c.save_model(args.out)
    print(json.dumps({"train_rows": int(X.shape[0]), "final_loss": loss}), flush=True)
    for hname, hitem in holdout_graphs(args.quick):
        _, hn, he = hitem
        # every row block, so that the choices line up with the costs
        _, _, hx, ht = collect(hitem)
        with tb.Counter() as c:
            c.load_model(args.out)
            pred = c.model_predict(hx)
        learned = learned_choice(pred, hx)
        plain = plain_choice(hitem)
        rows = np.arange(ht.shape[0])
        best = ht.min(1).sum()
        report = {
            "holdout": hname,
            "holdout_cost_ms": {"best": float(best) / 1e6, "plain": float(ht[rows, plain].sum()) / 1e6,
                                "learned": float(ht[rows, learned].sum()) / 1e6,
                                **{f"all_{v}": float(ht[:, i].sum()) / 1e6 for i, v in enumerate(tb.VARIANTS)}},
            "learned_picks": dict(zip(tb.VARIANTS, np.bincount(learned, minlength=3).tolist())),
            "plain_picks": dict(zip(tb.VARIANTS, np.bincount(plain, minlength=3).tolist())),
        }
        p_ms, p_tri, _ = timed_count(hn, he, "plain", args.out)
        l_ms, l_tri, _ = timed_count(hn, he, "learned", args.out)
        assert p_tri == l_tri
        report["holdout_count_ms"] = {"plain": p_ms, "learned": l_ms}
        print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
