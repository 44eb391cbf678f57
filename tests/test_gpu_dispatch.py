"""What the trained dispatcher gains over the plain fixed-threshold rule.

On a held-out graph (RMAT scale 18, seed 181: neither its scale nor its seed is
among the training graphs of tribit_b200/train_dispatch.py), the counter
records each 32-row block's cost under every variant (tribit_block_times:
warp-cycles of the block's pieces, scaled to the variant kernels' measured
time, as the trainer does). The summed cost of the learned network's choices
must stay within a stated regret of the per-block best and below the summed
cost of the plain rule's choices (bit tiles / merge / bitmap by fixed
thresholds, tribit_block_variants), and every count stays exact.
"""
import os

import numpy as np
import pytest

import oracle
import tribit_b200 as tb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODEL = os.path.join(ROOT, "tribit_b200", "models", "dispatch_mlp.bin")
MAX_REGRET = 0.15  # learned cost <= (1 + MAX_REGRET) x per-block best


def block_costs(c, want):
    """(row blocks x 3) cost of every variant (VARIANTS order), in ms."""
    cols = []
    for v in tb.VARIANTS:
        reps = []
        for _ in range(2):
            cyc, tri, ms = c.block_times(v)
            assert tri == want, v
            reps.append(cyc / max(float(cyc.sum()), 1.0) * ms)
        cols.append(np.minimum(*reps))
    return np.stack(cols, axis=1)


def test_learned_choices_beat_plain_rule_on_held_out_graph():
    import torch
    n, e = 1 << 18, tb.gen_rmat(18, 16, seed=181)
    want, m = oracle.count(e, n)
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter(dispatch="plain") as p:
        p.prepare_device(d.data_ptr(), d.numel(), n)
        plain = p.block_variants()
        p.launch_count()
        assert p.read_count().triangles == want
    with tb.Counter(dispatch="learned") as c:
        c.load_model(MODEL)
        r = c.prepare_device(d.data_ptr(), d.numel(), n)
        assert r.edges == m
        learned = c.block_variants()
        c.launch_count()
        assert c.read_count().triangles == want
        cost = block_costs(c, want)
    assert len(plain) == len(learned) == cost.shape[0]
    rows = np.arange(cost.shape[0])
    best = float(cost.min(axis=1).sum())
    got = float(cost[rows, learned].sum())
    base = float(cost[rows, plain].sum())
    print(f"held-out RMAT-18: best {best:.3f} ms, learned {got:.3f} ms, plain {base:.3f} ms, "
          f"all-merge {float(cost[:, 2].sum()):.3f} ms")
    assert got <= (1.0 + MAX_REGRET) * best, (got, best)
    assert got < base, (got, base)
