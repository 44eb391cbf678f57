"""Graphs counted in rank ranges (tribit_count_edges past the device budget)
against the oracle.

A context's device budget (tribit_set_device_budget) below what a one-piece
count needs (tribit_device_bytes) sends the count through the streamed path:
three passes of the entries through the GPU to rank them and bucket them by
rank range on the host, then one device count per pair of ranges. The count
and the undirected edge count must equal the oracle's for every budget, under
every dispatcher, and the context must stay usable for one-piece counts."""
import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.graphs import clique, comb

pytestmark = pytest.mark.gpu

GRAPHS = [
    ("rmat16", 1 << 16, lambda: tb.gen_rmat(16, 16, seed=16)),
    ("chung_lu", 30000, lambda: tb.gen_chung_lu(30000, 300000, 2.1, 3000.0, seed=3)),
    ("planted", 40000, lambda: tb.gen_planted(400, 100, 0.3, 2, seed=4)),
]


@pytest.mark.parametrize("name,n,make", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_streamed_counts_match_oracle(name, n, make):
    e = make()
    want = oracle.count(e, n)
    with tb.Counter() as c:
        need = c.device_bytes(e.size, n)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges == 1
        seen = set()
        for frac in (0.8, 0.6, 0.45):
            c.set_device_budget(int(need * frac))
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want, (name, frac, r.stream_ranges)
            assert r.stream_ranges > 1 and r.stream_tasks >= r.stream_ranges
            seen.add(r.stream_ranges)
        assert len(seen) >= 2  # smaller budgets cut more ranges
        c.set_device_budget(0)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges == 1


@pytest.mark.parametrize("dispatch", ["learned", "merge", "bitmap", "mma"])
def test_streamed_counts_under_every_dispatcher(dispatch):
    import os
    n, e = 1 << 15, tb.gen_rmat(15, 16, seed=151)
    want = oracle.count(e, n)
    with tb.Counter(dispatch=dispatch) as c:
        if dispatch == "learned":
            c.load_model(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                      "tribit_b200", "models", "dispatch_mlp.bin"))
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.5))
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges > 1


def test_streamed_duplicates_self_loops_and_dense_blocks():
    # Duplicated and reversed entries land in their lower endpoint's bucket;
    # self-loops vanish; dense cliques give rows that reach other ranges.
    sizes = [40] * 60 + [200] * 6
    offs = np.cumsum([0] + sizes)
    e = np.concatenate([clique(k, base=int(o)) for k, o in zip(sizes, offs)])
    rev = (e << np.uint64(32)) | (e >> np.uint64(32))
    loops = (np.arange(50, dtype=np.uint64) << np.uint64(32)) | np.arange(50, dtype=np.uint64)
    noisy = np.concatenate([e, rev[::3], e[::5], loops])
    n = int(offs[-1])
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(noisy.size, n) * 0.5))
        r = c.count_edges(noisy, n)
        assert r.triangles == sum(comb(k) for k in sizes) and r.edges == e.size and r.stream_ranges > 1


def test_streamed_id_range_error_and_recovery():
    n, e = 1 << 14, tb.gen_rmat(14, 16, seed=3)
    bad = e.copy()
    bad[len(bad) // 2] = (5 << 32) | (1 << 20)
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.5))
        with pytest.raises(tb.TribitError) as ex:
            c.count_edges(bad, n)
        assert ex.value.status == 5
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == oracle.count(e, n) and r.stream_ranges > 1
