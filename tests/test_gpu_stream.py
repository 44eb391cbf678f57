"""Graphs counted in rank ranges (tribit_count_edges past the device budget)
against the oracle.

A context's device budget (tribit_set_device_budget) below what a one-piece
count needs (tribit_device_bytes) sends the count through the streamed path:
passes of the entries through the GPU to rank them, then either the rows tier
(each range's rows built in turn into one resident oriented graph, counted
once; up to four ranges filled from one more pass of the entries each, more
from host buckets of oriented keys) or the pairs tier (host buckets, one
device count per pair of ranges). The count and the undirected edge count
must equal the oracle's for every budget, tier, range bound and dispatcher,
and the context must stay usable for one-piece counts."""
import os

import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.graphs import clique, comb

pytestmark = pytest.mark.gpu

ROWS, PAIRS = 1, 2
MODEL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tribit_b200", "models",
                     "dispatch_mlp.bin")

GRAPHS = [
    ("rmat16", 1 << 16, lambda: tb.gen_rmat(16, 16, seed=16)),
    ("chung_lu", 30000, lambda: tb.gen_chung_lu(30000, 300000, 2.1, 3000.0, seed=3)),
    ("planted", 40000, lambda: tb.gen_planted(400, 100, 0.3, 2, seed=4)),
]


def _schedule(r):
    return r.row_blocks, tuple(r.row_blocks_by_variant), r.hub_edges


@pytest.mark.parametrize("name,n,make", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_streamed_counts_match_oracle(name, n, make):
    e = make()
    want = oracle.count(e, n)
    with tb.Counter() as c:
        need = c.device_bytes(e.size, n)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges == 1 and r.stream_tier == 0
        one_piece = _schedule(r)
        for frac in (0.8, 0.5, 0.35):
            c.set_device_budget(int(need * frac))
            try:
                r = c.count_edges(e, n)
            except tb.TribitError as ex:  # the smallest budget may fit neither tier on a small graph
                assert ex.status == 8 and frac < 0.5, (name, frac, str(ex))
                continue
            assert (r.triangles, r.edges) == want, (name, frac, r.stream_tier, r.stream_ranges)
            assert r.stream_tier in (ROWS, PAIRS)
            if r.stream_tier == ROWS:
                # The rows tier builds the one-piece oriented graph, range by
                # range; a small budget may leave no room for the hub in-lists,
                # and the dispatcher's merge blocks then go to the bitmap sweep.
                assert r.stream_tasks == 1 and r.row_blocks == one_piece[0], (name, frac)
                mma, bitmap, merge = one_piece[1]
                assert _schedule(r) == one_piece or (r.hub_edges == 0 and frac < 0.8 and
                                                     _schedule(r)[1] == (mma, bitmap + merge, 0)), (name, frac)
        # Rows tier in a few ranges (filled from the streamed entries) and in
        # many (from host buckets): the same graph again.
        c.set_device_budget(int(need * 0.8))
        kept = int(np.count_nonzero((e >> np.uint64(32)) != (e & np.uint64(0xffffffff))))
        seen = set()
        for parts in (3, 11):
            c.set_stream_options("rows", kept // parts)
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want and r.stream_tier == ROWS, (name, parts)
            assert r.stream_ranges >= parts and _schedule(r) == one_piece
            seen.add(r.stream_ranges)
        assert len(seen) == 2
        # The pairs tier at the same budgets.
        seen = set()
        for frac in (0.8, 0.6, 0.45):
            c.set_device_budget(int(need * frac))
            c.set_stream_options("pairs", 0)
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want, (name, frac, r.stream_ranges)
            assert r.stream_tier == PAIRS and r.stream_ranges > 1 and r.stream_tasks >= r.stream_ranges
            seen.add(r.stream_ranges)
        assert len(seen) >= 2  # smaller budgets cut more ranges
        c.set_stream_options("auto", 0)
        c.set_device_budget(0)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges == 1 and r.stream_tier == 0


@pytest.mark.parametrize("tier,parts", [("rows", 3), ("rows", 8), ("pairs", 0)])
@pytest.mark.parametrize("dispatch", ["learned", "merge", "bitmap", "mma"])
def test_streamed_counts_under_every_dispatcher(dispatch, tier, parts):
    n, e = 1 << 15, tb.gen_rmat(15, 16, seed=151)
    want = oracle.count(e, n)
    with tb.Counter(dispatch=dispatch) as c:
        if dispatch == "learned":
            c.load_model(MODEL)
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.5))
        c.set_stream_options(tier, e.size // parts if parts else 0)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == want and r.stream_ranges > 1
        assert r.stream_tier == (ROWS if tier == "rows" else PAIRS)


@pytest.mark.parametrize("tier,parts", [("rows", 2), ("rows", 9), ("pairs", 0)])
def test_streamed_counts_from_pinned_host_memory(tier, parts):
    # Pinned host entries are copied straight from the caller's buffer.
    import torch
    n, e = 1 << 16, tb.gen_rmat(16, 16, seed=61)
    pinned = torch.empty(e.size, dtype=torch.int64, pin_memory=True)
    pinned.numpy()[:] = e.view(np.int64)
    host = pinned.numpy().view(np.uint64)
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.6))
        c.set_stream_options(tier, e.size // parts if parts else 0)
        r = c.count_edges(host, n)
        assert (r.triangles, r.edges) == oracle.count(e, n) and r.stream_ranges > 1


def test_rows_tier_leaves_the_graph_prepared():
    # After a rows-tier count the context holds the oriented graph: launching
    # the count again gives the same result, as after a one-piece count.
    n, e = 1 << 15, tb.gen_rmat(15, 16, seed=7)
    want = oracle.count(e, n)
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.6))
        c.set_stream_options("rows", e.size // 4)
        r = c.count_edges(e, n)
        assert r.stream_tier == ROWS and (r.triangles, r.edges) == want
        for _ in range(3):
            c.launch_count()
            assert c.read_count().triangles == want[0]


def test_streamed_duplicates_self_loops_and_dense_blocks():
    # Duplicated and reversed entries land in their lower endpoint's bucket;
    # self-loops vanish; dense cliques give rows that reach other ranges and
    # rows long enough for the CTA sort.
    sizes = [40] * 60 + [200] * 6 + [1500]
    offs = np.cumsum([0] + sizes)
    e = np.concatenate([clique(k, base=int(o)) for k, o in zip(sizes, offs)])
    rev = (e << np.uint64(32)) | (e >> np.uint64(32))
    loops = (np.arange(50, dtype=np.uint64) << np.uint64(32)) | np.arange(50, dtype=np.uint64)
    noisy = np.concatenate([e, rev[::3], e[::5], loops])
    n = int(offs[-1])
    want = sum(comb(k) for k in sizes)
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(noisy.size, n) * 0.5))
        for tier, bound in (("rows", noisy.size // 6), ("pairs", 0), ("auto", 0)):
            c.set_stream_options(tier, bound)
            r = c.count_edges(noisy, n)
            assert r.triangles == want and r.edges == e.size and r.stream_ranges >= 1, tier
            assert r.stream_tier in (ROWS, PAIRS)


def test_streamed_id_range_error_and_recovery():
    n, e = 1 << 14, tb.gen_rmat(14, 16, seed=3)
    bad = e.copy()
    bad[len(bad) // 2] = (5 << 32) | (1 << 20)
    with tb.Counter() as c:
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.5))
        for tier in ("rows", "pairs"):
            c.set_stream_options(tier, e.size // 3 if tier == "rows" else 0)
            with pytest.raises(tb.TribitError) as ex:
                c.count_edges(bad, n)
            assert ex.value.status == 5
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == oracle.count(e, n) and r.stream_ranges > 1


def test_stream_option_errors():
    n, e = 1 << 14, tb.gen_rmat(14, 16, seed=5)
    with tb.Counter() as c:
        assert tb.lib.tribit_set_stream_options(c.handle, 7, 0) == 1  # no such tier
        c.set_device_budget(int(c.device_bytes(e.size, n) * 0.5))
        # A range bound at the longest row cannot hold that row with anything else.
        c.set_stream_options("rows", 1)
        with pytest.raises(tb.TribitError) as ex:
            c.count_edges(e, n)
        assert ex.value.status == 8
        c.set_stream_options("auto", 0)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == oracle.count(e, n)


@pytest.mark.parametrize("pinned", [False, True])
def test_streamed_rows_tier_on_a_million_vertices(pinned):
    # Megabyte-sized uploads of the row starts and ranks through the pinned
    # staging buffers, then pieces of the entries through the same buffers
    # (pageable input): every buffer is refilled only after its last copy.
    import torch
    n, e = 1 << 20, tb.gen_rmat(20, 16, seed=20)
    host = e
    if pinned:
        t = torch.empty(e.size, dtype=torch.int64, pin_memory=True)
        t.numpy()[:] = e.view(np.int64)
        host = t.numpy().view(np.uint64)
    with tb.Counter() as c:
        want = c.count_edges(e, n)
        for parts in (2, 6):
            c.set_device_budget(int(c.device_bytes(e.size, n) * 0.6))
            c.set_stream_options("rows", e.size // parts)
            r = c.count_edges(host, n)
            assert (r.triangles, r.edges) == (want.triangles, want.edges) and r.stream_tier == ROWS, parts
            assert _schedule(r)[:2] == _schedule(want)[:2]
            c.set_device_budget(0)
            c.set_stream_options("auto", 0)
