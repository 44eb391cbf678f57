"""Larger graphs: RMAT scales 20 and 24 against the oracle, and at scale 22
the size-independent property that every orientation and dispatcher agrees."""
import os

import numpy as np
import pytest

import oracle
import tribit_b200 as tb

pytestmark = pytest.mark.gpu


def test_rmat20_vs_oracle():
    e = tb.gen_rmat(20, 16, seed=20)
    want, m = oracle.count(e, 1 << 20, order=1, threads=max(1, __import__("os").cpu_count() or 1))
    for mode in ("plain", "bitmap", "merge", "mma"):
        with tb.Counter(dispatch=mode) as c:
            r = c.count_edges(e, 1 << 20)
            assert (r.triangles, r.edges) == (want, m), mode


def test_planted_vs_oracle():
    e = tb.gen_planted(4000, 100, 0.3, 2, seed=33)
    n = 400000
    want, m = oracle.count(e, n)
    with tb.Counter() as c:
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == (want, m)


def test_rmat24_vs_oracle():
    """The benchmark graph itself (RMAT scale 24, edge factor 16, seed 24):
    its count from the oracle on every host core, against the learned
    dispatch (hash-staged hubs on every warp of the hub pass), merge and plain."""
    import os
    e = tb.gen_rmat(24, 16, seed=24)
    want, m = oracle.count(e, 1 << 24, order=1, threads=max(1, os.cpu_count() or 1))
    model = os.path.join(os.path.dirname(tb.__file__), "models", "dispatch_mlp.bin")
    for mode in ("learned", "merge", "plain"):
        with tb.Counter(dispatch=mode) as c:
            if mode == "learned":
                c.load_model(model)
            r = c.count_edges(e, 1 << 24)
            assert (r.triangles, r.edges) == (want, m), mode


def test_degree_slot_rows_with_duplicates_and_loops():
    """Inputs of 2^27 entries or more build their rows in degree-sized slots:
    33 copies of RMAT-18 (every other one reversed) plus self-loops, so rows
    hold tens of thousands of entries before deduplication and are sorted in
    global scratch. The simple graph, and so the count, is RMAT-18's."""
    n = 1 << 18
    base = tb.gen_rmat(18, 16, seed=18)
    rev = (base << np.uint64(32)) | (base >> np.uint64(32))
    loops = (np.arange(1000, dtype=np.uint64) << np.uint64(32)) | np.arange(1000, dtype=np.uint64)
    e = np.concatenate([base if k % 2 == 0 else rev for k in range(33)] + [loops])
    assert e.size >= 1 << 27
    want = oracle.count(base, n)
    for mode in ("plain", "merge"):
        with tb.Counter(dispatch=mode) as c:
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want, mode


@pytest.mark.parametrize("name,n,make", [
    ("er", 1 << 20, lambda: tb.gen_er(1 << 20, 16 << 20, seed=41)),
    ("chung_lu", 1 << 20, lambda: tb.gen_chung_lu(1 << 20, 16 << 20, 2.1, 3000.0, seed=42)),
])
def test_long_bitmap_piece_lists_match_oracle(name, n, make):
    """Over a million bitmap pieces on one graph: sparse Erdos-Renyi rows, and
    Chung-Lu rows from a few neighbours to thousands (split into pieces, the
    longest staged as hashes), against the oracle, and the same count on
    repeated launches of the prepared graph."""
    e = make()
    want = oracle.count(e, n)
    for mode in ("bitmap", "learned"):
        with tb.Counter(dispatch=mode) as c:
            if mode == "learned":
                c.load_model(os.path.join(os.path.dirname(tb.__file__), "models", "dispatch_mlp.bin"))
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want, (name, mode)
            for _ in range(2):
                c.launch_count()
                assert c.read_count().triangles == want[0], (name, mode)


def test_rmat22_modes_agree():
    e = tb.gen_rmat(22, 16, seed=22)
    got = set()
    for mode in ("plain", "bitmap", "merge"):
        with tb.Counter(dispatch=mode) as c:
            got.add(c.count_edges(e, 1 << 22).triangles)
    assert len(got) == 1


def test_matches_reference_binary_on_large_graphs():
    """Counts the reference binary printed on a B200 for the same seeded graphs
    (tests/golden/ref_counts.json): RMAT 20 and 22 and the 2M-vertex planted
    partition."""
    import json
    import os
    ref = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_counts.json")))
    from tests.golden.make_golden import generate
    with tb.Counter() as c:
        for rec in ref:
            if rec["name"] not in ("rmat_s20", "rmat_s22", "planted_20000x100"):
                continue
            n, e = generate(rec["params"])
            assert c.count_edges(e, n).triangles == rec["triangles"], rec["name"]
