"""Row construction of the preprocessing (a counting sort of the oriented
entries by their lower endpoint, then a sort + dedup of each row): rows of
every sorting class -- the warp's register sorts (up to 1,024 entries), a
CTA's shared-memory sort (up to 8,192) and its global-scratch sort (longer) --
with duplicated and reversed entries, against the oracle."""
import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.graphs import clique, comb, wheel

pytestmark = pytest.mark.gpu


def noisy(e, seed, copies=3):
    """e with every entry repeated, half of the copies reversed, shuffled."""
    rng = np.random.default_rng(seed)
    a, b = e >> np.uint64(32), e & np.uint64(0xFFFFFFFF)
    rev = (b << np.uint64(32)) | a
    parts = [e] + [np.where(rng.random(e.size) < 0.5, rev, e) for _ in range(copies - 1)]
    out = np.concatenate(parts)
    rng.shuffle(out)
    return out


@pytest.mark.parametrize("n", [1500, 5000, 20000])
def test_long_rows_in_id_order(n):
    # In id order the wheel's hub (vertex 0) owns one row of n - 1 entries
    # (x 3 with the copies): the CTA sorts, in shared memory and in scratch.
    e = noisy(wheel(n), seed=n)
    with tb.Counter(order="id") as c:
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == (n - 1, 2 * (n - 1))


def test_clique_rows_of_every_class_in_degree_order():
    # A 1,100-clique under degree order: rows of 0..1,099 entries, x 2 with the
    # copies, so every warp class and the CTA class occur.
    k = 1100
    e = noisy(clique(k), seed=7, copies=2)
    with tb.Counter() as c:
        r = c.count_edges(e, k)
        assert (r.triangles, r.edges) == (comb(k), k * (k - 1) // 2)


@pytest.mark.parametrize("order", ["degree", "id"])
def test_random_graph_with_duplicates_matches_oracle(order):
    n = 3000
    e = noisy(tb.gen_chung_lu(n, 60_000, 2.0, 1500.0, seed=11), seed=12)
    want, m = oracle.count(e, n)
    for mode in ("plain", "merge"):
        with tb.Counter(order=order, dispatch=mode) as c:
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == (want, m), (order, mode)


def test_self_loops_and_empty_rows():
    # Self-loops are dropped; vertices without edges leave empty rows.
    e = np.concatenate([clique(40, base=100), np.array([(5 << 32) | 5, (7 << 32) | 7], dtype=np.uint64)])
    with tb.Counter() as c:
        r = c.count_edges(e, 1000)
        assert (r.triangles, r.edges) == (comb(40), 40 * 39 // 2)
