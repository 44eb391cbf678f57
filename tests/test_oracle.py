"""The CPU oracle against closed-form known answers and the golden fixtures."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from tests.conftest import WIKI_VOTE, WIKI_VOTE_SHA256_16
import tribit_b200 as tb
from tests.graphs import clique, comb, numpy_count, star, wheel, zip_pairs

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_counts.json")))


@pytest.mark.parametrize("n", [3, 4, 5, 10, 33, 64, 100])
def test_clique(n):
    e = clique(n)
    for order in (0, 1):
        assert oracle.count(e, n, order=order) == (comb(n), n * (n - 1) // 2)
    assert oracle.count_tribit(e, n)[0] == comb(n)


@pytest.mark.parametrize("n", [5, 6, 40, 100])
def test_wheel(n):
    assert oracle.count(wheel(n), n)[0] == n - 1
    assert oracle.count_tribit(wheel(n), n)[0] == n - 1


def test_star_empty_single():
    assert oracle.count(star(50), 50) == (0, 49)
    assert oracle.count(np.zeros(0, dtype=np.uint64), 10) == (0, 0)
    assert oracle.count(zip_pairs([(0, 1), (1, 2), (0, 2)]), 3) == (1, 3)
    assert oracle.count_tribit(np.zeros(0, dtype=np.uint64), 10) == (0, 0)


def test_duplicates_selfloops_unfolded():
    base = zip_pairs([(0, 1), (1, 2), (2, 0), (2, 3), (3, 0)])
    noisy = np.concatenate([base, zip_pairs([(1, 0), (2, 1), (0, 2), (3, 3), (1, 1), (0, 1), (3, 2)])])
    assert oracle.count(noisy, 4) == oracle.count(base, 4) == (2, 5)


def test_disjoint_cliques():
    e = np.concatenate([clique(k, base=sum(range(3, k))) for k in range(3, 12)])
    n = sum(range(3, 12))
    assert oracle.count(e, n)[0] == sum(comb(k) for k in range(3, 12))


def test_random_against_dense_numpy():
    rng = np.random.default_rng(0)
    for trial in range(20):
        n = int(rng.integers(2, 120))
        m = int(rng.integers(0, 2000))
        a = rng.integers(0, n, size=m, dtype=np.uint64)
        b = rng.integers(0, n, size=m, dtype=np.uint64)
        e = (a << np.uint64(32)) | b
        want = numpy_count(e, n)
        assert oracle.count(e, n, order=0)[0] == want
        assert oracle.count(e, n, order=1)[0] == want
        assert oracle.count_tribit(e, n)[0] == want


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["name"] != "wiki-Vote" and c["entries"] <= 400000],
                         ids=lambda c: c["name"])
def test_golden_generated(case):
    from tests.golden.make_golden import checksum, generate
    n, e = generate(case["params"])
    assert checksum(e) == case["entries_sha256_16"], "generator output drifted"
    t, m = oracle.count(e, n)
    assert (t, m) == (case["triangles"], case["edges"])
    assert oracle.count_tribit(e, n) == (case["triangles"], case["reference_blocks_of_threads"])


def test_wiki_vote_reference_fixture():
    rec = [c for c in GOLDEN if c["name"] == "wiki-Vote"][0]
    with open(WIKI_VOTE, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest()[:16] == rec["params"]["file_sha256_16"] == WIKI_VOTE_SHA256_16
    st, n, e = oracle.read_mtx(WIKI_VOTE)
    assert st == 0 and n == rec["num_nodes"] == 8297 and len(e) == rec["entries"]
    assert oracle.count(e, n) == (608389, 100762)
    assert oracle.count_tribit(e, n) == (608389, 28449)


def test_row_counts_sum():
    e = tb.gen_rmat(11, 8, seed=3)
    g = oracle.CSR(e, 1 << 11)
    rows = g.row_counts()
    t, _ = g.count(threads=4)
    assert int(rows.sum()) == t == oracle.count(e, 1 << 11)[0]


REF = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_counts.json")))


@pytest.mark.parametrize("rec", [r for r in REF if r["name"] in {c["name"] for c in GOLDEN}], ids=lambda r: r["name"])
def test_reference_binary_output_pins_oracle(rec):
    """What the reference binary printed on a B200 equals the oracle's count and
    its restatement of the reference's work decomposition."""
    want = [c for c in GOLDEN if c["name"] == rec["name"]][0]
    assert rec["status"] == "ok" and rec["cuda"] == "No cuda error detected"
    assert rec["triangles"] == want["triangles"]
    assert rec["blocks_of_threads"] == want["reference_blocks_of_threads"]


def test_reference_binary_rmat18_pins_oracle():
    import ctypes
    rec = [r for r in REF if r["name"] == "rmat_s18"][0]
    e = tb.gen_rmat(18, 16, seed=rec["params"]["seed"])
    t, _ = oracle.count(e, 1 << 18)
    assert t == rec["triangles"]
    f = oracle.fold_dedup(e)
    oracle._lib.oracle_tribit_blocks.restype = ctypes.c_uint64
    oracle._lib.oracle_tribit_blocks.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    assert oracle._lib.oracle_tribit_blocks(f.ctypes.data, f.size) == rec["blocks_of_threads"]


@pytest.mark.parametrize("scale,ef,seed", [(8, 16, 1), (12, 4, 7), (16, 16, 24)])
def test_oracle_rmat_generator_matches_product(scale, ef, seed):
    # The benchmark's reference arm generates its graph with the oracle's own
    # R-MAT restatement (it must not load the product library); both must give
    # the same words, for any host thread count.
    import tribit_b200 as tb
    want = tb.gen_rmat(scale, ef, seed=seed)
    for threads in (1, 3, 8):
        np.testing.assert_array_equal(oracle.gen_rmat(scale, ef, seed=seed, threads=threads), want)


def test_merge_work_figure():
    # W = sum over oriented edges (u, v) of d+(u) + d+(v), from the CSR's own
    # rows, against the same sum taken edge by edge in Python.
    rng = np.random.default_rng(9)
    n = 300
    a = rng.integers(0, n, 4000, dtype=np.uint64)
    b = rng.integers(0, n, 4000, dtype=np.uint64)
    g = oracle.CSR(zip_pairs(zip(a, b)), n, order=1)
    rp = np.ctypeslib.as_array(g._g.row_ptr, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(g._g.col, shape=(g.m,)).copy()
    d = np.diff(rp)
    want = sum(int(d[u]) + int(d[v]) for u in range(n) for v in col[rp[u]:rp[u + 1]])
    assert g.work() == want and want > 0
    g.close()
