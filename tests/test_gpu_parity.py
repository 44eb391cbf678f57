"""GPU counts vs the CPU oracle, through the C-ABI (tribit_count_edges & co).

Bit-exact parity: every count and every deduplicated edge count must equal
the oracle's on the same seeded input."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.golden.make_golden import checksum, generate
from tests.graphs import clique, comb, numpy_count, star, wheel, zip_pairs

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_counts.json")))
GENERATED = [c for c in GOLDEN if "gen" in c["params"]]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODES = ["plain", "bitmap", "merge", "mma"]


@pytest.fixture(scope="module")
def counters():
    cs = {(o, d): tb.Counter(order=o, dispatch=d) for o in ("degree", "id") for d in MODES}
    yield cs
    for c in cs.values():
        c.close()


@pytest.mark.parametrize("case", GENERATED, ids=lambda c: c["name"])
def test_golden_cases_all_modes(counters, case):
    n, e = generate(case["params"])
    assert checksum(e) == case["entries_sha256_16"]
    for (order, mode), c in counters.items():
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == (case["triangles"], case["edges"]), (order, mode)
        assert r.blocks_of_threads > 0


@pytest.mark.parametrize("n", [3, 4, 31, 32, 33, 64, 100, 200])
def test_cliques(counters, n):
    for c in counters.values():
        r = c.count_edges(clique(n), n)
        assert (r.triangles, r.edges) == (comb(n), n * (n - 1) // 2)


@pytest.mark.parametrize("n", [5, 33, 1000])
def test_wheels_and_stars(counters, n):
    for c in counters.values():
        assert c.count_edges(wheel(n), n).triangles == n - 1
        assert c.count_edges(star(n), n).triangles == 0


def test_empty_and_tiny(counters):
    for c in counters.values():
        r = c.count_edges(np.zeros(0, dtype=np.uint64), 10)
        assert (r.triangles, r.edges) == (0, 0)
        r = c.count_edges(np.zeros(0, dtype=np.uint64), 0)
        assert r.triangles == 0
        assert c.count_edges(zip_pairs([(0, 1)]), 2).triangles == 0
        assert c.count_edges(zip_pairs([(0, 1), (1, 2), (2, 0)]), 3).triangles == 1
        # only self-loops
        assert c.count_edges(zip_pairs([(1, 1), (2, 2)]), 3).edges == 0


def test_duplicates_selfloops_unfolded(counters):
    base = zip_pairs([(0, 1), (1, 2), (2, 0), (2, 3), (3, 0)])
    noisy = np.concatenate([base, zip_pairs([(1, 0), (2, 1), (0, 2), (3, 3), (1, 1), (0, 1), (3, 2)] * 50)])
    for c in counters.values():
        r = c.count_edges(noisy, 4)
        assert (r.triangles, r.edges) == (2, 5)


def test_disjoint_cliques(counters):
    sizes = list(range(3, 40))
    offs = np.cumsum([0] + sizes)
    e = np.concatenate([clique(k, base=int(o)) for k, o in zip(sizes, offs)])
    want = sum(comb(k) for k in sizes)
    for c in counters.values():
        assert c.count_edges(e, int(offs[-1])).triangles == want


def test_random_small_vs_dense(counters):
    rng = np.random.default_rng(7)
    for _ in range(25):
        n = int(rng.integers(2, 300))
        m = int(rng.integers(0, 6000))
        a = rng.integers(0, n, size=m, dtype=np.uint64)
        b = rng.integers(0, n, size=m, dtype=np.uint64)
        e = (a << np.uint64(32)) | b
        want = numpy_count(e, n)
        for c in counters.values():
            assert c.count_edges(e, n).triangles == want


def test_id_range_error(counters):
    e = zip_pairs([(0, 1), (1, 2), (2, 7)])
    for c in counters.values():
        with pytest.raises(tb.TribitError) as ex:
            c.count_edges(e, 5)
        assert ex.value.status == 5
        # the context stays usable
        assert c.count_edges(clique(5), 5).triangles == 10


def test_big_rows_take_cta_and_global_paths():
    # id order: hub 0 has every rim vertex as a higher neighbour, so its row
    # overflows the warp slice (> 256 bit blocks) and, at 300k neighbours,
    # the CTA table (> 8192 bit blocks) too.
    for n in (3000, 40000, 300001):
        e = wheel(n)
        for mode in MODES:
            with tb.Counter(order="id", dispatch=mode) as c:
                assert c.count_edges(e, n).triangles == n - 1
    # dense hub neighbourhoods: a clique of 1500 on top of a hub
    k = 1500
    e = np.concatenate([clique(k, base=1), star(k + 1)])
    for order in ("id", "degree"):
        for mode in MODES:
            with tb.Counter(order=order, dispatch=mode) as c:
                assert c.count_edges(e, k + 1).triangles == comb(k + 1)


def test_hub_pass_takes_short_tails_and_stays_exact():
    # Power-law graphs: in merge row blocks, edges into high-rank hubs whose
    # bit rows are longer than u's tail go to the hub pass; the rest stay with
    # their rows. Every split must give the oracle's count.
    for scale, seed in ((12, 1), (15, 2), (17, 3)):
        n = 1 << scale
        e = tb.gen_rmat(scale, 16, seed=seed)
        want, m = oracle.count(e, n)
        with tb.Counter(dispatch="merge") as c:
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == (want, m)
            assert 0 < r.hub_edges < m
        with tb.Counter(dispatch="bitmap") as c:
            r = c.count_edges(e, n)
            assert r.triangles == want and r.hub_edges == 0
    # A clique on top of a star: every rim vertex's tail is shorter than the
    # rows of the higher-ranked clique members it points to.
    k = 300
    e = np.concatenate([clique(k, base=1), star(k + 1)])
    for order in ("degree", "id"):
        with tb.Counter(order=order, dispatch="merge") as c:
            r = c.count_edges(e, k + 1)
            assert r.triangles == comb(k + 1)


def test_repeated_and_resized_calls(counters):
    c = counters[("degree", "plain")]
    cases = [generate(x["params"]) + (x,) for x in GENERATED[:4]]
    for _ in range(2):
        for n, e, x in cases[::-1] + cases:
            assert c.count_edges(e, n).triangles == x["triangles"]


def test_two_phase_device_api():
    torch = pytest.importorskip("torch")
    case = [c for c in GENERATED if c["name"] == "rmat_s14"][0]
    n, e = generate(case["params"])
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter() as c:
        r = c.prepare_device(d.data_ptr(), d.numel(), n)
        assert r.edges == case["edges"]
        for _ in range(3):
            c.launch_count()
        r = c.read_count()
        assert r.triangles == case["triangles"]
        s = torch.cuda.Stream()
        c.set_stream(s.cuda_stream)
        c.launch_count()
        assert c.read_count().triangles == case["triangles"]
        r = c.count_edges_device(d.data_ptr(), d.numel(), n)
        assert r.triangles == case["triangles"]


def test_batch_per_graph_counts():
    rng = np.random.default_rng(3)
    graphs = []
    for g in range(60):
        n = int(rng.integers(1, 3000))
        kind = g % 3
        if kind == 0:
            e = tb.gen_er(n, int(rng.integers(0, 20 * n)), seed=g)
        elif kind == 1:
            e = tb.gen_chung_lu(n, int(rng.integers(0, 15 * n)), 2.3, max(2.0, n / 4), seed=g)
        else:
            k = int(min(n, rng.integers(3, 60)))
            e = clique(k)
        graphs.append((n, e))
    offs = np.cumsum([0] + [len(e) for _, e in graphs]).astype(np.uint64)
    allv = np.concatenate([e for _, e in graphs]).astype(np.uint64)
    nn = np.array([n for n, _ in graphs], dtype=np.uint32)
    want = np.array([oracle.count(e, n)[0] for n, e in graphs], dtype=np.uint64)
    for order in ("degree", "id"):
        for mode in MODES:
            with tb.Counter(order=order, dispatch=mode) as c:
                got, r = c.count_batch(allv, offs, nn)
                np.testing.assert_array_equal(got, want)
                assert r.triangles == int(want.sum())


def test_batch_id_range_per_graph():
    e = np.concatenate([clique(4), zip_pairs([(0, 3)])])  # graph 1 has only 3 vertices
    with tb.Counter() as c:
        with pytest.raises(tb.TribitError) as ex:
            c.count_batch(e, [0, 6, 7], [4, 3])
        assert ex.value.status == 5


def test_cli_summary_block(tmp_path):
    case = [c for c in GENERATED if c["name"] == "chung_lu_7115"][0]
    n, e = generate(case["params"])
    p = tmp_path / "c1.mtx"
    tb.write_mtx(str(p), n, e)
    cli = os.path.join(ROOT, "tribit_b200", "bin", "tribit")
    r = subprocess.run([cli, "-i", str(p)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    # the reference harness regexes (artifact/sc26/run_benchmarks/run_single_gpu.py:78-83)
    assert int(re.search(r"Triangles\s*:\s*(\d+)", out).group(1)) == case["triangles"]
    assert int(re.search(r"Blocks of threads\s*:\s*(\d+)", out).group(1)) > 0
    assert float(re.search(r"Preprocessing \(ms\)\s*:\s*([\d.]+)", out).group(1)) > 0
    assert float(re.search(r"Kernel \(ms\)\s*:\s*([\d.]+)", out).group(1)) > 0
    assert "Triangle Counting Summary" in out and "No cuda error detected at" in out
    lines = out.splitlines()
    assert lines[0].startswith("Thrust version: ") and lines[1].startswith("CUB version: ")
    assert lines[2] == f"Reading data from {p}..."


def test_wiki_vote_reference_fixture_all_modes():
    """The reference's one shipped graph (wiki-Vote.mtx at the root of
    sixt99/TriBIT) under every dispatcher and both orientations: the count the
    reference binary printed for it on a B200 (tests/golden/ref_counts.json)."""
    from tests.conftest import WIKI_VOTE
    ref = [r for r in json.load(open(os.path.join(ROOT, "tests", "golden", "ref_counts.json")))
           if r["name"] == "wiki-Vote"][0]
    assert ref["triangles"] == 608389
    n, e = tb.read_mtx(WIKI_VOTE)
    assert n == 8297
    model = os.path.join(ROOT, "tribit_b200", "models", "dispatch_mlp.bin")
    for order in ("degree", "id"):
        for mode in MODES + ["learned"]:
            with tb.Counter(order=order, dispatch=mode) as c:
                if mode == "learned":
                    c.load_model(model)
                r = c.count_edges(e, n)
                assert (r.triangles, r.edges) == (ref["triangles"], 100762), (order, mode)
                assert c.count_mtx(WIKI_VOTE).triangles == ref["triangles"], (order, mode)


def test_cli_on_wiki_vote_matches_reference_binary():
    from tests.conftest import WIKI_VOTE
    ref = [r for r in json.load(open(os.path.join(ROOT, "tests", "golden", "ref_counts.json")))
           if r["name"] == "wiki-Vote"][0]
    cli = os.path.join(ROOT, "tribit_b200", "bin", "tribit")
    r = subprocess.run([cli, "-i", WIKI_VOTE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # the reference harness regexes (artifact/sc26/run_benchmarks/run_single_gpu.py:78-83)
    assert int(re.search(r"Triangles\s*:\s*(\d+)", r.stdout).group(1)) == ref["triangles"]
    assert f"Graph              : {WIKI_VOTE}" in r.stdout
