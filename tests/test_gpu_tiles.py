"""The bit-tile variant's two arithmetic engines -- legacy mma.sync b1
AND+POPC and tcgen05.mma kind::i8 on bits unpacked to 0/1 with s32 in TMEM --
must give the oracle's count on blocks that fit one tile (dense cliques, small
dense graphs), on blocks that do not (the row-by-row fallback), and per graph
in a batch."""
import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.graphs import clique, comb, wheel

pytestmark = pytest.mark.gpu


def cliques_on_consecutive_ids(sizes):
    parts, base = [], 0
    for k in sizes:
        parts.append(clique(k, base=base))
        base += k
    return base, np.concatenate(parts)


CASES = [
    ("cliques_16x300", *cliques_on_consecutive_ids([300] * 16)),
    ("cliques_mixed", *cliques_on_consecutive_ids([3, 33, 64, 100, 129, 257, 512, 1000])),
    ("er_2048_dense", 2048, tb.gen_er(2048, 400_000, seed=5)),
    ("rmat_14", 1 << 14, tb.gen_rmat(14, 16, seed=14)),
    ("wheel_1000", 1000, wheel(1000)),
]


@pytest.mark.parametrize("engine", tb.TILE_ENGINES)
@pytest.mark.parametrize("name,n,e", CASES, ids=[c[0] for c in CASES])
def test_tile_engine_counts_exactly(engine, name, n, e):
    want, m = oracle.count(e, n)
    with tb.Counter(dispatch="mma") as c:
        c.set_tile_engine(engine)
        r = c.count_edges(e, n)
        assert (r.triangles, r.edges) == (want, m)
        if name.startswith("cliques"):
            assert r.row_blocks_by_variant[0] > 0


def test_tile_engines_on_a_batch_and_replay():
    e, off, nn = tb.gen_batch(48, seed=9, min_n=64, max_n=4096)
    want = np.array([oracle.count(e[off[g]:off[g + 1]], int(nn[g]))[0] for g in range(48)], dtype=np.uint64)
    for engine in tb.TILE_ENGINES:
        with tb.Counter(dispatch="mma") as c:
            c.set_tile_engine(engine)
            got, r = c.count_batch(e, off, nn)
            np.testing.assert_array_equal(got, want)
            c.capture_count()
            c.launch_count()
            np.testing.assert_array_equal(c.batch_counts(48), want)


def test_plain_rule_with_tiles_on_and_tcgen05():
    n, e = cliques_on_consecutive_ids([512] * 4)
    with tb.Counter() as c:
        c.set_tile_engine("tcgen05")
        c.set_tuning(0, 64, 64.0)  # plain rule with bit tiles on
        r = c.count_edges(e, n)
        assert r.triangles == 4 * comb(512) and r.row_blocks_by_variant[0] > 0


def test_unknown_tile_engine_is_rejected():
    with tb.Counter() as c:
        assert tb.lib.tribit_set_tile_engine(c._h, 7) == 1  # TRIBIT_ERR_INVALID_ARGUMENT


def test_tile_wait_times_out_and_the_context_recovers():
    # The tcgen05 tile kernel's mbarrier wait is bounded: with its MMAs never
    # committed it gives up, frees its TMEM and the host reads TRIBIT_ERR_TIMEOUT;
    # the context and the GPU stay usable.
    import torch
    n, e = cliques_on_consecutive_ids([256] * 8)
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter(dispatch="mma") as c:
        c.set_tile_engine("tcgen05")
        c.prepare_device(d.data_ptr(), d.numel(), n)
        assert tb.lib.tribit_test_tile_timeout(c._h, 1024) == 0
        with pytest.raises(tb.TribitError) as ex:
            c.read_count()
        assert ex.value.status == 10  # TRIBIT_ERR_TIMEOUT
        c.prepare_device(d.data_ptr(), d.numel(), n)
        c.launch_count()
        assert c.read_count().triangles == 8 * comb(256)


@pytest.mark.parametrize("polls", [1, 2, 3, 4, 8, 16, 64, 256, 4096])
def test_tile_wait_budget_gives_exact_count_or_timeout(polls):
    # With a poll budget near the MMA's own latency some CTAs' waits succeed
    # and some run out. The decision is taken for the whole CTA, the committed
    # MMAs are drained before TMEM is freed, and the launch reports either the
    # exact count or TRIBIT_ERR_TIMEOUT -- never a wrong count.
    n, e = cliques_on_consecutive_ids([256] * 24)
    want = 24 * comb(256)
    with tb.Counter(dispatch="mma") as c:
        c.set_tile_engine("tcgen05")
        c.set_tile_wait_polls(polls)
        for _ in range(3):
            try:
                r = c.count_edges(e, n)
            except tb.TribitError as ex:
                assert ex.status == 10  # TRIBIT_ERR_TIMEOUT
                continue
            assert r.triangles == want and r.row_blocks_by_variant[0] > 0
        c.set_tile_wait_polls(0)  # the default budget
        assert c.count_edges(e, n).triangles == want
