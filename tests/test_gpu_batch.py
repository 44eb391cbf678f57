"""Batched counting, CUDA-graph replay and tuning: per-graph counts exact
against the oracle, unchanged by replay and by every tuning setting."""
import numpy as np
import pytest
import torch

import oracle
import tribit_b200 as tb

pytestmark = pytest.mark.gpu


def test_gen_batch_shape_and_determinism():
    e, off, nn = tb.gen_batch(64, seed=5, min_n=64, max_n=4096)
    assert off[0] == 0 and off[-1] == e.size and nn.min() >= 64 and nn.max() <= 4096
    e2, off2, nn2 = tb.gen_batch(64, seed=5, min_n=64, max_n=4096)
    assert np.array_equal(e, e2) and np.array_equal(off, off2) and np.array_equal(nn, nn2)
    for g in range(64):
        part = e[off[g]:off[g + 1]]
        assert int((part >> np.uint64(32)).max()) < nn[g] and int((part & np.uint64(0xFFFFFFFF)).max()) < nn[g]


@pytest.mark.parametrize("model", ["kernels", "queue"])
@pytest.mark.parametrize("dispatch", ["plain", "bitmap", "merge", "mma"])
def test_batch_counts_and_graph_replay(dispatch, model):
    # Per-graph counts under both launch models: one persistent kernel per
    # variant, or the row pieces and hub pass in one queue-driven kernel.
    e, off, nn = tb.gen_batch(96, seed=7, min_n=64, max_n=8192)
    want = np.array([oracle.count(e[off[g]:off[g + 1]], int(nn[g]))[0] for g in range(96)], dtype=np.uint64)
    with tb.Counter(dispatch=dispatch) as c:
        c.set_tuning(0, 64, 64.0, launch_model=model)
        got, r = c.count_batch(e, off, nn)
        np.testing.assert_array_equal(got, want)
        assert r.triangles == int(want.sum())
        c.capture_count()
        for _ in range(3):
            c.launch_count()
            np.testing.assert_array_equal(c.batch_counts(96), want)
            assert c.read_count().triangles == int(want.sum())


def test_tuning_settings_keep_counts_exact():
    n = 1 << 15
    e = tb.gen_rmat(15, 16, seed=3)
    want = oracle.count(e, n)[0]
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter() as c:
        c.prepare_device(d.data_ptr(), d.numel(), n)
        for model in tb.LAUNCH_MODELS:
            for ctas in (1, 4, 7):
                for width in (32, 96, 256):
                    for tile in (0.0, 64.0, 1e30):
                        c.set_tuning(ctas, width, tile, launch_model=model)
                        c.launch_count()
                        assert c.read_count().triangles == want, (model, ctas, width, tile)
        best = c.autotune(reps=1)
        assert best.count_ms > 0 and best.piece_width in (32, 64, 128)
        t = c.tuning()
        assert (t.ctas_per_sm, t.piece_width, t.launch_model) == (best.ctas_per_sm, best.piece_width,
                                                                  best.launch_model)
        c.launch_count()
        assert c.read_count().triangles == want
        c.capture_count()
        c.launch_count()
        assert c.read_count().triangles == want
    with pytest.raises(tb.TribitError):
        with tb.Counter() as c:
            c.set_tuning(4, 48, 64.0)  # not a multiple of 32


@pytest.mark.parametrize("dispatch", ["learned", "plain", "merge", "bitmap", "mma"])
def test_queue_kernel_matches_oracle(dispatch):
    # The queue launch model on graphs that reach every one of its phases:
    # hub and row pieces (RMAT), dense tiles (cliques), and heavy rows, one CTA
    # each (a dense Erdos-Renyi graph: 4,209 oriented rows span more than 256
    # bit blocks).
    import os
    from tests.graphs import clique
    cases = [(1 << 16, tb.gen_rmat(16, 16, seed=61)),
             (64 * 40, np.concatenate([clique(40, base=40 * k) for k in range(64)])),
             (16000, tb.gen_er(16000, 4_800_000, seed=9))]
    model = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tribit_b200", "models",
                         "dispatch_mlp.bin")
    with tb.Counter(dispatch=dispatch) as c:
        if dispatch == "learned":
            c.load_model(model)
        c.set_tuning(0, 64, 64.0, launch_model="queue")
        for n, e in cases:
            want = oracle.count(e, n)
            r = c.count_edges(e, n)
            assert (r.triangles, r.edges) == want, (dispatch, n)
            for _ in range(2):
                c.launch_count()
                assert c.read_count().triangles == want[0]
