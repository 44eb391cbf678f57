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


@pytest.mark.parametrize("dispatch", ["plain", "bitmap", "merge", "mma"])
def test_batch_counts_and_graph_replay(dispatch):
    e, off, nn = tb.gen_batch(96, seed=7, min_n=64, max_n=8192)
    want = np.array([oracle.count(e[off[g]:off[g + 1]], int(nn[g]))[0] for g in range(96)], dtype=np.uint64)
    with tb.Counter(dispatch=dispatch) as c:
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
        for ctas in (1, 4, 7):
            for width in (32, 96, 256):
                for tile in (0.0, 64.0, 1e30):
                    c.set_tuning(ctas, width, tile)
                    c.launch_count()
                    assert c.read_count().triangles == want, (ctas, width, tile)
        best = c.autotune(reps=1)
        assert best.count_ms > 0 and best.piece_width in (32, 64, 128)
        t = c.tuning()
        assert (t.ctas_per_sm, t.piece_width) == (best.ctas_per_sm, best.piece_width)
        c.launch_count()
        assert c.read_count().triangles == want
        c.capture_count()
        c.launch_count()
        assert c.read_count().triangles == want
    with pytest.raises(tb.TribitError):
        with tb.Counter() as c:
            c.set_tuning(4, 48, 64.0)  # not a multiple of 32
