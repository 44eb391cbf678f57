"""The learned dispatcher's GPU kernels (tribit_model_*) against the CPU float64
restatement in oracle/mlp.py, and exactness of counts under learned dispatch."""
import numpy as np
import pytest

import oracle
from oracle import mlp
import tribit_b200 as tb

pytestmark = pytest.mark.gpu


def _data(rows, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, 16)).astype(np.float32) * rng.uniform(0.5, 4, size=16).astype(np.float32) + 3
    y = np.stack([x[:, 0] + 0.5 * x[:, 1], np.abs(x[:, 2]) * 0.7 - x[:, 3], x[:, 4] * x[:, 5] * 0.1], 1)
    return x, (y + 10).astype(np.float32)


def _norm(x, y):
    return np.concatenate([x.mean(0), x.std(0) + 1e-3, y.mean(0), y.std(0) + 1e-3]).astype(np.float32)


def test_gradients_match_cpu_float64():
    x, y = _data(700)
    with tb.Counter() as c:
        c.model_init(_norm(x, y), seed=3)
        p = c.model_params(effective=True)
        # BF16 weights: every weight the kernels use is representable in BF16
        w = np.concatenate([p[:1024], p[1088:5184], p[5248:5440]])
        assert np.array_equal(w, (w.view(np.uint32) & 0xFFFF0000).view(np.float32))
        g, loss = c.model_gradients(x, y)
        _, want_loss, want = mlp.forward_backward(p, _norm(x, y), x, y)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    scale = np.abs(want).max()
    assert np.abs(g - want).max() <= 1e-4 * scale, np.abs(g - want).max() / scale
    # per-block relative agreement where gradients are not tiny
    big = np.abs(want) > 1e-3 * scale
    assert np.median(np.abs(g[big] - want[big]) / np.abs(want[big])) < 1e-4


def test_predictions_match_cpu():
    x, y = _data(300, seed=1)
    with tb.Counter() as c:
        c.model_init(_norm(x, y), seed=5)
        got = c.model_predict(x)
        want = mlp.predict(c.model_params(effective=True), _norm(x, y), x)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4)


def test_training_reduces_loss_and_save_load_roundtrip(tmp_path):
    x, y = _data(20000, seed=2)
    with tb.Counter() as c:
        c.model_init(_norm(x, y), seed=7)
        _, loss0 = c.model_gradients(x, y)
        loss = c.model_train(x, y, epochs=25, batch=1024, lr=3e-3, seed=1)
        _, loss1 = c.model_gradients(x, y)
        assert loss1 < 0.15 * loss0, (loss0, loss1)
        assert abs(loss - loss1) < 0.5 * loss0
        path = str(tmp_path / "m.bin")
        c.save_model(path)
        pred = c.model_predict(x[:100])
    with tb.Counter() as c2:
        c2.load_model(path)
        np.testing.assert_array_equal(c2.model_predict(x[:100]), pred)


def test_learned_dispatch_without_model_is_an_error():
    with tb.Counter(dispatch="learned") as c:
        with pytest.raises(tb.TribitError) as ex:
            c.count_edges(tb.gen_rmat(10, 8, seed=1), 1 << 10)
        assert ex.value.status == 11


def test_learned_dispatch_counts_exactly():
    graphs = [(1 << 14, tb.gen_rmat(14, 16, seed=41)), (7115, tb.gen_chung_lu(7115, 115300, 2.0, 1000.0, seed=1)),
              (20000, tb.gen_planted(200, 100, 0.3, 2, seed=8))]
    rng = np.random.default_rng(0)
    for seed in (1, 2, 3):
        with tb.Counter(dispatch="learned") as c:
            norm = np.concatenate([np.zeros(16), np.ones(16), np.zeros(3), np.ones(3)]).astype(np.float32)
            c.model_init(norm, seed=seed)
            p = c.model_params()
            p[5440:5443] = rng.normal(size=3)  # push the argmin around
            c.set_model_params(p)
            for n, e in graphs:
                assert c.count_edges(e, n).triangles == oracle.count(e, n)[0]


def test_learned_dispatch_keeps_bit_tiles_to_blocks_that_fit_one_tile():
    # A network that rates bit tiles cheapest everywhere may still only send
    # the row blocks whose columns span 1..64 blocks to them.
    import torch
    e = tb.gen_rmat(15, 16, seed=43)
    n = 1 << 15
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter(dispatch="learned") as c:
        norm = np.concatenate([np.zeros(16), np.ones(16), np.zeros(3), np.ones(3)]).astype(np.float32)
        c.model_init(norm, seed=1)
        p = c.model_params()
        p[5440:5443] = [-1e4, 0.0, 1e4]  # predicted: MMA cheapest, then bitmap
        c.set_model_params(p)
        r = c.prepare_device(d.data_ptr(), d.numel(), n)
        span = np.exp2(c.block_features()[:, 13]) - 1
        eligible = int(((span > 0.5) & (span <= 64.5)).sum())
        mma, bitmap, merge = r.row_blocks_by_variant
        assert 0 < mma <= eligible and merge == 0 and bitmap > 0
        c.launch_count()
        assert c.read_count().triangles == oracle.count(e, n)[0]


def test_block_features_and_times():
    import torch
    e = tb.gen_rmat(16, 16, seed=9)
    n = 1 << 16
    want = oracle.count(e, n)[0]
    d = torch.from_numpy(e.view(np.int64)).cuda()
    with tb.Counter() as c:
        c.prepare_device(d.data_ptr(), d.numel(), n)
        f = c.block_features()
        assert f.shape == ((n + 31) // 32, 16) and np.isfinite(f).all()
        for v in tb.VARIANTS:
            t, tri, ms = c.block_times(v)
            assert tri == want and ms > 0
            assert t.shape[0] == f.shape[0] and (t >= 0).all() and t.sum() > 0
        c.launch_count()
        assert c.read_count().triangles == want
