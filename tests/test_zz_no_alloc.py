"""tribit_count_edges_noalloc against the context entry point, on the GPU.

The no-allocation entry point exists for callers that cannot allocate device
memory while they count -- a process whose device memory is owned by a
framework allocator or by a pool reserved up front, or a loop that cannot
afford the implicit synchronisation of cudaMalloc. It takes every buffer from
a fixed 32 MiB array inside the library. These tests call it through the
C-ABI and require exactly the counts tribit_count_edges gives for the same
graphs, on two calls in a row (the second call finds the first call's data
still in the shared array), and a clean refusal for a graph that does not fit.

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import oracle
import tribit_b200 as tb

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _graphs():
    return [
        (7115, tb.gen_chung_lu(7115, 115300, 2.0, 1000.0, seed=1)),  # ~100.8k edges
        (1 << 14, tb.gen_rmat(14, 16, seed=14)),
        (5000, tb.gen_er(5000, 60000, seed=4)),
        (1 << 16, tb.gen_rmat(16, 16, seed=16)),  # ~1.05M entries: too large for the hub lists
    ]


def test_noalloc_matches_counted_entry_point_twice():
    graphs = _graphs()
    with tb.Counter() as c:
        want = [c.count_edges(e, n) for n, e in graphs]
    # The context entry point is itself pinned to the oracle; check it here too.
    assert [(w.triangles, w.edges) for w in want] == [oracle.count(e, n) for n, e in graphs]
    stream = torch.cuda.Stream()
    out = torch.empty(4, dtype=torch.int64, device="cuda")
    hub_lists = set()
    for call in range(2):
        for (n, e), w in zip(graphs, want):
            d = torch.from_numpy(e.view(np.int64)).cuda()
            out.fill_(-1)
            torch.cuda.synchronize()
            tb.count_edges_noalloc(d.data_ptr(), d.numel(), n, out.data_ptr(), stream.cuda_stream)
            stream.synchronize()
            r = out.cpu().numpy().view(np.uint64)
            assert (int(r[0]), int(r[1]), int(r[2])) == (w.triangles, w.edges, 0), (call, n)
            hub_lists.add((n, int(r[3])))
    # The small graphs run with the merge variant's hub lists, the largest without.
    assert (1 << 14, 1) in hub_lists and (1 << 16, 0) in hub_lists, hub_lists


def test_noalloc_flags_bad_ids_and_refuses_oversized_graphs():
    e = np.array([(0 << 32) | 1, (1 << 32) | 2, (2 << 32) | 9], dtype=np.uint64)
    d = torch.from_numpy(e.view(np.int64)).cuda()
    out = torch.zeros(4, dtype=torch.int64, device="cuda")
    tb.count_edges_noalloc(d.data_ptr(), d.numel(), 4, out.data_ptr(), 0)
    torch.cuda.synchronize()
    assert int(out[2].item()) & 1
    assert tb.lib.tribit_noalloc_scratch_bytes() == 32 << 20
    big = tb.gen_rmat(20, 16, seed=1)  # ~16.8M entries: far beyond 32 MiB of scratch
    d = torch.from_numpy(big.view(np.int64)).cuda()
    with pytest.raises(tb.TribitError) as ex:
        tb.count_edges_noalloc(d.data_ptr(), d.numel(), 1 << 20, out.data_ptr(), 0)
    assert ex.value.status == 6
