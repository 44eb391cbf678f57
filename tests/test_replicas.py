"""Multi-GPU runs are replicas: every rank counts its own seeded graph with no
data-path collective, and the bench reduces only the job totals (edges summed,
time maxed over ranks). These tests run the rank logic as world-size-2 gloo
process groups on the CPU."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r counted 1000 + r edges in 2 + r seconds.
        edges, secs = bench.reduce_replicas(dist, 1000 + rank, 2.0 + rank, "cpu")
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"edges": edges, "seconds": secs}, f)
    finally:
        dist.destroy_process_group()


def test_reduce_replicas_sums_edges_and_takes_slowest_rank(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        got = json.load(open(tmp_path / f"rank{r}.json"))
        assert got == {"edges": 2001, "seconds": 3.0}


def test_reduce_replicas_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_replicas(None, 17, 1.5, "cpu") == (17, 1.5)


def test_replica_graphs_differ_per_rank_but_keep_the_workload_size():
    sys.path.insert(0, ROOT)
    import bench
    import tribit_b200 as tb
    spec = dict(bench.WORKLOADS["chung_lu"])
    n0, e0 = bench.make_graph(tb, spec, 0)
    n1, e1 = bench.make_graph(tb, spec, 1)
    assert n0 == n1 and e0.size == e1.size
    assert not np.array_equal(e0, e1)
    n0b, e0b = bench.make_graph(tb, spec, 0)
    assert np.array_equal(e0, e0b)


def test_reference_arm_prints_once_under_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--workload", "chung_lu", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["unit"] == "edges/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
