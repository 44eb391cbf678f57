"""The launch-timing loop the profiles cite (python -m tribit_b200.measure):
its named workloads on the CPU, one short run of the module on the GPU."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from tribit_b200 import measure

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_named_workloads_are_seeded_and_sized():
    n, e = measure.workload("c1", 0, 0)
    assert n == 7115 and e.dtype == np.uint64 and e.size == 115300
    n2, e2 = measure.workload("c1", 0, 0)
    assert np.array_equal(e, e2)
    n, e = measure.workload("rmat", 10, 3)
    assert n == 1 << 10 and e.size == 16 << 10
    assert int((e >> np.uint64(32)).max()) < n and int((e & np.uint64(0xFFFFFFFF)).max()) < n
    with pytest.raises(ValueError):
        measure.workload("nope", 10, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["kernels", "queue"])
def test_module_counts_and_times(model):
    out = subprocess.run([sys.executable, "-m", "tribit_b200.measure", "--scale", "12", "--seed", "5", "--steps", "2",
                          "--launch-model", model, "--dispatch", "plain"],
                         cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    n, e = measure.workload("rmat", 12, 5)
    assert line["triangles"] == oracle.count(e, n)[0]
    assert line["count_ms"] > 0 and line["prep_ms"] > 0 and line["launch_model"] == model
