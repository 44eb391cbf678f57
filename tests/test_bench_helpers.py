"""The bench line's roofline inputs, on the CPU: the measured HBM peak and the
committed per-launch DRAM traffic of the counting kernels."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_is_read_from_the_committed_profile():
    rows = [line.split() for line in open(os.path.join(ROOT, "profiles", "traffic.txt"))
            if line.strip() and not line.startswith("#")]
    assert rows, "profiles/traffic.txt lists no workload"
    for workload, nbytes, dispatch in rows:
        assert bench.profiled_traffic(workload, dispatch) == float(nbytes)
    assert bench.profiled_traffic("rmat24", "no-such-dispatch") is None
    assert bench.profiled_traffic("no-such-workload", "learned") is None


def test_peak_is_the_measured_copy_bandwidth_when_present():
    peak, kind = bench.measured_peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        assert (peak, kind) == (json.load(open(path))["hbm_gbs"], "measured")
    else:
        assert kind == "fallback" and peak > 0


def test_reference_arm_graph_loads_no_product_code():
    # The reference arm builds its R-MAT graph with the oracle's generator, so
    # neither the product package nor its library is loaded by it.
    import subprocess
    import sys
    code = ("import sys, json; sys.path.insert(0, %r); import bench; "
            "n, e = bench.reference_graph({'gen': 'rmat', 'scale': 12, 'edge_factor': 16, 'seed': 12}); "
            "print(json.dumps([n, int(e.size), 'tribit_b200' in sys.modules, "
            "any('libtribit' in l for l in open('/proc/self/maps'))]))") % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    import json
    n, size, imported, mapped = json.loads(out.stdout.strip().splitlines()[-1])
    assert (n, size) == (1 << 12, 16 << 12) and not imported and not mapped
