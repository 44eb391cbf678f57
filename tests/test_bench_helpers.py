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
