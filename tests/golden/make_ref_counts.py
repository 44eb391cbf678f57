"""Runs the reference binary (oracle/_ref/tribit_ref: sixt99/TriBIT
src/single_gpu/tribit.cu rebuilt unchanged for sm_100a by `make -C oracle ref`)
on a GPU and records what it prints into tests/golden/ref_counts.json.

Inputs are the seeded graphs of known_counts.json (written as Matrix Market
files to a scratch folder) plus any extra .mtx paths given on the command
line. For each it stores the reference's "Triangles", "Blocks of threads",
"Preprocessing (ms)" and "Kernel (ms)" lines, parsed with the regexes of the
reference's own harness (artifact/sc26/run_benchmarks/run_single_gpu.py:78-83).
The CPU tests then pin the oracle -- its merge count and its restatement of the
reference's work decomposition -- to these numbers.

  python tests/golden/make_ref_counts.py [--out FILE] [--scratch DIR] [--timeout S] [extra.mtx ...]
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import tribit_b200 as tb  # noqa: E402
from tests.golden.make_golden import CASES, generate  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "tribit_ref")
FIELDS = {
    "blocks_of_threads": r"Blocks of threads\s*:\s*(\d+)",
    "preprocessing_ms": r"Preprocessing \(ms\)\s*:\s*([\d.]+)",
    "kernel_ms": r"Kernel \(ms\)\s*:\s*([\d.]+)",
    "triangles": r"Triangles\s*:\s*(\d+)",
}
EXTRA_CASES = [
    {"name": "rmat_s18", "gen": "rmat", "scale": 18, "edge_factor": 16, "seed": 18},
    {"name": "rmat_s20", "gen": "rmat", "scale": 20, "edge_factor": 16, "seed": 20},
    {"name": "rmat_s22", "gen": "rmat", "scale": 22, "edge_factor": 16, "seed": 22},
    {"name": "planted_20000x100", "gen": "planted", "communities": 20000, "size": 100, "p_in": 0.3, "inter": 2,
     "seed": 3},
]


def run_ref(path, timeout):
    try:
        r = subprocess.run([REF, "-i", path], capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"status": "timeout"}
    rec = {"status": "ok" if r.returncode == 0 else f"exit {r.returncode}"}
    for k, rx in FIELDS.items():
        m = re.search(rx, r.stdout)
        if m:
            rec[k] = float(m.group(1)) if "ms" in k else int(m.group(1))
    if r.returncode != 0:
        rec["stderr_tail"] = r.stderr.strip().splitlines()[-3:]
    err = re.search(r"(Cuda error at .*|No cuda error detected at .*)", r.stdout)
    if err:
        rec["cuda"] = err.group(1).split(" at ")[0]
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_counts.json"))
    ap.add_argument("--scratch", default="/tmp/tribit_ref_inputs")
    ap.add_argument("--timeout", type=int, default=600)
    ap.add_argument("--extra-cases", action="store_true", help="also run the larger RMAT / planted graphs")
    ap.add_argument("mtx", nargs="*")
    args = ap.parse_args()
    if not os.access(REF, os.X_OK):
        sys.exit(f"{REF} missing: run `make -C oracle ref` where the reference tree is mounted")
    os.makedirs(args.scratch, exist_ok=True)
    out = []
    cases = CASES + (EXTRA_CASES if args.extra_cases else [])
    for c in cases:
        n, e = generate(c)
        p = os.path.join(args.scratch, c["name"] + ".mtx")
        tb.write_mtx(p, n, e)
        rec = {"name": c["name"], "params": c, **run_ref(p, args.timeout)}
        print(json.dumps(rec), flush=True)
        out.append(rec)
        os.remove(p)
    for p in args.mtx:
        with open(p, "rb") as f:
            sha = hashlib.sha256(f.read()).hexdigest()[:16]
        rec = {"name": os.path.basename(p).rsplit(".", 1)[0], "file_sha256_16": sha, **run_ref(p, args.timeout)}
        print(json.dumps(rec), flush=True)
        out.append(rec)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
