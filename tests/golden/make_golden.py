"""Regenerates tests/golden/known_counts.json.

Each case is a seeded synthetic graph from the tribit_b200 generators (or the
reference's bundled wiki-Vote.mtx when the reference tree is mounted) with its
exact count. Counts come from the CPU oracle (oracle/, merge intersection and
the restated reference bit-block algorithm, which must agree) and, as an
independent third method, scipy's sparse trace(A^3)/6 on the symmetrised
matrix. A case is written only when all three agree. The entry checksum pins
the generator output so that drift in a generator is caught before a count
mismatch is blamed on a kernel.

Run from the repository root: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import tribit_b200 as tb  # noqa: E402

# The committed copy of the reference's bundled wiki-Vote.mtx (sixt99/TriBIT,
# wiki-Vote.mtx at the repository root).
WIKI = os.environ.get("TRIBIT_WIKI_VOTE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "wiki-Vote.mtx"))

CASES = [
    # the small Chung-Lu graph: n=7,115, beta 2.0, max degree cap 1,000, ~100.8k edges
    {"name": "chung_lu_7115", "gen": "chung_lu", "n": 7115, "n_entries": 115300, "beta": 2.0, "max_degree": 1000.0,
     "seed": 1},
    {"name": "rmat_s10", "gen": "rmat", "scale": 10, "edge_factor": 16, "seed": 11},
    {"name": "rmat_s12", "gen": "rmat", "scale": 12, "edge_factor": 16, "seed": 12},
    {"name": "rmat_s14", "gen": "rmat", "scale": 14, "edge_factor": 16, "seed": 14},
    {"name": "rmat_s16", "gen": "rmat", "scale": 16, "edge_factor": 16, "seed": 16},
    {"name": "er_2000", "gen": "er", "n": 2000, "n_entries": 40000, "seed": 5},
    {"name": "er_50000", "gen": "er", "n": 50000, "n_entries": 800000, "seed": 6},
    {"name": "chung_lu_30000_b2.5", "gen": "chung_lu", "n": 30000, "n_entries": 300000, "beta": 2.5,
     "max_degree": 2000.0, "seed": 7},
    {"name": "planted_200x100", "gen": "planted", "communities": 200, "size": 100, "p_in": 0.3, "inter": 2,
     "seed": 8},
]


def generate(c):
    g = c["gen"]
    if g == "rmat":
        return 1 << c["scale"], tb.gen_rmat(c["scale"], c["edge_factor"], seed=c["seed"])
    if g == "er":
        return c["n"], tb.gen_er(c["n"], c["n_entries"], seed=c["seed"])
    if g == "chung_lu":
        return c["n"], tb.gen_chung_lu(c["n"], c["n_entries"], c["beta"], c["max_degree"], seed=c["seed"])
    if g == "planted":
        return c["communities"] * c["size"], tb.gen_planted(c["communities"], c["size"], c["p_in"], c["inter"],
                                                            seed=c["seed"])
    raise ValueError(g)


def checksum(entries):
    return hashlib.sha256(np.ascontiguousarray(entries, dtype=np.uint64).tobytes()).hexdigest()[:16]


def scipy_count(entries, n):
    e = oracle.fold_dedup(entries)
    a = (e >> np.uint64(32)).astype(np.int64)
    b = (e & np.uint64(0xFFFFFFFF)).astype(np.int64)
    A = sp.coo_matrix((np.ones(a.size, dtype=np.int64), (a, b)), shape=(n, n)).tocsr()
    A = A + A.T
    return int((A @ A).multiply(A).sum() // 6)


def record(name, n, entries, extra):
    t_merge, m = oracle.count(entries, n, order=1)
    t_id, _ = oracle.count(entries, n, order=0)
    t_ref, blocks = oracle.count_tribit(entries, n)
    t_sp = scipy_count(entries, n)
    assert t_merge == t_id == t_ref == t_sp, (name, t_merge, t_id, t_ref, t_sp)
    rec = {"name": name, "num_nodes": int(n), "entries": int(len(entries)), "entries_sha256_16": checksum(entries),
           "edges": m, "triangles": t_merge, "reference_blocks_of_threads": blocks}
    rec.update(extra)
    print(json.dumps(rec))
    return rec


def main():
    out = []
    for c in CASES:
        n, e = generate(c)
        out.append(record(c["name"], n, e, {"params": c}))
    if os.path.exists(WIKI):
        st, n, e = oracle.read_mtx(WIKI)
        assert st == 0
        with open(WIKI, "rb") as f:
            sha = hashlib.sha256(f.read()).hexdigest()[:16]
        out.append(record("wiki-Vote", n, e, {"params": {"file": "wiki-Vote.mtx (sixt99/TriBIT root; copy in tests/golden)", "file_sha256_16": sha}}))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_counts.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
