"""Small graph builders shared by the tests (entries as (a << 32) | b words)."""
import itertools

import numpy as np


def zip_pairs(pairs):
    p = np.asarray(list(pairs), dtype=np.uint64).reshape(-1, 2)
    return (p[:, 0] << np.uint64(32)) | p[:, 1]


def clique(n, base=0):
    return zip_pairs((base + i, base + j) for i, j in itertools.combinations(range(n), 2))


def wheel(n):
    """Hub 0 joined to a cycle 1..n-1: n-1 triangles for n >= 5."""
    rim = list(range(1, n))
    pairs = [(0, v) for v in rim] + [(rim[i], rim[(i + 1) % len(rim)]) for i in range(len(rim))]
    return zip_pairs(pairs)


def star(n):
    return zip_pairs((0, v) for v in range(1, n))


def comb(n):
    return n * (n - 1) * (n - 2) // 6


def numpy_count(entries, n):
    """Independent dense check: trace(A^3) / 6 on the symmetrised simple graph."""
    e = np.asarray(entries, dtype=np.uint64)
    a = (e >> np.uint64(32)).astype(np.int64)
    b = (e & np.uint64(0xFFFFFFFF)).astype(np.int64)
    keep = a != b
    A = np.zeros((n, n), dtype=np.int64)
    A[a[keep], b[keep]] = 1
    A[b[keep], a[keep]] = 1
    return int(np.trace(A @ A @ A) // 6)
