"""CPU oracle for exact triangle counting -- TEST INFRASTRUCTURE ONLY.

ctypes binding of ``oracle/oracle.c`` (see ``oracle.h`` for what each function
restates from the reference, sixt99/TriBIT src/single_gpu/tribit.cu). Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it,
and only as the checker; the product (``tribit_b200``) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


if not os.path.exists(_SO):
    build()

_lib = ctypes.CDLL(_SO)
_u64 = ctypes.c_uint64
_p = ctypes.c_void_p


class _CSR(ctypes.Structure):
    _fields_ = [("n", _u64), ("m", _u64), ("row_ptr", ctypes.POINTER(_u64)), ("col", ctypes.POINTER(ctypes.c_uint32))]


def _decl(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)


_decl("oracle_read_mtx", ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_p), ctypes.POINTER(_u64))
_decl("oracle_free", None, _p)
_decl("oracle_fold_dedup", _u64, _p, _u64)
_decl("oracle_csr_build", ctypes.c_int, _p, _u64, _u64, ctypes.c_int, ctypes.POINTER(_CSR))
_decl("oracle_csr_free", None, ctypes.POINTER(_CSR))
_decl("oracle_count_csr", _u64, ctypes.POINTER(_CSR), ctypes.c_int, ctypes.POINTER(ctypes.c_double))
_decl("oracle_count_csr_sample", _u64, ctypes.POINTER(_CSR), ctypes.c_int, _u64, _u64, ctypes.POINTER(ctypes.c_double))
_decl("oracle_count_rows", None, ctypes.POINTER(_CSR), _p)
_decl("oracle_count_entries", _u64, _p, _u64, _u64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_u64))
_decl("oracle_count_tribit", _u64, _p, _u64, _u64, ctypes.POINTER(_u64))
_decl("oracle_write_mtx", ctypes.c_int, ctypes.c_char_p, _u64, _p, _u64)
_decl("oracle_gen_rmat", ctypes.c_int, ctypes.c_int, _u64, ctypes.c_double, ctypes.c_double, ctypes.c_double, _u64,
      ctypes.c_int, _p)


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def read_mtx(path):
    """Restatement of read_mtx (tribit.cu:228-269) -> (status, num_nodes, entries)."""
    n = _u64()
    p = _p()
    c = _u64()
    st = _lib.oracle_read_mtx(str(path).encode(), ctypes.byref(n), ctypes.byref(p), ctypes.byref(c))
    if st != 0:
        return st, 0, np.zeros(0, dtype=np.uint64)
    buf = (ctypes.c_uint64 * max(c.value, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=np.uint64, count=c.value).copy()
    _lib.oracle_free(p)
    return 0, n.value, arr


def fold_dedup(entries) -> np.ndarray:
    e = _arr(entries).copy()
    m = _lib.oracle_fold_dedup(e.ctypes.data, e.size)
    return e[:m].copy()


def count(entries, num_nodes: int, order: int = 1, threads: int = 8):
    """Merge-intersection count -> (triangles, undirected edges)."""
    e = _arr(entries)
    m = _u64()
    t = _lib.oracle_count_entries(e.ctypes.data, e.size, num_nodes, order, threads, ctypes.byref(m))
    return int(t), int(m.value)


def count_tribit(entries, num_nodes: int):
    """The reference's own L/U bit-block algorithm -> (triangles, blocks_of_threads)."""
    e = _arr(entries)
    b = _u64()
    t = _lib.oracle_count_tribit(e.ctypes.data, e.size, num_nodes, ctypes.byref(b))
    return int(t), int(b.value)


class CSR:
    """Oriented CSR of a folded, deduplicated edge list (order 0 id, 1 degree)."""

    def __init__(self, entries, num_nodes: int, order: int = 1):
        edges = fold_dedup(entries)
        self._g = _CSR()
        st = _lib.oracle_csr_build(edges.ctypes.data, edges.size, num_nodes, order, ctypes.byref(self._g))
        if st != 0:
            raise MemoryError("oracle CSR build failed")
        self.n = int(self._g.n)
        self.m = int(self._g.m)

    def count(self, threads: int = 8):
        """-> (triangles, wall seconds) over `threads` host threads."""
        s = ctypes.c_double()
        t = _lib.oracle_count_csr(ctypes.byref(self._g), threads, ctypes.byref(s))
        return int(t), s.value

    def count_sample(self, threads: int, stride: int, offset: int = 0):
        """Triangles whose lowest vertex lies in 32-row blocks b % stride == offset -> (count, seconds)."""
        s = ctypes.c_double()
        t = _lib.oracle_count_csr_sample(ctypes.byref(self._g), threads, stride, offset, ctypes.byref(s))
        return int(t), s.value

    def work(self) -> int:
        """W = sum over oriented edges (u, v) of d+(u) + d+(v): the element
        reads of a sorted-merge count on this CSR."""
        if self.m == 0:
            return 0
        rp = np.ctypeslib.as_array(self._g.row_ptr, shape=(self.n + 1,))
        col = np.ctypeslib.as_array(self._g.col, shape=(self.m,))
        d = np.diff(rp).astype(np.uint64)
        return int((d * d).sum() + d[col].sum())

    def row_counts(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.uint64)
        _lib.oracle_count_rows(ctypes.byref(self._g), out.ctypes.data)
        return out

    def close(self):
        if getattr(self, "_g", None) is not None:
            _lib.oracle_csr_free(ctypes.byref(self._g))
            self._g = None

    __del__ = close


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
             threads: int | None = None) -> np.ndarray:
    """Seeded R-MAT entries, identical to tribit_b200.gen_rmat, without the product library."""
    if threads is None:
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    out = np.empty(edge_factor << scale, dtype=np.uint64)
    st = _lib.oracle_gen_rmat(scale, edge_factor, a, b, c, seed, threads, out.ctypes.data)
    if st != 0:
        raise ValueError(f"oracle_gen_rmat failed with status {st}")
    return out


def write_mtx(path, num_nodes: int, entries):
    """Entries -> symmetric pattern .mtx (the reference binary's input format)."""
    e = _arr(entries)
    st = _lib.oracle_write_mtx(str(path).encode(), num_nodes, e.ctypes.data, e.size)
    if st != 0:
        raise OSError(f"oracle_write_mtx({path}) failed with status {st}")
