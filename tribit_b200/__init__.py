"""tribit_b200 -- exact triangle counting on one NVIDIA B200 (sm_100a).

Python binding of the C-ABI in ``include/tribit.h`` (ctypes over the in-tree
``libtribit.so``). It mirrors the reference single-GPU counter of
sixt99/TriBIT: ``read_mtx`` follows ``read_mtx`` (src/single_gpu/tribit.cu:228)
and ``Counter.count_edges`` follows ``count_triangles``
(src/single_gpu/tribit.cu:656) -- same zipped (a << 32) | b input words, same
exact uint64 count -- with status codes raised as ``TribitError`` instead of
process exits.

There is no CPU fallback: importing this package without the built library
raises ImportError, and every count runs the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from dataclasses import dataclass

import numpy as np

__all__ = [
    "TribitError", "Counter", "Result", "read_mtx", "write_mtx", "gen_rmat", "gen_er",
    "gen_chung_lu", "gen_planted", "lib", "LIB_PATH", "ORDERS", "DISPATCH", "VARIANTS",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtribit.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing; build it with `make -C tribit_b200` "
        "(or __graft_entry__.build()). tribit_b200 has no CPU fallback.")

lib = ctypes.CDLL(LIB_PATH)

ORDERS = {"degree": 0, "id": 1}
DISPATCH = {"plain": 0, "learned": 1, "merge": 2, "bitmap": 3, "mma": 4}
STREAM_TIERS = {"auto": 0, "rows": 1, "pairs": 2}
VARIANTS = ("mma", "bitmap", "merge")
TILE_ENGINES = ("mma_sync", "tcgen05")
LAUNCH_MODELS = ("kernels", "queue", "auto")

_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_p = ctypes.c_void_p


class _Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("order", ctypes.c_int), ("dispatch", ctypes.c_int),
                ("ctas_per_sm", ctypes.c_int), ("reserved", _u32 * 8)]


class _Result(ctypes.Structure):
    _fields_ = [("triangles", _u64), ("num_nodes", _u64), ("entries", _u64), ("edges", _u64),
                ("blocks_of_threads", _u64), ("row_blocks", _u64), ("row_blocks_by_variant", _u64 * 3),
                ("h2d_ms", ctypes.c_float), ("preprocess_ms", ctypes.c_float), ("kernel_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("count_kernels", _u32), ("hub_edges", _u32),
                ("load_ms", ctypes.c_float), ("load_gpu_parse", _u32), ("stream_ranges", _u32),
                ("stream_tasks", _u32), ("stream_tier", _u32)]


def _decl(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_decl("tribit_default_options", None, ctypes.POINTER(_Options))
_decl("tribit_create", ctypes.c_int, ctypes.POINTER(_Options), ctypes.POINTER(_p))
_decl("tribit_destroy", None, _p)
_decl("tribit_set_stream", ctypes.c_int, _p, _p)
_decl("tribit_status_string", ctypes.c_char_p, ctypes.c_int)
_decl("tribit_last_error", ctypes.c_char_p, _p)
_decl("tribit_version", ctypes.c_char_p)
_decl("tribit_count_edges", ctypes.c_int, _p, _p, _u64, _u64, ctypes.POINTER(_Result))
_decl("tribit_set_device_budget", ctypes.c_int, _p, _u64)
_decl("tribit_set_stream_options", ctypes.c_int, _p, ctypes.c_int, _u64)
_decl("tribit_device_bytes", ctypes.c_int, _p, _u64, _u64, ctypes.POINTER(_u64))
_decl("tribit_count_edges_device", ctypes.c_int, _p, _p, _u64, _u64, ctypes.POINTER(_Result))
_decl("tribit_prepare_device", ctypes.c_int, _p, _p, _u64, _u64, ctypes.POINTER(_Result))
_decl("tribit_launch_count", ctypes.c_int, _p)
_decl("tribit_read_count", ctypes.c_int, _p, ctypes.POINTER(_Result))
_decl("tribit_read_mtx", ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_p), ctypes.POINTER(_u64))
_decl("tribit_free_host", None, _p)
_decl("tribit_read_bvgraph", ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_p),
      ctypes.POINTER(_u64))
_decl("tribit_count_bvgraph", ctypes.c_int, _p, ctypes.c_char_p, ctypes.POINTER(_Result))
_decl("tribit_count_mtx", ctypes.c_int, _p, ctypes.c_char_p, ctypes.POINTER(_Result))
_decl("tribit_load_mtx", ctypes.c_int, _p, ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_u64))
_decl("tribit_count_loaded", ctypes.c_int, _p, ctypes.POINTER(_Result))
_decl("tribit_loaded_entries", ctypes.c_int, _p, _p, _u64, ctypes.POINTER(_u64))
_decl("tribit_count_batch", ctypes.c_int, _p, _p, _p, _p, _u32, _p, ctypes.POINTER(_Result))
_decl("tribit_model_load", ctypes.c_int, _p, ctypes.c_char_p)
_decl("tribit_model_save", ctypes.c_int, _p, ctypes.c_char_p)
_decl("tribit_model_num_params", _u32)
_decl("tribit_model_init", ctypes.c_int, _p, _u64, _p)
_decl("tribit_model_get_params", ctypes.c_int, _p, _p, ctypes.c_int)
_decl("tribit_model_set_params", ctypes.c_int, _p, _p)
_decl("tribit_model_predict", ctypes.c_int, _p, _p, _u64, _p)
_decl("tribit_model_gradients", ctypes.c_int, _p, _p, _p, _u64, _p, ctypes.POINTER(ctypes.c_float))
_decl("tribit_model_train", ctypes.c_int, _p, _p, _p, _u64, _u32, _u32, ctypes.c_float, _u64,
      ctypes.POINTER(ctypes.c_float))
_decl("tribit_block_features", ctypes.c_int, _p, _p, _u64, ctypes.POINTER(_u64))
_decl("tribit_block_variants", ctypes.c_int, _p, _p, _u64, ctypes.POINTER(_u64))
_decl("tribit_block_times", ctypes.c_int, _p, ctypes.c_int, _p, _u64, ctypes.POINTER(_u64),
      ctypes.POINTER(ctypes.c_float))
class Tuning(ctypes.Structure):
    """tribit_tuning: launch parameters of the counting kernels."""
    _fields_ = [("ctas_per_sm", ctypes.c_int), ("piece_width", _u32), ("tile_min_nnz", ctypes.c_float),
                ("count_ms", ctypes.c_float), ("merge_ratio", ctypes.c_float), ("launch_model", _u32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_decl("tribit_get_tuning", ctypes.c_int, _p, ctypes.POINTER(Tuning))
_decl("tribit_set_tuning", ctypes.c_int, _p, ctypes.POINTER(Tuning))
_decl("tribit_autotune", ctypes.c_int, _p, _u32, ctypes.POINTER(Tuning))
_decl("tribit_set_tile_engine", ctypes.c_int, _p, ctypes.c_int)
_decl("tribit_test_tile_timeout", ctypes.c_int, _p, _u32)
_decl("tribit_set_tile_wait_polls", ctypes.c_int, _p, _u32)
_decl("tribit_capture_count", ctypes.c_int, _p)
_decl("tribit_read_batch_counts", ctypes.c_int, _p, _p, _u32)
_decl("tribit_gen_batch", ctypes.c_int, _u32, _u32, _u32, _u64, _p, _p, _p)
_decl("tribit_count_edges_noalloc", ctypes.c_int, _p, _u64, _u64, _p, _p)
_decl("tribit_noalloc_scratch_bytes", _u64)
_decl("tribit_gen_rmat", ctypes.c_int, ctypes.c_int, _u64, ctypes.c_double, ctypes.c_double, ctypes.c_double, _u64, _p)
_decl("tribit_gen_er", ctypes.c_int, _u32, _u64, _u64, _p)
_decl("tribit_gen_chung_lu", ctypes.c_int, _u32, _u64, ctypes.c_double, ctypes.c_double, _u64, _p)
_decl("tribit_gen_planted", ctypes.c_int, _u32, _u32, ctypes.c_double, _u32, _u64, _p, ctypes.POINTER(_u64))
_decl("tribit_write_mtx", ctypes.c_int, ctypes.c_char_p, _u64, _p, _u64)


class TribitError(RuntimeError):
    """A non-zero tribit_status from the C-ABI."""

    def __init__(self, status: int, detail: str = ""):
        self.status = status
        msg = lib.tribit_status_string(status).decode()
        super().__init__(f"{msg} (status {status})" + (f": {detail}" if detail else ""))


def _check(st: int, ctx=None):
    if st != 0:
        detail = lib.tribit_last_error(ctx).decode() if ctx else ""
        raise TribitError(st, detail)


@dataclass
class Result:
    triangles: int
    num_nodes: int
    entries: int
    edges: int
    blocks_of_threads: int
    row_blocks: int
    row_blocks_by_variant: tuple
    h2d_ms: float
    preprocess_ms: float
    kernel_ms: float
    total_ms: float
    count_kernels: int
    hub_edges: int
    load_ms: float = 0.0
    load_gpu_parse: int = 0
    stream_ranges: int = 0
    stream_tasks: int = 0
    stream_tier: int = 0

    @classmethod
    def _from(cls, r: _Result) -> "Result":
        return cls(r.triangles, r.num_nodes, r.entries, r.edges, r.blocks_of_threads, r.row_blocks,
                   tuple(r.row_blocks_by_variant), r.h2d_ms, r.preprocess_ms, r.kernel_ms, r.total_ms,
                   r.count_kernels, r.hub_edges, r.load_ms, r.load_gpu_parse, r.stream_ranges, r.stream_tasks,
                   r.stream_tier)


def _entries(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a


class Counter:
    """A tribit context on one CUDA device (tribit_create / tribit_destroy)."""

    def __init__(self, device: int = 0, order: str = "degree", dispatch: str = "plain", ctas_per_sm: int = 0):
        o = _Options()
        lib.tribit_default_options(ctypes.byref(o))
        o.device = device
        o.order = ORDERS[order]
        o.dispatch = DISPATCH[dispatch]
        o.ctas_per_sm = ctas_per_sm
        h = _p()
        _check(lib.tribit_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.tribit_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        _check(lib.tribit_set_stream(self._h, stream_ptr or None), self._h)

    def load_model(self, path: str):
        _check(lib.tribit_model_load(self._h, path.encode()), self._h)

    # -- tuning and CUDA-graph replay ----------------------------------------
    def tuning(self) -> Tuning:
        t = Tuning()
        _check(lib.tribit_get_tuning(self._h, ctypes.byref(t)), self._h)
        return t

    def set_tuning(self, ctas_per_sm: int = 0, piece_width: int = 64, tile_min_nnz: float = 64.0,
                   merge_ratio: float | None = None, launch_model: str | None = None):
        """merge_ratio / launch_model None keep the context's current plain-rule
        merge threshold / launch model ("kernels", "queue" or "auto")."""
        cur = self.tuning()
        if merge_ratio is None:
            merge_ratio = cur.merge_ratio
        model = cur.launch_model if launch_model is None else LAUNCH_MODELS.index(launch_model)
        t = Tuning(ctas_per_sm, piece_width, tile_min_nnz, 0.0, merge_ratio, model)
        _check(lib.tribit_set_tuning(self._h, ctypes.byref(t)), self._h)

    def set_tile_engine(self, engine: str):
        """Arithmetic of the bit-tile variant: "mma_sync" (b1 AND+POPC) or "tcgen05" (kind::i8)."""
        _check(lib.tribit_set_tile_engine(self._h, TILE_ENGINES.index(engine)), self._h)

    def set_tile_wait_polls(self, max_polls: int):
        """Poll budget of the tcgen05 tiles' bounded wait (0 = default); a
        launch whose wait runs out reports TRIBIT_ERR_TIMEOUT, never a wrong count."""
        _check(lib.tribit_set_tile_wait_polls(self._h, max_polls), self._h)

    def autotune(self, reps: int = 2) -> Tuning:
        t = Tuning()
        _check(lib.tribit_autotune(self._h, reps, ctypes.byref(t)), self._h)
        return t

    def capture_count(self):
        _check(lib.tribit_capture_count(self._h), self._h)

    def batch_counts(self, num_graphs: int) -> np.ndarray:
        out = np.zeros(num_graphs, dtype=np.uint64)
        _check(lib.tribit_read_batch_counts(self._h, out.ctypes.data, num_graphs), self._h)
        return out

    # -- learned dispatcher ------------------------------------------------
    def model_init(self, norm, seed: int = 1):
        nrm = np.ascontiguousarray(norm, dtype=np.float32)
        assert nrm.size == 38
        _check(lib.tribit_model_init(self._h, seed, nrm.ctypes.data), self._h)

    def save_model(self, path: str):
        _check(lib.tribit_model_save(self._h, path.encode()), self._h)

    def model_params(self, effective: bool = False) -> np.ndarray:
        out = np.zeros(lib.tribit_model_num_params(), dtype=np.float32)
        _check(lib.tribit_model_get_params(self._h, out.ctypes.data, int(effective)), self._h)
        return out

    def set_model_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib.tribit_model_set_params(self._h, p.ctypes.data), self._h)

    def model_predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 16)
        y = np.zeros((x.shape[0], 3), dtype=np.float32)
        _check(lib.tribit_model_predict(self._h, x.ctypes.data, x.shape[0], y.ctypes.data), self._h)
        return y

    def model_gradients(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 16)
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1, 3)
        g = np.zeros(lib.tribit_model_num_params(), dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib.tribit_model_gradients(self._h, x.ctypes.data, y.ctypes.data, x.shape[0], g.ctypes.data,
                                          ctypes.byref(loss)), self._h)
        return g, loss.value

    def model_train(self, x, y, epochs: int = 10, batch: int = 4096, lr: float = 1e-3, seed: int = 1) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 16)
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1, 3)
        loss = ctypes.c_float()
        _check(lib.tribit_model_train(self._h, x.ctypes.data, y.ctypes.data, x.shape[0], epochs, batch, lr, seed,
                                      ctypes.byref(loss)), self._h)
        return loss.value

    def block_features(self) -> np.ndarray:
        nrb = _u64()
        _check(lib.tribit_block_features(self._h, None, 0, ctypes.byref(nrb)), self._h)
        out = np.zeros((nrb.value, 16), dtype=np.float32)
        _check(lib.tribit_block_features(self._h, out.ctypes.data, out.size, ctypes.byref(nrb)), self._h)
        return out

    def block_variants(self) -> np.ndarray:
        """The dispatcher's variant index (see VARIANTS) of every 32-row block."""
        nrb = _u64()
        _check(lib.tribit_block_variants(self._h, None, 0, ctypes.byref(nrb)), self._h)
        out = np.zeros(nrb.value, dtype=np.uint8)
        _check(lib.tribit_block_variants(self._h, out.ctypes.data, out.size, ctypes.byref(nrb)), self._h)
        return out

    def block_times(self, variant: str):
        nrb = _u64()
        _check(lib.tribit_block_features(self._h, None, 0, ctypes.byref(nrb)), self._h)
        out = np.zeros(nrb.value, dtype=np.float32)
        tri = _u64()
        ms = ctypes.c_float()
        _check(lib.tribit_block_times(self._h, VARIANTS.index(variant), out.ctypes.data, out.size,
                                      ctypes.byref(tri), ctypes.byref(ms)), self._h)
        return out, tri.value, ms.value

    def count_edges(self, entries, num_nodes: int) -> Result:
        e = _entries(entries)
        r = _Result()
        _check(lib.tribit_count_edges(self._h, e.ctypes.data, e.size, int(num_nodes), ctypes.byref(r)), self._h)
        return Result._from(r)

    def set_device_budget(self, nbytes: int):
        """Device memory later count_edges calls may use (0 = what is free); a
        graph needing more is counted in rank ranges (Result.stream_ranges > 1)."""
        _check(lib.tribit_set_device_budget(self._h, int(nbytes)), self._h)

    def set_stream_options(self, tier: str = "auto", range_entries: int = 0):
        """How a count past the device budget runs: "rows" builds the oriented
        rows one rank range at a time and counts them once, "pairs" counts each
        pair of ranges as its own graph, "auto" takes rows when they fit.
        range_entries bounds a range's oriented entries (0: the budget's)."""
        _check(lib.tribit_set_stream_options(self._h, STREAM_TIERS[tier], int(range_entries)), self._h)

    def device_bytes(self, n_entries: int, num_nodes: int) -> int:
        """Device memory a one-piece count_edges of this size takes."""
        b = _u64()
        _check(lib.tribit_device_bytes(self._h, int(n_entries), int(num_nodes), ctypes.byref(b)), self._h)
        return b.value

    def count_edges_device(self, ptr: int, n_entries: int, num_nodes: int) -> Result:
        r = _Result()
        _check(lib.tribit_count_edges_device(self._h, ptr, n_entries, int(num_nodes), ctypes.byref(r)), self._h)
        return Result._from(r)

    def prepare_device(self, ptr: int, n_entries: int, num_nodes: int) -> Result:
        r = _Result()
        _check(lib.tribit_prepare_device(self._h, ptr, n_entries, int(num_nodes), ctypes.byref(r)), self._h)
        return Result._from(r)

    def launch_count(self):
        _check(lib.tribit_launch_count(self._h), self._h)

    def read_count(self) -> Result:
        r = _Result()
        _check(lib.tribit_read_count(self._h, ctypes.byref(r)), self._h)
        return Result._from(r)

    def count_mtx(self, path: str) -> Result:
        r = _Result()
        _check(lib.tribit_count_mtx(self._h, path.encode(), ctypes.byref(r)), self._h)
        return Result._from(r)

    def load_mtx(self, path: str):
        """tribit_load_mtx: the file parsed into device memory -> (num_nodes, entries)."""
        n, e = _u64(), _u64()
        _check(lib.tribit_load_mtx(self._h, str(path).encode(), ctypes.byref(n), ctypes.byref(e)), self._h)
        return n.value, e.value

    def count_loaded(self) -> Result:
        r = _Result()
        _check(lib.tribit_count_loaded(self._h, ctypes.byref(r)), self._h)
        return Result._from(r)

    def loaded_entries(self) -> np.ndarray:
        cnt = _u64()
        _check(lib.tribit_loaded_entries(self._h, None, 0, ctypes.byref(cnt)), self._h)
        out = np.zeros(cnt.value, dtype=np.uint64)
        _check(lib.tribit_loaded_entries(self._h, out.ctypes.data if out.size else None, out.size,
                                         ctypes.byref(cnt)), self._h)
        return out

    def count_bvgraph(self, basename: str) -> Result:
        r = _Result()
        _check(lib.tribit_count_bvgraph(self._h, str(basename).encode(), ctypes.byref(r)), self._h)
        return Result._from(r)

    def count_batch(self, entries, offsets, num_nodes):
        """Counts len(num_nodes) graphs in one launch; returns (counts, Result)."""
        e = _entries(entries)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nn = np.ascontiguousarray(num_nodes, dtype=np.uint32)
        g = nn.size
        if off.size != g + 1:
            raise ValueError("offsets must have len(num_nodes) + 1 entries")
        out = np.zeros(g, dtype=np.uint64)
        r = _Result()
        _check(lib.tribit_count_batch(self._h, e.ctypes.data if e.size else None, off.ctypes.data, nn.ctypes.data, g,
                                      out.ctypes.data, ctypes.byref(r)), self._h)
        return out, Result._from(r)


def count_edges_noalloc(entries_ptr: int, n_entries: int, num_nodes: int, result_ptr: int, stream_ptr: int = 0):
    """tribit_count_edges_noalloc: counts the graph at device address entries_ptr
    without allocating anything, for callers whose device memory is owned by
    someone else (a framework allocator or a pool reserved up front) or who
    cannot afford cudaMalloc's implicit synchronisation. All scratch comes
    from one fixed 32 MiB device array inside the library. Asynchronous on
    stream_ptr: result_ptr (4 x uint64 in device memory) receives
    [triangles, edges, error flags, 0]. Raises TribitError (status 6) for a
    graph too large for the scratch array."""
    _check(lib.tribit_count_edges_noalloc(entries_ptr, n_entries, int(num_nodes), result_ptr, stream_ptr or None))


def read_mtx(path: str):
    """Reads a Matrix Market file with the reference's semantics -> (num_nodes, entries)."""
    n = _u64()
    ptr = _p()
    cnt = _u64()
    _check(lib.tribit_read_mtx(str(path).encode(), ctypes.byref(n), ctypes.byref(ptr), ctypes.byref(cnt)))
    # The entries stay in the library's buffer (no copy); it is freed with the
    # array (views keep the array, and so the buffer, alive).
    addr = ptr.value
    try:
        buf = (ctypes.c_uint64 * max(cnt.value, 1)).from_address(addr)
        arr = np.frombuffer(buf, dtype=np.uint64, count=cnt.value)
        weakref.finalize(arr, lib.tribit_free_host, ctypes.c_void_p(addr))
    except BaseException:
        lib.tribit_free_host(ctypes.c_void_p(addr))
        raise
    return n.value, arr


def _host_words(ptr: int, count: int) -> np.ndarray:
    """The library's malloc'd entry buffer as an array (freed with the array)."""
    try:
        buf = (ctypes.c_uint64 * max(count, 1)).from_address(ptr)
        arr = np.frombuffer(buf, dtype=np.uint64, count=count)
        weakref.finalize(arr, lib.tribit_free_host, ctypes.c_void_p(ptr))
    except BaseException:
        lib.tribit_free_host(ctypes.c_void_p(ptr))
        raise
    return arr


def read_bvgraph(basename: str):
    """Reads a WebGraph BVGraph (basename.properties / .graph / .offsets) -> (num_nodes, entries)."""
    n = _u64()
    ptr = _p()
    cnt = _u64()
    _check(lib.tribit_read_bvgraph(str(basename).encode(), ctypes.byref(n), ctypes.byref(ptr), ctypes.byref(cnt)))
    return n.value, _host_words(ptr.value, cnt.value)


def write_mtx(path: str, num_nodes: int, entries):
    e = _entries(entries)
    _check(lib.tribit_write_mtx(str(path).encode(), num_nodes, e.ctypes.data, e.size))


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1) -> np.ndarray:
    out = np.empty(edge_factor << scale, dtype=np.uint64)
    _check(lib.tribit_gen_rmat(scale, edge_factor, a, b, c, seed, out.ctypes.data))
    return out


def gen_er(n: int, n_entries: int, seed: int = 1) -> np.ndarray:
    out = np.empty(n_entries, dtype=np.uint64)
    _check(lib.tribit_gen_er(n, n_entries, seed, out.ctypes.data))
    return out


def gen_chung_lu(n: int, n_entries: int, beta: float, max_degree: float, seed: int = 1) -> np.ndarray:
    out = np.empty(n_entries, dtype=np.uint64)
    _check(lib.tribit_gen_chung_lu(n, n_entries, beta, max_degree, seed, out.ctypes.data))
    return out


def gen_batch(num_graphs: int, seed: int = 1, min_n: int = 64, max_n: int = 65536):
    """The batched workload -> (entries, entry_offsets, num_nodes)."""
    nn = np.zeros(num_graphs, dtype=np.uint32)
    off = np.zeros(num_graphs + 1, dtype=np.uint64)
    _check(lib.tribit_gen_batch(num_graphs, min_n, max_n, seed, nn.ctypes.data, off.ctypes.data, None))
    e = np.empty(int(off[-1]), dtype=np.uint64)
    _check(lib.tribit_gen_batch(num_graphs, min_n, max_n, seed, nn.ctypes.data, off.ctypes.data, e.ctypes.data))
    return e, off, nn


def gen_planted(communities: int, size: int, p_in: float, inter_per_vertex: int, seed: int = 1) -> np.ndarray:
    cnt = _u64(0)
    _check(lib.tribit_gen_planted(communities, size, p_in, inter_per_vertex, seed, None, ctypes.byref(cnt)))
    out = np.empty(cnt.value, dtype=np.uint64)
    _check(lib.tribit_gen_planted(communities, size, p_in, inter_per_vertex, seed, out.ctypes.data, ctypes.byref(cnt)))
    return out
