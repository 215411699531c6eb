"""jupiter_b200 -- B200-native subgraph-pattern counting behind a plain C-ABI.

The compute lives in ``libjgpm.so`` (hand-written CUDA for sm_100a, built in-tree by
``jupiter_b200.build``); this module is a thin ctypes host layer that mirrors the
reference's operator surface:

* ``Graph.load(prefix, use_dag)``   -- Graph::Graph(prefix, use_dag) (include/graph.h:41-42)
* ``Graph.count(pattern, ...)``     -- SubgraphSolver's pattern dispatch, round loop and
                                       count reduction (src/jupiter_gpm.cu:356-908)
* ``setop(...)`` / ``setop_batch``  -- the intersect / difference templates
                                       (include/set_intersect.cuh, include/set_difference.cuh)
* ``setop_split(...)``              -- the fused splits fuse_set / dif_int_set
                                       (include/set_difference.cuh:248-475)
* ``solve(prefix, pattern, rounds)`` -- the CLI `jupiter_gpm <graph> <pattern> [rounds]`
                                       (src/main.cc:7-47), printing the same result line.

There is no CPU fallback: importing works without a GPU (so the library can be inspected),
but every compute call raises ``JgpmError`` when the library or a CUDA device is missing.
"""
import ctypes
import os
import time

import numpy as np

__all__ = [
    "JgpmError", "Graph", "setop", "setop_batch", "setop_split", "setop_split_batch",
    "solve", "lib", "library_path",
    "OP_INTERSECT", "OP_INTERSECT_COUNT", "OP_DIFFERENCE", "OP_DIFFERENCE_COUNT",
    "SPLIT_FUSE", "SPLIT_DIF_INT",
    "COUNT_STATS", "COUNT_FORCE_PLAN", "COUNT_FORCE_ENUM", "STATUS", "batch_count",
    "autotune", "Tuning", "Server",
]

_PKG = os.path.dirname(os.path.abspath(__file__))

OP_INTERSECT, OP_INTERSECT_COUNT, OP_DIFFERENCE, OP_DIFFERENCE_COUNT = 0, 1, 2, 3
SPLIT_FUSE, SPLIT_DIF_INT = 0, 1
COUNT_STATS, COUNT_FORCE_PLAN, COUNT_FORCE_ENUM = 1, 2, 4

STATUS = {
    0: "JGPM_OK", -1: "JGPM_EINVAL", -2: "JGPM_ENOMEM", -3: "JGPM_ECUDA", -4: "JGPM_EIO",
    -5: "JGPM_EPATTERN", -6: "JGPM_ETIMEDOUT", -7: "JGPM_EOVERFLOW", -8: "JGPM_ENODEV",
    -9: "JGPM_EBUSY", -10: "JGPM_ECAPACITY", -11: "JGPM_EADMISSION", -12: "JGPM_ENOTFOUND",
}
METHODS = {1: "bitmap-clique", 2: "plan", 3: "wedge", 4: "edge-triangle", 5: "census"}

_P64 = ctypes.POINTER(ctypes.c_int64)
_P32 = ctypes.POINTER(ctypes.c_int32)
_PU64 = ctypes.POINTER(ctypes.c_uint64)


class JgpmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class _GraphInfo(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_int32), ("num_arcs", ctypes.c_int64),
                ("max_degree", ctypes.c_int32), ("num_dag_arcs", ctypes.c_int64),
                ("max_out_degree", ctypes.c_int32), ("device", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64)]


class _Stats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("setop_elements", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("rounds", ctypes.c_int32),
                ("method", ctypes.c_int32), ("launches", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class _Job(ctypes.Structure):
    _fields_ = [("graph", ctypes.c_void_p), ("pattern", ctypes.c_char_p)]


class Tuning(ctypes.Structure):
    """Work-split knobs of the batched (and plain clique) kernels."""
    _fields_ = [("min_group", ctypes.c_int32), ("split_degree", ctypes.c_int32),
                ("roots_per_task", ctypes.c_int32), ("intersect", ctypes.c_int32),
                ("graphs", ctypes.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class _BatchStats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("launches", ctypes.c_int32),
                ("tasks", ctypes.c_int32), ("used", Tuning)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_uint64), ("max_inflight", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("device", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("tuning", Tuning)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("rejected", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("evictions", ctypes.c_uint64), ("restores", ctypes.c_uint64),
                ("resident_bytes", ctypes.c_uint64), ("peak_frontier_bytes", ctypes.c_uint64),
                ("mean_batch", ctypes.c_double)]


def library_path():
    return os.environ.get("JGPM_LIBRARY", os.path.join(_PKG, "libjgpm.so"))


_lib = None


def lib():
    """The loaded libjgpm.so (raises JgpmError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise JgpmError(-8, f"{path} is missing; run `python -m jupiter_b200.build`")
    L = ctypes.CDLL(path)
    L.jgpm_version.restype = ctypes.c_char_p
    L.jgpm_last_error.restype = ctypes.c_char_p
    L.jgpm_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.jgpm_set_device.argtypes = [ctypes.c_int]
    G = ctypes.c_void_p
    PG = ctypes.POINTER(ctypes.c_void_p)
    L.jgpm_graph_load.argtypes = [ctypes.c_char_p, ctypes.c_int, PG]
    L.jgpm_graph_from_csr.argtypes = [_P64, _P32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int,
                                      PG]
    L.jgpm_graph_from_edges.argtypes = [_P32, _P32, ctypes.c_int64, ctypes.c_int32,
                                        ctypes.c_int, PG]
    L.jgpm_graph_rmat.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                  ctypes.c_int, PG]
    L.jgpm_rmat_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_uint64, _P32, _P32,
                                  _P64]
    L.jgpm_graph_get_info.argtypes = [G, ctypes.POINTER(_GraphInfo)]
    L.jgpm_graph_copy_csr.argtypes = [G, ctypes.c_int, _P64, _P32]
    L.jgpm_graph_save.argtypes = [G, ctypes.c_char_p, ctypes.c_int]
    L.jgpm_graph_free.argtypes = [G]
    L.jgpm_graph_free.restype = None
    L.jgpm_graph_stream.argtypes = [G, ctypes.POINTER(ctypes.c_void_p)]
    L.jgpm_count.argtypes = [G, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _PU64,
                             ctypes.POINTER(_Stats)]
    L.jgpm_count_ex.argtypes = [G, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                _PU64, ctypes.POINTER(_Stats)]
    L.jgpm_count_roots.argtypes = [G, ctypes.c_char_p, ctypes.c_int, ctypes.c_int64,
                                   ctypes.c_int64, ctypes.c_int64, _PU64, ctypes.POINTER(_Stats)]
    L.jgpm_count_shard.argtypes = [G, ctypes.c_char_p, ctypes.c_int, ctypes.c_int32,
                                   ctypes.c_int32, _PU64, ctypes.POINTER(_Stats)]
    L.jgpm_list.argtypes = [G, ctypes.c_char_p, ctypes.c_int, _P32, ctypes.c_int64,
                            _P64, ctypes.POINTER(_Stats)]
    L.jgpm_census4.argtypes = [G, _PU64, ctypes.POINTER(_Stats)]
    L.jgpm_setop.argtypes = [ctypes.c_int, _P32, ctypes.c_int32, _P32, ctypes.c_int32,
                             ctypes.c_int32, ctypes.c_int32, _P32, _P32]
    L.jgpm_setop_batch.argtypes = [ctypes.c_int, _P32, _P64, _P32, _P64, ctypes.c_int64, _P32,
                                   _P32, _P32, _P32, _P64]
    L.jgpm_setop_split.argtypes = [ctypes.c_int, _P32, ctypes.c_int32, _P32, ctypes.c_int32,
                                   ctypes.c_int32, _P32, _P32, _P32, _P32]
    L.jgpm_setop_split_batch.argtypes = [ctypes.c_int, _P32, _P64, _P32, _P64, ctypes.c_int64,
                                         _P32, _P32, _P32, _P32, _P32]
    L.jgpm_batch_count.argtypes = [ctypes.POINTER(_Job), ctypes.c_int32, ctypes.POINTER(Tuning),
                                   _PU64, ctypes.POINTER(_BatchStats)]
    V = ctypes.c_void_p
    L.jgpm_server_create.argtypes = [ctypes.POINTER(_ServerConfig), ctypes.POINTER(V)]
    L.jgpm_server_add_graph.argtypes = [V, V, ctypes.POINTER(ctypes.c_int32)]
    L.jgpm_server_submit.argtypes = [V, ctypes.c_int32, ctypes.c_char_p, _PU64]
    L.jgpm_server_wait.argtypes = [V, ctypes.c_uint64, ctypes.c_int32, _PU64,
                                   ctypes.POINTER(ctypes.c_double)]
    L.jgpm_server_get_stats.argtypes = [V, ctypes.POINTER(_ServerStats)]
    L.jgpm_server_replay.argtypes = [V, ctypes.c_int32, ctypes.c_int64, _P32,
                                     ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.POINTER(ctypes.c_double), _PU64,
                                     ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double)]
    L.jgpm_server_destroy.argtypes = [V]
    L.jgpm_graph_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
    L.jgpm_autotune.argtypes = [ctypes.POINTER(_Job), ctypes.c_int32, ctypes.c_int32,
                                ctypes.POINTER(Tuning)]
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise JgpmError(rc, lib().jgpm_last_error().decode())


def _p32(a):
    return a.ctypes.data_as(_P32)


def _p64(a):
    return a.ctypes.data_as(_P64)


def device_count():
    n = ctypes.c_int()
    _check(lib().jgpm_device_count(ctypes.byref(n)))
    return n.value


def version():
    return lib().jgpm_version().decode()


def rmat_edges(n, num_edges, a=0.57, b=0.19, c=0.19, seed=1):
    """The seeded R-MAT edge list computed on the host (the device generator's definition)."""
    src = np.empty(max(num_edges, 1), dtype=np.int32)
    dst = np.empty(max(num_edges, 1), dtype=np.int32)
    k = ctypes.c_int64()
    _check(lib().jgpm_rmat_edges(int(n), int(num_edges), a, b, c, int(seed), _p32(src),
                                 _p32(dst), ctypes.byref(k)))
    return src[: k.value].copy(), dst[: k.value].copy()


class Graph:
    """A graph resident on one GPU (symmetric CSR, plus the degree-oriented DAG on demand)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    # -- constructors ---------------------------------------------------------------
    @classmethod
    def load(cls, prefix, use_dag=False):
        """Reads the reference's prefix.meta.txt/.vertex.bin/.edge.bin CSR."""
        h = ctypes.c_void_p()
        _check(lib().jgpm_graph_load(prefix.encode(), int(bool(use_dag)), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_csr(cls, rowptr, col, use_dag=False):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        col = np.ascontiguousarray(col, dtype=np.int32)
        h = ctypes.c_void_p()
        _check(lib().jgpm_graph_from_csr(_p64(rowptr), _p32(col), len(rowptr) - 1, len(col),
                                         int(bool(use_dag)), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_edges(cls, src, dst, n, use_dag=False):
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        h = ctypes.c_void_p()
        _check(lib().jgpm_graph_from_edges(_p32(src), _p32(dst), len(src), int(n),
                                           int(bool(use_dag)), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def rmat(cls, n, edge_factor, a=0.57, b=0.19, c=0.19, seed=1, use_dag=False):
        """Seeded R-MAT graph generated on the device (edge_factor * n edges drawn)."""
        h = ctypes.c_void_p()
        _check(lib().jgpm_graph_rmat(int(n), int(edge_factor) * int(n), a, b, c, int(seed),
                                     int(bool(use_dag)), ctypes.byref(h)))
        return cls(h.value)

    # -- queries ----------------------------------------------------------------------
    def info(self):
        i = _GraphInfo()
        _check(lib().jgpm_graph_get_info(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _GraphInfo._fields_}

    def csr(self, dag=False):
        if dag:
            self.count("triangle")  # builds the DAG if needed
        info = self.info()
        m = info["num_dag_arcs"] if dag else info["num_arcs"]
        rowptr = np.empty(info["num_vertices"] + 1, dtype=np.int64)
        col = np.empty(max(m, 1), dtype=np.int32)
        _check(lib().jgpm_graph_copy_csr(self._h, int(bool(dag)), _p64(rowptr), _p32(col)))
        return rowptr, col[:m].copy()

    def set_tuning(self, tuning):
        """Lane-group / split knobs of this graph's plain clique kernels (counts unchanged)."""
        _check(lib().jgpm_graph_set_tuning(self._h, ctypes.byref(tuning)))

    def stream(self):
        """The cudaStream_t (as an int) on which this graph's kernels run."""
        s = ctypes.c_void_p()
        _check(lib().jgpm_graph_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def save(self, prefix, dag=False):
        _check(lib().jgpm_graph_save(self._h, prefix.encode(), int(bool(dag))))

    def count(self, pattern, induced=False, chunk_size=1, stats=False, flags=0, details=False):
        """Exact count of `pattern`.  With stats=True (the canonical plan's set-op elements,
        an extra untimed pass) or details=True returns (count, dict)."""
        out = ctypes.c_uint64()
        st = _Stats()
        f = flags | (COUNT_STATS if stats else 0)
        _check(lib().jgpm_count_ex(self._h, pattern.encode(), int(bool(induced)),
                                   int(chunk_size), f, ctypes.byref(out), ctypes.byref(st)))
        if stats or details:
            return out.value, {"count": st.count, "setop_elements": st.setop_elements,
                               "kernel_ms": st.kernel_ms, "rounds": st.rounds,
                               "method": METHODS.get(st.method, st.method),
                               "launches": st.launches}
        return out.value

    def count_roots(self, pattern, begin=0, end=-1, stride=1, induced=False, details=False):
        """Count of the embeddings rooted at root arcs begin, begin + stride, ... < end of the
        plan's CSR (the literal nested-loop plan; end < 0 means all arcs)."""
        out = ctypes.c_uint64()
        st = _Stats()
        _check(lib().jgpm_count_roots(self._h, pattern.encode(), int(bool(induced)), int(begin),
                                      int(end), int(stride), ctypes.byref(out),
                                      ctypes.byref(st)))
        if details:
            return out.value, {"kernel_ms": st.kernel_ms, "launches": st.launches}
        return out.value

    def count_shard(self, pattern, shard, nshards, induced=False, details=False):
        """Shard `shard` of `nshards` of the count of `pattern`; the shards add up to it."""
        out = ctypes.c_uint64()
        st = _Stats()
        _check(lib().jgpm_count_shard(self._h, pattern.encode(), int(bool(induced)), int(shard),
                                      int(nshards), ctypes.byref(out), ctypes.byref(st)))
        if details:
            return out.value, {"kernel_ms": st.kernel_ms, "launches": st.launches,
                               "method": METHODS.get(st.method, st.method)}
        return out.value

    def list(self, pattern, induced=False, capacity=None):
        """The embeddings of `pattern` as an (n, k) int32 array (listing mode).  capacity =
        None sizes the buffer with a first counting pass."""
        total = ctypes.c_int64()
        st = _Stats()
        if capacity is None:
            _check(lib().jgpm_list(self._h, pattern.encode(), int(bool(induced)), None, 0,
                                   ctypes.byref(total), ctypes.byref(st)))
            capacity = total.value
        k = 4
        if not induced:
            k = {"triangle": 3, "P0": 3, "3-clique": 3, "4-clique": 4, "P13": 4,
                 "5-clique": 5, "P14": 5, "6-clique": 6, "P15": 6, "7-clique": 7,
                 "P16": 7}.get(pattern, 4)
            if pattern.startswith("k-clique:"):
                k = int(pattern.split(":")[1])
        out = np.zeros((max(capacity, 1), k), dtype=np.int32)
        _check(lib().jgpm_list(self._h, pattern.encode(), int(bool(induced)), _p32(out),
                               int(capacity), ctypes.byref(total), ctypes.byref(st)))
        return out[: min(total.value, capacity)], total.value

    def census4(self):
        """Vertex-induced counts [3-star, 4-path, tailed triangle, 4-cycle, diamond, K4]."""
        out = np.zeros(6, dtype=np.uint64)
        st = _Stats()
        _check(lib().jgpm_census4(self._h, out.ctypes.data_as(_PU64), ctypes.byref(st)))
        return [int(x) for x in out]

    def close(self):
        if self._h and self._h.value:
            lib().jgpm_graph_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _jobs_array(jobs):
    arr = (_Job * len(jobs))()
    keep = []
    for i, (g, pattern) in enumerate(jobs):
        b = pattern.encode()
        keep.append(b)
        arr[i].graph = g._h.value
        arr[i].pattern = b
    return arr, keep


def batch_count(jobs, tuning=None):
    """Counts many (graph, pattern) jobs in one persistent launch.
    Returns (counts, stats dict)."""
    arr, keep = _jobs_array(jobs)
    counts = np.zeros(max(len(jobs), 1), dtype=np.uint64)
    st = _BatchStats()
    _check(lib().jgpm_batch_count(arr, len(jobs), ctypes.byref(tuning) if tuning else None,
                                  counts.ctypes.data_as(_PU64), ctypes.byref(st)))
    return [int(x) for x in counts[:len(jobs)]], {
        "kernel_ms": st.kernel_ms, "launches": st.launches, "tasks": st.tasks,
        "tuning": st.used.as_dict()}


def autotune(jobs, sample_jobs=256):
    """Times candidate tunings on a sample of the batch; returns the fastest Tuning."""
    arr, keep = _jobs_array(jobs)
    t = Tuning()
    _check(lib().jgpm_autotune(arr, len(jobs), int(sample_jobs), ctypes.byref(t)))
    return t


class Server:
    """Continuous-batching query server over a memory-budgeted graph pool (one device)."""

    def __init__(self, memory_budget_bytes=150 << 30, max_inflight=4, max_batch=256, device=0,
                 tuning=None):
        cfg = _ServerConfig()
        cfg.memory_budget_bytes = int(memory_budget_bytes)
        cfg.max_inflight = int(max_inflight)
        cfg.max_batch = int(max_batch)
        cfg.device = int(device)
        if tuning is not None:
            cfg.tuning = tuning
        h = ctypes.c_void_p()
        _check(lib().jgpm_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._graphs = []

    def add_graph(self, graph):
        """Hands the graph to the pool (the server frees it); returns its graph id."""
        gid = ctypes.c_int32()
        _check(lib().jgpm_server_add_graph(self._h, graph._h, ctypes.byref(gid)))
        graph._h = ctypes.c_void_p()  # owned by the server now
        return gid.value

    def submit(self, graph_id, pattern):
        t = ctypes.c_uint64()
        _check(lib().jgpm_server_submit(self._h, int(graph_id), pattern.encode(),
                                        ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        c = ctypes.c_uint64()
        lat = ctypes.c_double()
        _check(lib().jgpm_server_wait(self._h, int(ticket), int(timeout_ms), ctypes.byref(c),
                                      ctypes.byref(lat)))
        return c.value, lat.value

    def stats(self):
        st = _ServerStats()
        _check(lib().jgpm_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def replay(self, graph_ids, patterns, arrival_s, plain=False):
        """Open-loop trace replay inside the library; returns (counts, latency_ms, wall_s)."""
        n = len(graph_ids)
        gids = np.ascontiguousarray(graph_ids, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        pats = (ctypes.c_char_p * max(n, 1))(*[p.encode() for p in patterns])
        counts = np.zeros(max(n, 1), dtype=np.uint64)
        lat = np.zeros(max(n, 1), dtype=np.float64)
        wall = ctypes.c_double()
        _check(lib().jgpm_server_replay(
            self._h, 1 if plain else 0, n, _p32(gids), pats,
            arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), counts.ctypes.data_as(_PU64),
            lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(wall)))
        return [int(x) for x in counts[:n]], lat[:n].copy(), wall.value

    def close(self):
        if self._h and self._h.value:
            lib().jgpm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setop(op, a, b, upper=None, exclude=None):
    """One sorted-set operation; returns a count (the *_COUNT ops) or an int32 array."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    up = np.iinfo(np.int32).max if upper is None else int(upper)
    ex = -1 if exclude is None else int(exclude)
    cap = min(len(a), len(b)) if op == OP_INTERSECT else len(a)
    out = np.empty(max(cap, 1), dtype=np.int32)
    n = ctypes.c_int32()
    _check(lib().jgpm_setop(op, _p32(a), len(a), _p32(b), len(b), up, ex, _p32(out),
                            ctypes.byref(n)))
    if op in (OP_INTERSECT_COUNT, OP_DIFFERENCE_COUNT):
        return n.value
    return out[: n.value].copy()


def setop_batch(op, a_lists, b_lists, upper=None, exclude=None):
    """Many set operations in one launch; returns counts (and result lists when materialising)."""
    a_off = np.zeros(len(a_lists) + 1, dtype=np.int64)
    b_off = np.zeros(len(b_lists) + 1, dtype=np.int64)
    a_off[1:] = np.cumsum([len(x) for x in a_lists])
    b_off[1:] = np.cumsum([len(x) for x in b_lists])
    a = np.concatenate([np.asarray(x, dtype=np.int32) for x in a_lists] + [np.zeros(0, np.int32)])
    b = np.concatenate([np.asarray(x, dtype=np.int32) for x in b_lists] + [np.zeros(0, np.int32)])
    nops = len(a_lists)
    counts = np.zeros(max(nops, 1), dtype=np.int32)
    up = None if upper is None else np.ascontiguousarray(upper, dtype=np.int32)
    ex = None if exclude is None else np.ascontiguousarray(exclude, dtype=np.int32)
    mat = op in (OP_INTERSECT, OP_DIFFERENCE)
    out = out_off = None
    if mat:
        caps = [min(len(x), len(y)) if op == OP_INTERSECT else len(x)
                for x, y in zip(a_lists, b_lists)]
        out_off = np.zeros(nops + 1, dtype=np.int64)
        out_off[1:] = np.cumsum(caps)
        out = np.empty(max(int(out_off[-1]), 1), dtype=np.int32)
    _check(lib().jgpm_setop_batch(op, _p32(a), _p64(a_off), _p32(b), _p64(b_off), nops,
                                  _p32(up) if up is not None else None,
                                  _p32(ex) if ex is not None else None, _p32(counts),
                                  _p32(out) if mat else None, _p64(out_off) if mat else None))
    counts = counts[:nops]
    if mat:
        return counts, [out[out_off[i]: out_off[i] + counts[i]].copy() for i in range(nops)]
    return counts


def _split_lists(kind, a, b, r):
    """(c, d, e) of one pair from its count (e None for SPLIT_DIF_INT)."""
    if kind == SPLIT_FUSE:
        return (len(a) - r, r, len(b) - r)
    return (r, len(a) - r, None)


def setop_split(kind, a, b, upper=None):
    """One fused split (SPLIT_FUSE: A \\ B, A & B, B \\ A; SPLIT_DIF_INT: A below upper
    minus B, and the rest of A); returns (count, c, d, e), e None for SPLIT_DIF_INT."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    up = np.iinfo(np.int32).max if upper is None else int(upper)
    c = np.empty(max(len(a), 1), np.int32)
    d = np.empty(max(len(a), 1), np.int32)
    e = np.empty(max(len(b), 1), np.int32)
    n = ctypes.c_int32()
    _check(lib().jgpm_setop_split(kind, _p32(a), len(a), _p32(b), len(b), up, _p32(c), _p32(d),
                                  _p32(e) if kind == SPLIT_FUSE else None, ctypes.byref(n)))
    nc, nd, ne = _split_lists(kind, a, b, n.value)
    return n.value, c[:nc].copy(), d[:nd].copy(), (e[:ne].copy() if ne is not None else None)


def setop_split_batch(kind, a_lists, b_lists, upper=None):
    """Many fused splits in one launch; returns the counts and, per pair, (c, d, e)."""
    nops = len(a_lists)
    a_off = np.zeros(nops + 1, dtype=np.int64)
    b_off = np.zeros(nops + 1, dtype=np.int64)
    a_off[1:] = np.cumsum([len(x) for x in a_lists])
    b_off[1:] = np.cumsum([len(x) for x in b_lists])
    a = np.concatenate([np.asarray(x, dtype=np.int32) for x in a_lists] + [np.zeros(0, np.int32)])
    b = np.concatenate([np.asarray(x, dtype=np.int32) for x in b_lists] + [np.zeros(0, np.int32)])
    counts = np.zeros(max(nops, 1), dtype=np.int32)
    c = np.empty(max(len(a), 1), np.int32)
    d = np.empty(max(len(a), 1), np.int32)
    e = np.empty(max(len(b), 1), np.int32)
    up = None if upper is None else np.ascontiguousarray(upper, dtype=np.int32)
    _check(lib().jgpm_setop_split_batch(kind, _p32(a), _p64(a_off), _p32(b), _p64(b_off), nops,
                                        _p32(up) if up is not None else None, _p32(counts),
                                        _p32(c), _p32(d),
                                        _p32(e) if kind == SPLIT_FUSE else None))
    counts = counts[:nops]
    out = []
    for i in range(nops):
        nc, nd, ne = _split_lists(kind, a_lists[i], b_lists[i], int(counts[i]))
        a0, b0 = int(a_off[i]), int(b_off[i])
        out.append((c[a0: a0 + nc].copy(), d[a0: a0 + nd].copy(),
                    e[b0: b0 + ne].copy() if ne is not None else None))
    return counts, out


def solve(prefix, pattern, rounds=1, print_result=True):
    """The reference CLI flow (src/main.cc:7-47, src/jupiter_gpm.cu:27-925) on one GPU:
    load, orient for the clique patterns, count, print `gpu count:<n>  runtime:<s>s`."""
    use_dag = pattern in ("P13", "P14", "P15", "P16")
    with Graph.load(prefix, use_dag=use_dag) as g:
        c, st = g.count(pattern, chunk_size=rounds, details=True)
    if print_result:
        print(f"=====================gpu count:{c}  runtime:{st['kernel_ms'] / 1e3:.6f}s")
    return c
