"""ctypes binding of the CPU oracle (oracle/liboracle.so) and the reference-code driver
(oracle/_ref/libjref.so).  Test infrastructure: imported only by tests/, the smoke check
and the bench's CPU-baseline leg."""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import build_oracle as _bo  # noqa: E402

_P64 = ctypes.POINTER(ctypes.c_int64)
_P32 = ctypes.POINTER(ctypes.c_int32)
_PU64 = ctypes.POINTER(ctypes.c_uint64)

_lib = None
_ref = None


def _p(a, t):
    return a.ctypes.data_as(t)


def lib():
    global _lib
    if _lib is None:
        path = _bo.oracle_lib_path()
        if not os.path.exists(path) or os.environ.get("JGPM_REBUILD_ORACLE"):
            _bo.build_oracle()
        L = ctypes.CDLL(path)
        L.orc_rmat_edges.restype = ctypes.c_int64
        L.orc_rmat_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                     _P32, _P32, ctypes.c_int]
        L.orc_build_csr.restype = ctypes.c_int64
        L.orc_build_csr.argtypes = [ctypes.c_int32, ctypes.c_int64, _P32, _P32, _P64, _P32]
        L.orc_orient.restype = ctypes.c_int64
        L.orc_orient.argtypes = [ctypes.c_int32, _P64, _P32, _P64, _P32]
        L.orc_count.restype = ctypes.c_int
        L.orc_count.argtypes = [ctypes.c_char_p, ctypes.c_int32, _P64, _P32, ctypes.c_int64,
                                ctypes.c_int64, ctypes.c_int64, ctypes.c_int, _PU64, _PU64]
        L.orc_count_clique.restype = ctypes.c_int
        L.orc_count_clique.argtypes = [ctypes.c_int, ctypes.c_int32, _P64, _P32, ctypes.c_int,
                                       _PU64, _PU64]
        L.orc_census4.restype = ctypes.c_int
        L.orc_census4.argtypes = [ctypes.c_int32, _P64, _P32, _PU64]
        L.orc_fuse_set.restype = ctypes.c_int32
        L.orc_fuse_set.argtypes = [_P32, ctypes.c_int32, _P32, ctypes.c_int32, _P32, _P32, _P32]
        L.orc_dif_int_set.restype = ctypes.c_int32
        L.orc_dif_int_set.argtypes = [_P32, ctypes.c_int32, _P32, ctypes.c_int32,
                                      ctypes.c_int32, _P32, _P32]
        L.orc_search_2phase.restype = None
        L.orc_search_2phase.argtypes = [_P32, ctypes.c_int32, ctypes.c_int32, _P32,
                                        ctypes.c_int64, ctypes.POINTER(ctypes.c_uint8), _P32]
        L.orc_count_smaller.restype = ctypes.c_uint32
        L.orc_count_smaller.argtypes = [ctypes.c_int32, _P32, ctypes.c_int32]
        L.orc_search_bound.restype = None
        L.orc_search_bound.argtypes = [_P32, ctypes.c_int32, _P32, ctypes.c_int64, _P32]
        L.orc_hindex_count.restype = ctypes.c_int64
        L.orc_hindex_count.argtypes = [_P32, ctypes.c_int32, _P32, ctypes.c_int32]
        L.orc_count_embeddings.restype = ctypes.c_uint64
        L.orc_count_embeddings.argtypes = [ctypes.c_int, ctypes.c_int, _P32, ctypes.c_int32,
                                           _P64, _P32]
        _lib = L
    return _lib


def threads():
    return int(os.environ.get("JGPM_ORACLE_THREADS", os.cpu_count() or 1))


class Csr:
    def __init__(self, n, rowptr, col):
        self.n = int(n)
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)

    @property
    def m(self):
        return int(self.rowptr[-1])

    def degrees(self):
        return np.diff(self.rowptr)


def rmat_edges(n, num_edges, a, b, c, seed):
    src = np.empty(num_edges, dtype=np.int32)
    dst = np.empty(num_edges, dtype=np.int32)
    k = lib().orc_rmat_edges(n, num_edges, a, b, c, seed, _p(src, _P32), _p(dst, _P32),
                             threads())
    return src[:k].copy(), dst[:k].copy()


def build_csr(n, src, dst):
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    rowptr = np.empty(n + 1, dtype=np.int64)
    col = np.empty(2 * len(src), dtype=np.int32)
    m = lib().orc_build_csr(n, len(src), _p(src, _P32), _p(dst, _P32), _p(rowptr, _P64),
                            _p(col, _P32))
    return Csr(n, rowptr, col[:m].copy())


def orient(g):
    rowptr = np.empty(g.n + 1, dtype=np.int64)
    col = np.empty(max(g.m, 1), dtype=np.int32)
    m = lib().orc_orient(g.n, _p(g.rowptr, _P64), _p(g.col, _P32), _p(rowptr, _P64),
                         _p(col, _P32))
    return Csr(g.n, rowptr, col[:m].copy())


def rmat_graph(n, edge_factor, a=0.57, b=0.19, c=0.19, seed=1):
    src, dst = rmat_edges(n, edge_factor * n, a, b, c, seed)
    return build_csr(n, src, dst)


def count(pattern, g, begin=0, end=None, stride=1, nthreads=None):
    """Returns (count, set-op elements) of a plan; g is the DAG for cliques/P0, else symmetric."""
    if end is None:
        end = g.m
    c = ctypes.c_uint64()
    e = ctypes.c_uint64()
    rc = lib().orc_count(pattern.encode(), g.n, _p(g.rowptr, _P64), _p(g.col, _P32), begin, end,
                         stride, nthreads or threads(), ctypes.byref(c), ctypes.byref(e))
    if rc != 0:
        raise ValueError("oracle: unknown pattern " + pattern)
    return c.value, e.value


def census4(g):
    out = np.zeros(6, dtype=np.uint64)
    rc = lib().orc_census4(g.n, _p(g.rowptr, _P64), _p(g.col, _P32), _p(out, _PU64))
    if rc != 0:
        raise ValueError("census4: graph too large")
    return [int(x) for x in out]


def fuse_set(a, b):
    """(|A & B|, A \\ B, A & B, B \\ A) as the reference's fuse_set gives them; with an empty
    operand its count 0 and None for the unwritten lists."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    c = np.empty(max(len(a), 1), np.int32)
    d = np.empty(max(len(a), 1), np.int32)
    e = np.empty(max(len(b), 1), np.int32)
    r = int(lib().orc_fuse_set(_p(a, _P32), len(a), _p(b, _P32), len(b), _p(c, _P32),
                               _p(d, _P32), _p(e, _P32)))
    if len(a) == 0 or len(b) == 0:
        return r, None, None, None
    return r, c[: len(a) - r].copy(), d[:r].copy(), e[: len(b) - r].copy()


def search_2phase(lst, keys, width=32):
    """(found, marked index) of each key by the reference's cached two-phase search with
    `width` pivots (32: the warp form, 256: the CTA form)."""
    lst = np.ascontiguousarray(lst, dtype=np.int32)
    keys = np.ascontiguousarray(keys, dtype=np.int32)
    found = np.zeros(len(keys), np.uint8)
    marked = np.zeros(len(keys), np.int32)
    lib().orc_search_2phase(_p(lst, _P32), len(lst), int(width), _p(keys, _P32), len(keys),
                            found.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                            _p(marked, _P32))
    return found.astype(bool), marked


def count_smaller(bound, lst):
    """The reference's count_smaller(bound, list) as it computes it."""
    lst = np.ascontiguousarray(lst, dtype=np.int32)
    return int(lib().orc_count_smaller(int(bound), _p(lst, _P32), len(lst)))


def search_bound(lst, keys):
    """The position the reference's binary_search_bound returns for each key."""
    lst = np.ascontiguousarray(lst, dtype=np.int32)
    keys = np.ascontiguousarray(keys, dtype=np.int32)
    pos = np.zeros(len(keys), np.int32)
    lib().orc_search_bound(_p(lst, _P32), len(lst), _p(keys, _P32), len(keys), _p(pos, _P32))
    return pos


def hindex_count(a, b):
    """|A & B| by the reference's hash-bin intersection (-1 if a bin would overflow)."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    return int(lib().orc_hindex_count(_p(a, _P32), len(a), _p(b, _P32), len(b)))


def dif_int_set(a, b, upper=None):
    """(|c|, c, d) as the reference's dif_int_set gives them (upper None: the unbounded form);
    with an empty operand its count 0 and None for the unwritten lists."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    up = np.iinfo(np.int32).max if upper is None else int(upper)
    c = np.empty(max(len(a), 1), np.int32)
    d = np.empty(max(len(a), 1), np.int32)
    r = int(lib().orc_dif_int_set(_p(a, _P32), len(a), _p(b, _P32), len(b), up, _p(c, _P32),
                                  _p(d, _P32)))
    if len(a) == 0 or len(b) == 0:
        return r, None, None
    return r, c[:r].copy(), d[: len(a) - r].copy()


def count_embeddings(k, edges, g):
    he = np.ascontiguousarray(np.array(edges, dtype=np.int32).reshape(-1))
    return int(lib().orc_count_embeddings(k, len(edges), _p(he, _P32), g.n,
                                          _p(g.rowptr, _P64), _p(g.col, _P32)))


def write_reference_files(g, prefix, max_degree=None):
    """Writes the reference's on-disk CSR (common/graph.cc:26-46 reads it;
    :727-753 writes it): prefix.meta.txt, prefix.vertex.bin (int64), prefix.edge.bin (int32)."""
    md = int(max_degree if max_degree is not None else (g.degrees().max() if g.n else 0))
    with open(prefix + ".meta.txt", "w") as f:
        f.write(f"{g.n}\n{g.m}\n4 8 1 2\n{md}\n0\n0\n0\n")
    g.rowptr.astype(np.int64).tofile(prefix + ".vertex.bin")
    g.col.astype(np.int32).tofile(prefix + ".edge.bin")


# ---------------------------------------------------------------- reference-code driver
def ref_lib():
    """The reference's own host code driving the plans, or None if it is not built."""
    global _ref
    if _ref is None:
        path = _bo.build_ref()
        if path is None or not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.ref_graph_load.restype = ctypes.c_void_p
        L.ref_graph_load.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.ref_graph_free.argtypes = [ctypes.c_void_p]
        L.ref_graph_info.argtypes = [ctypes.c_void_p, _P64, _P64]
        L.ref_graph_copy.argtypes = [ctypes.c_void_p, _P64, _P32]
        L.ref_count.restype = ctypes.c_int
        L.ref_count.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64,
                                ctypes.c_int64, ctypes.c_int, _PU64,
                                ctypes.POINTER(ctypes.c_double)]
        _ref = L
    return _ref


class RefGraph:
    """A graph loaded by the reference's Graph(prefix, use_dag) loader."""

    def __init__(self, prefix, use_dag):
        L = ref_lib()
        if L is None:
            raise RuntimeError("reference host library not built")
        self.L = L
        self.h = L.ref_graph_load(prefix.encode(), 1 if use_dag else 0)
        nv = ctypes.c_int64()
        ne = ctypes.c_int64()
        L.ref_graph_info(self.h, ctypes.byref(nv), ctypes.byref(ne))
        self.n, self.m = nv.value, ne.value

    def csr(self):
        rowptr = np.empty(self.n + 1, dtype=np.int64)
        col = np.empty(max(self.m, 1), dtype=np.int32)
        self.L.ref_graph_copy(self.h, _p(rowptr, _P64), _p(col, _P32))
        return Csr(self.n, rowptr, col[: self.m].copy())

    def count(self, pattern, begin=0, end=None, stride=1, nthreads=None):
        if end is None:
            end = self.m
        c = ctypes.c_uint64()
        t = ctypes.c_double()
        rc = self.L.ref_count(self.h, pattern.encode(), begin, end, stride,
                              nthreads or threads(), ctypes.byref(c), ctypes.byref(t))
        if rc != 0:
            raise ValueError("reference driver: unknown pattern " + pattern)
        return c.value, t.value

    def close(self):
        if self.h:
            self.L.ref_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
