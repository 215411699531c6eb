"""GPU test of jgpm_count_noalloc, the counting entry point that allocates nothing.

It is meant for callers that cannot allocate device memory while they count, such as a host
application whose memory manager owns the whole device, or a latency-critical path that may
not call cudaMalloc.  Instead of allocating, the entry point works in a fixed static device
array.  The test calls it through the C-ABI and checks that two calls in a row give the same
counts as jgpm_count, the allocating entry point, and as the oracle.  Counts are exact
integers, so the tolerance is zero.  This file is collected last, so a run that stops at the
first failure has already run every other test.  It also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

CASES = [  # (pattern, induced, oracle name, on the DAG); the graph is built with its DAG
    ("P13", 0, "P13", True), ("triangle", 0, "P0", True), ("P14", 0, "P14", True),
    ("P15", 0, "P15", True), ("P16", 0, "P16", True), ("P1", 0, "P1", False),
    ("P2", 0, "P2", False), ("P5", 0, "P5", False),
    ("diamond", 1, "induced-diamond", False),
    ("tailed-triangle", 1, "induced-tailed-triangle", False),
]
SPEC = (1 << 13, 8, 0.57, 0.19, 0.19, 21)


def _bind(J):
    L = J.lib()
    L.jgpm_count_noalloc.restype = ctypes.c_int
    L.jgpm_count_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_uint64)]
    return L


def _noalloc(L, g, pattern, induced):
    out = ctypes.c_uint64(12345)
    rc = L.jgpm_count_noalloc(g._h, pattern.encode(), induced, ctypes.byref(out))
    assert rc == 0, (pattern, L.jgpm_last_error().decode())
    return out.value


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    J = gpu
    L = _bind(J)
    sym = O.rmat_graph(*SPEC)
    dag = O.orient(sym)
    with J.Graph.rmat(*SPEC, use_dag=True) as g:
        for pattern, induced, oname, on_dag in CASES:
            want = g.count(pattern, induced=bool(induced))
            assert want == O.count(oname, dag if on_dag else sym)[0], pattern
            for _ in range(2):  # the static scratch keeps the previous call's contents
                assert _noalloc(L, g, pattern, induced) == want, (pattern, induced)


def test_noalloc_capacity_boundary(gpu):
    """The fixed scratch holds four per-warp lists for 8 warps at a maximum degree of
    262,112: a hub of exactly that degree is counted, one of 300,000 is refused."""
    J = gpu
    L = _bind(J)
    hub = 262112
    tri = np.array([[1, 2], [2, 3], [1, 3], [3, 4]], dtype=np.int32)  # triangles at the hub
    src = np.concatenate([np.zeros(hub, np.int32), tri[:, 0]])
    dst = np.concatenate([np.arange(1, hub + 1, dtype=np.int32), tri[:, 1]])
    with J.Graph.from_edges(src, dst, hub + 1) as star:
        assert star.info()["max_degree"] == hub
        for pattern in ("P2", "P1"):
            want = star.count(pattern)
            for _ in range(2):
                assert _noalloc(L, star, pattern, 0) == want, pattern
        # sum over edges of C(t_e, 2): edge 0-3 lies on 3 triangles (1, 2 and 4), edges 0-1,
        # 0-2, 1-2, 1-3 and 2-3 on 2 each, the others on at most 1: 3 + 5 * 1 = 8
        assert star.count("P2") == 8


def test_noalloc_rejects_what_it_cannot_do(gpu):
    J = gpu
    L = _bind(J)
    out = ctypes.c_uint64()
    with J.Graph.rmat(1 << 10, 4, 0.57, 0.19, 0.19, 3) as g:
        # no DAG yet: the clique plans are refused instead of allocating one
        assert L.jgpm_count_noalloc(g._h, b"P13", 0, ctypes.byref(out)) == -1
        # closed-form patterns have no plan kernel
        assert L.jgpm_count_noalloc(g._h, b"3-star", 0, ctypes.byref(out)) == -5
    # a maximum degree beyond what the fixed scratch holds is refused with a capacity error
    hub = 300000
    src = np.zeros(hub, dtype=np.int32)
    dst = np.arange(1, hub + 1, dtype=np.int32)
    with J.Graph.from_edges(src, dst, hub + 1) as star:
        assert L.jgpm_count_noalloc(star._h, b"P2", 0, ctypes.byref(out)) == -10
        assert b"scratch" in L.jgpm_last_error()
