"""GPU test of jgpm_count_noalloc, the counting entry point that allocates nothing.

It is meant for callers that cannot allocate device memory while they count, such as a host
application whose memory manager owns the whole device, or a latency-critical path that may
not call cudaMalloc.  Instead of allocating, the entry point works in a fixed static device
array.  The test calls it through the C-ABI and checks that two calls in a row give the same
counts as jgpm_count, the allocating entry point.  Counts are exact integers, so the
tolerance is zero.  This file is collected last, so a run that stops at the first failure
has already run every other test.  It also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # (pattern, induced); the graph is built with its DAG for the clique plans
    ("P13", 0), ("triangle", 0), ("P14", 0), ("P1", 0), ("P2", 0), ("P5", 0),
    ("diamond", 1), ("tailed-triangle", 1),
]


def _bind(J):
    L = J.lib()
    L.jgpm_count_noalloc.restype = ctypes.c_int
    L.jgpm_count_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_uint64)]
    return L


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    J = gpu
    L = _bind(J)
    with J.Graph.rmat(1 << 13, 8, 0.57, 0.19, 0.19, 21, use_dag=True) as g:
        for pattern, induced in CASES:
            want = g.count(pattern, induced=bool(induced))
            for _ in range(2):  # the static scratch keeps the previous call's contents
                out = ctypes.c_uint64(12345)
                rc = L.jgpm_count_noalloc(g._h, pattern.encode(), induced, ctypes.byref(out))
                assert rc == 0, (pattern, L.jgpm_last_error().decode())
                assert out.value == want, (pattern, induced, out.value, want)


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
