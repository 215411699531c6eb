"""Test graphs: closed-form families and the seeded R-MAT cases used by the parity tests."""
import hashlib
import itertools

import numpy as np

import oracle_api as O


def edges_complete(n):
    return [(i, j) for i in range(n) for j in range(i + 1, n)]


def edges_cycle(n):
    return [(i, (i + 1) % n) for i in range(n)]


def edges_star(k):
    return [(0, i) for i in range(1, k + 1)]


def edges_complete_bipartite(a, b):
    return [(i, a + j) for i in range(a) for j in range(b)]


def edges_wheel(n):
    """Hub 0 joined to the cycle 1..n."""
    return [(0, i) for i in range(1, n + 1)] + [(i, i % n + 1) for i in range(1, n + 1)]


def edges_petersen():
    outer = [(i, (i + 1) % 5) for i in range(5)]
    spokes = [(i, i + 5) for i in range(5)]
    inner = [(5 + i, 5 + (i + 2) % 5) for i in range(5)]
    return outer + spokes + inner


NAMED = {
    "K6": (6, edges_complete(6)),
    "K9": (9, edges_complete(9)),
    "C7": (7, edges_cycle(7)),
    "C4": (4, edges_cycle(4)),
    "S5": (6, edges_star(5)),
    "K34": (7, edges_complete_bipartite(3, 4)),
    "W6": (7, edges_wheel(6)),
    "petersen": (10, edges_petersen()),
}

# (name, n, edge_factor, a, b, c, seed)
RMAT_SMALL = [
    ("rmat-n64-ef4-s1", 64, 4, 0.57, 0.19, 0.19, 1),
    ("rmat-n100-ef8-s2", 100, 8, 0.45, 0.1375, 0.1375, 2),
    ("rmat-n256-ef8-s3", 256, 8, 0.57, 0.19, 0.19, 3),
    ("rmat-n1000-ef16-s4", 1000, 16, 0.60, 0.10, 0.10, 4),
    ("rmat-n4096-ef8-s5", 4096, 8, 0.57, 0.19, 0.19, 5),
]

# The triangle-count workload itself: R-MAT scale 16, edge factor 16, seed 1.
RMAT_TRIANGLE = ("rmat-s16-ef16-s1", 1 << 16, 16, 0.57, 0.19, 0.19, 1)
# The k-clique workload: R-MAT scale 22, edge factor 4, seed 1 (citation-graph shape).
RMAT_CLIQUE = ("rmat-s22-ef4-s1", 1 << 22, 4, 0.57, 0.19, 0.19, 1)


def named_csr(name):
    n, e = NAMED[name]
    src = np.array([u for u, v in e], dtype=np.int32)
    dst = np.array([v for u, v in e], dtype=np.int32)
    return O.build_csr(n, src, dst)


def rmat_csr(spec):
    _, n, ef, a, b, c, seed = spec
    return O.rmat_graph(n, ef, a, b, c, seed)


def csr_digest(g):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.rowptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(g.col, dtype=np.int32).tobytes())
    return h.hexdigest()[:16]


# Edge-induced pattern graphs of the reference plans, read off the loop nests of
# src/message_passing_gpu_kernels.cuh (vertex 0 = v0, 1 = v1, ...).
PATTERN_EDGES = {
    "P1": (4, [(0, 1), (0, 2), (1, 3), (2, 3)]),
    "P2": (4, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3)]),
    "P3": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (3, 4)]),
    "P4": (5, [(0, 1), (0, 2), (1, 2), (1, 3), (0, 4), (3, 4)]),
    "P5": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3), (0, 4), (1, 4)]),
    "P6": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 4), (3, 4)]),
    "P7": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (2, 3), (0, 4), (1, 4)]),
    "P8": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (2, 3), (0, 4), (1, 4), (3, 4)]),
    "P9": (5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3), (0, 4), (1, 4), (2, 4)]),
    "P10": (6, [(0, 1), (0, 2), (1, 2), (0, 3), (2, 3), (0, 4), (1, 4), (0, 5), (3, 5)]),
    "P11": (6, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (0, 4), (2, 4), (1, 5), (2, 5)]),
    "P12": (6, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3), (0, 4), (1, 4), (2, 4),
                (0, 5), (1, 5)]),
    "vsgm_last_pattern": (6, [(0, 1), (0, 2), (1, 3), (2, 3), (0, 4), (1, 4), (0, 5), (1, 5)]),
}


def automorphisms(k, edges):
    es = {frozenset(e) for e in edges}
    c = 0
    for p in itertools.permutations(range(k)):
        if {frozenset((p[u], p[v])) for u, v in edges} == es:
            c += 1
    return c


NONCLIQUE_PLANS = ["P1", "P2", "P3", "P4", "P5", "P6", "P7", "P8", "P9", "P10", "P11", "P12",
                   "vsgm_last_pattern"]
CLIQUE_PLANS = {"P0": 3, "P13": 4, "P14": 5, "P15": 6, "P16": 7}
INDUCED = ["induced-3-star", "induced-4-path", "induced-tailed-triangle", "induced-4-cycle",
           "induced-diamond"]
CENSUS_ORDER = ["3-star", "4-path", "tailed-triangle", "4-cycle", "diamond", "4-clique"]
