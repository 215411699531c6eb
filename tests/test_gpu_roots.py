"""GPU parity of jgpm_count_roots, the count over a strided sample of root arcs, against the
oracle's restatement of the same plans on the same sample (oracle/oracle.cc over_arcs), bit
for bit.  Counts over disjoint samples add up to the full count."""
import zlib

import numpy as np
import pytest

import graphs as G
import oracle_api as O

pytestmark = pytest.mark.gpu

# (library name, induced, oracle name, runs on the DAG)
PLANS = [
    ("triangle", 0, "P0", True), ("4-clique", 0, "P13", True), ("5-clique", 0, "P14", True),
    ("6-clique", 0, "P15", True), ("P1", 0, "P1", False), ("P2", 0, "P2", False),
    ("P3", 0, "P3", False), ("P7", 0, "P7", False), ("P9", 0, "P9", False),
    ("vsgm_last_pattern", 0, "vsgm_last_pattern", False),
    ("4-cycle", 1, "induced-4-cycle", False), ("diamond", 1, "induced-diamond", False),
    ("tailed-triangle", 1, "induced-tailed-triangle", False),
    ("4-path", 1, "induced-4-path", False), ("3-star", 1, "induced-3-star", False),
]


@pytest.fixture(scope="module")
def graph(gpu):
    spec = ("rmat-n2000-ef8-s9", 2000, 8, 0.57, 0.19, 0.19, 9)
    sym = G.rmat_csr(spec)
    g = gpu.Graph.rmat(*spec[1:])
    yield g, sym, O.orient(sym)
    g.close()


@pytest.mark.parametrize("name,induced,oname,dag", PLANS)
def test_root_samples_match_oracle(graph, name, induced, oname, dag):
    g, sym, dg = graph
    csr = dg if dag else sym
    m = csr.m
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    samples = [(0, m, 1), (0, m, 7), (int(rng.integers(0, m // 2)), m, 13),
               (int(m // 3), int(2 * m // 3), 3), (m - 1, m, 1), (5, 5, 1)]
    for b, e, s in samples:
        want = O.count(oname, csr, b, e, s)[0]
        got = g.count_roots(name, b, e, s, induced=bool(induced))
        assert got == want, (name, induced, b, e, s, got, want)
    # all arcs = the plain count; a partition of the arcs by residue adds up to it
    full = g.count(name, induced=bool(induced))
    assert g.count_roots(name, induced=bool(induced)) == full
    assert sum(g.count_roots(name, r, -1, 5, induced=bool(induced)) for r in range(5)) == full
    # the slots of one vertex are its rooted embeddings
    v = int(np.argmax(np.diff(csr.rowptr)))
    b, e = int(csr.rowptr[v]), int(csr.rowptr[v + 1])
    assert g.count_roots(name, b, e, 1, induced=bool(induced)) == O.count(oname, csr, b, e, 1)[0]


def test_root_samples_reject_bad_arguments(gpu, graph):
    g, sym, _ = graph
    for args, code in [(("P1", 10, 5, 1), -1), (("P1", 0, sym.m + 1, 1), -1),
                       (("P1", 0, -1, 0), -1), (("3-star", 0, -1, 1), -5),
                       (("k-clique:8", 0, -1, 1), -5)]:
        with pytest.raises(gpu.JgpmError) as e:
            g.count_roots(*args)
        assert e.value.code == code, args
