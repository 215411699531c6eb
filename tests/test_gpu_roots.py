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


SHARD_PATTERNS = [("triangle", 0), ("4-clique", 0), ("5-clique", 0), ("k-clique:6", 0),
                  ("k-clique:8", 0), ("P1", 0), ("P2", 0), ("P5", 0), ("4-cycle", 1),
                  ("tailed-triangle", 1)]


@pytest.mark.parametrize("name,induced", SHARD_PATTERNS)
def test_shards_add_up_to_the_count(graph, name, induced):
    g = graph[0]
    full = g.count(name, induced=bool(induced))
    for n in (2, 3, 7):
        parts = [g.count_shard(name, r, n, induced=bool(induced)) for r in range(n)]
        assert sum(parts) == full, (name, n, parts, full)
    assert g.count_shard(name, 0, 1, induced=bool(induced)) == full


def test_shards_cover_every_tier(gpu):
    """K_1101 puts roots in the edge-rooted list tier (out-degree > 1024 in the DAG of K_n is
    reached by ids 0..75), the wide bitmap band and every other tier; the crown's hub and
    B vertices (out-degree 5000) take the list tier's chunked tasks.  The shards add up."""
    from math import comb
    n = 1101
    iu = np.triu_indices(n, 1)
    with gpu.Graph.from_edges(iu[0].astype(np.int32), iu[1].astype(np.int32), n) as g:
        for k, want in ((3, comb(n, 3)), (4, comb(n, 4))):
            for ns in (2, 5):
                assert sum(g.count_shard(f"k-clique:{k}", r, ns) for r in range(ns)) == want
    na, nb, grp = 5000, 5001, 1250
    a = np.arange(na, dtype=np.int64)
    b = np.arange(na, na + nb, dtype=np.int64)
    h = na + nb
    gq = a.reshape(grp, 4)
    t = np.triu_indices(4, 1)
    s = np.concatenate([np.repeat(a, nb), np.full(na, h), gq[:, t[0]].ravel()]).astype(np.int32)
    d = np.concatenate([np.tile(b, na), a, gq[:, t[1]].ravel()]).astype(np.int32)
    with gpu.Graph.from_edges(s, d, h + 1) as g:
        for ns in (2, 3):
            assert sum(g.count_shard("5-clique", r, ns) for r in range(ns)) == grp * (1 + nb)


def test_shard_arguments(gpu, graph):
    g = graph[0]
    for args in (("4-clique", 2, 2), ("4-clique", -1, 2), ("P1", 0, 0)):
        with pytest.raises(gpu.JgpmError) as e:
            g.count_shard(*args)
        assert e.value.code == -1, args
