"""GPU parity of listing mode (jgpm_list) against brute-force listings of the patterns'
definitions on the small golden graphs: k-cliques and the vertex-induced patterns as vertex
sets, the reference's edge-induced 4-cycle (P1) and diamond (P2) as their exact tuples (a K4
holds three 4-cycles and six diamonds on the same four vertices).  On larger graphs the
listing holds exactly jgpm_count's number of distinct embeddings."""
import itertools

import numpy as np
import pytest

import graphs as G

pytestmark = pytest.mark.gpu

SMALL = ["K6", "K9", "C7", "C4", "S5", "K34", "W6", "petersen"]
SMALL_RMAT = [G.RMAT_SMALL[0], G.RMAT_SMALL[1], G.RMAT_SMALL[2]]  # n = 64, 100, 256


def adjacency(n, edges):
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    return adj


def cliques(adj, k):
    out = set()

    def grow(cl, cand):
        if len(cl) == k:
            out.add(tuple(sorted(cl)))
            return
        for v in sorted(cand):
            if v > cl[-1]:
                grow(cl + [v], cand & adj[v])
    for v in range(len(adj)):
        grow([v], adj[v])
    return out


def four_cycles(adj):  # (a, b, c, d): a the largest vertex, b > d its two cycle neighbours
    out = []
    for a in range(len(adj)):
        low = sorted(x for x in adj[a] if x < a)
        for b, d in itertools.combinations(low, 2):
            b, d = max(b, d), min(b, d)
            for c in sorted(adj[b] & adj[d]):
                if c < a:
                    out.append((a, b, c, d))
    return sorted(out)


def diamonds(adj):  # (u, v, w1, w2): the shared edge u > v, then w1 < w2
    out = []
    for u in range(len(adj)):
        for v in adj[u]:
            if v < u:
                w = sorted(adj[u] & adj[v])
                out += [(u, v, w1, w2) for w1, w2 in itertools.combinations(w, 2)]
    return sorted(out)


KINDS = {(3, (1, 1, 2, 2)): "4-path", (3, (1, 1, 1, 3)): "3-star",
         (4, (2, 2, 2, 2)): "4-cycle", (4, (1, 2, 2, 3)): "tailed-triangle",
         (5, (2, 2, 3, 3)): "diamond"}


def induced_all(adj):
    """Every 4-vertex subset, by the pattern its induced subgraph is (one pass)."""
    out = {k: set() for k in KINDS.values()}
    for s in itertools.combinations(range(len(adj)), 4):
        deg = tuple(sorted(sum(1 for y in s if y != x and y in adj[x]) for x in s))
        kind = KINDS.get((sum(deg) // 2, deg))
        if kind:
            out[kind].add(s)
    return out


def graph_cases(J):
    for name in SMALL:
        n, edges = G.NAMED[name]
        e = np.array(edges, dtype=np.int32).reshape(-1, 2)
        yield name, J.Graph.from_edges(e[:, 0], e[:, 1], n), n, edges
    for spec in SMALL_RMAT:
        g = J.Graph.rmat(*spec[1:])
        rowptr, col = g.csr()
        n = spec[1]
        src = np.repeat(np.arange(n), np.diff(rowptr))
        yield spec[0], g, n, [(int(a), int(b)) for a, b in zip(src, col) if a < b]


def test_listing_matches_brute_force(gpu):
    for name, g, n, edges in graph_cases(gpu):
        with g:
            adj = adjacency(n, edges)
            for k in (3, 4, 5):
                rows, total = g.list(f"k-clique:{k}")
                got = [tuple(sorted(r)) for r in rows.tolist()]
                assert len(got) == total == len(set(got)), (name, k)
                assert set(got) == cliques(adj, k), (name, k)
            rows, total = g.list("4-cycle")
            assert sorted(map(tuple, rows.tolist())) == four_cycles(adj), name
            rows, total = g.list("diamond")
            assert sorted(map(tuple, rows.tolist())) == diamonds(adj), name
            if n <= 64:
                want = induced_all(adj)
                for p in ("4-cycle", "diamond", "tailed-triangle", "4-path", "3-star"):
                    rows, total = g.list(p, induced=True)
                    got = [tuple(sorted(r)) for r in rows.tolist()]
                    assert len(got) == total == len(set(got)), (name, p)
                    assert set(got) == want[p], (name, p)


@pytest.mark.parametrize("pattern,induced", [("triangle", 0), ("4-clique", 0), ("5-clique", 0),
                                             ("k-clique:6", 0), ("4-cycle", 0), ("diamond", 0),
                                             ("tailed-triangle", 1), ("4-path", 1),
                                             ("3-star", 1), ("4-cycle", 1)])
def test_listing_size_and_uniqueness_match_count(gpu, pattern, induced):
    # the vertex-induced stars and paths number in the tens of millions at 4096 vertices
    n = 1024 if induced else 4096
    with gpu.Graph.rmat(n, 8, 0.57, 0.19, 0.19, 5) as g:
        rows, total = g.list(pattern, induced=bool(induced))
        assert total == g.count(pattern, induced=bool(induced)) == len(rows)
        key = rows if pattern in ("4-cycle", "diamond") and not induced else np.sort(rows, axis=1)
        assert len(np.unique(key, axis=0)) == total


def test_listing_truncates_to_capacity(gpu):
    with gpu.Graph.rmat(2000, 8, 0.57, 0.19, 0.19, 9) as g:
        full, total = g.list("4-clique")
        part, total2 = g.list("4-clique", capacity=10)
        assert total2 == total > 10 and len(part) == 10
        whole = {tuple(sorted(r)) for r in full.tolist()}
        assert all(tuple(sorted(r)) in whole for r in part.tolist())
        with pytest.raises(gpu.JgpmError) as e:
            g.list("P5")
        assert e.value.code == -5


def test_listing_into_device_memory(gpu):
    import ctypes
    import torch
    with gpu.Graph.rmat(2000, 8, 0.57, 0.19, 0.19, 9) as g:
        host, total = g.list("triangle")
        buf = torch.zeros((total, 3), dtype=torch.int32, device="cuda")
        t = ctypes.c_int64()
        rc = gpu.lib().jgpm_list(g._h, b"triangle", 0,
                                 ctypes.cast(buf.data_ptr(), ctypes.POINTER(ctypes.c_int32)),
                                 total, ctypes.byref(t), None)
        assert rc == 0 and t.value == total
        torch.cuda.synchronize()
        dev = buf.cpu().numpy()
        assert {tuple(sorted(r)) for r in dev.tolist()} == {tuple(sorted(r)) for r in host.tolist()}
