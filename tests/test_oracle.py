"""CPU tests: the oracle restatement against the golden fixtures (reference code + brute force),
closed forms and the induced/non-induced identities.  No GPU needed."""
import json
import math
import os

import numpy as np
import pytest

import graphs as G
import oracle_api as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_counts.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}
SMALL = [c["name"] for c in GOLDEN["cases"] if c["n"] <= 5000]


def csr_of(case):
    if case["kind"] == "named":
        return G.named_csr(case["name"])
    spec = (case["name"], case["n"], case["edge_factor"], case["a"], case["b"], case["c"],
            case["seed"])
    return G.rmat_csr(spec)


@pytest.mark.parametrize("name", SMALL + [G.RMAT_TRIANGLE[0]])
def test_orientation_matches_reference_loader(name):
    case = CASES[name]
    g = csr_of(case)
    assert G.csr_digest(g) == case["sym_digest"]
    assert G.csr_digest(O.orient(g)) == case["ref"]["dag_digest"]


@pytest.mark.parametrize("name", SMALL)
def test_oracle_plans_match_reference_code(name):
    case = CASES[name]
    g = csr_of(case)
    dag = O.orient(g)
    ref = case["ref"]
    for k, p in ((3, "P0"), (4, "P13"), (5, "P14"), (6, "P15"), (7, "P16")):
        if f"clique{k}" in ref:
            assert O.count(p, dag)[0] == ref[f"clique{k}"], (p, name)
    for p in ["P1", "P2"] + G.INDUCED:
        if p in ref:
            assert O.count(p, g)[0] == ref[p], (p, name)


def test_triangle_workload_matches_reference_code():
    case = CASES[G.RMAT_TRIANGLE[0]]
    g = csr_of(case)
    dag = O.orient(g)
    assert O.count("P0", dag)[0] == case["ref"]["clique3"]
    assert O.count("P13", dag)[0] == case["ref"]["clique4"]
    assert O.count("P2", g)[0] == case["ref"]["P2"]


@pytest.mark.parametrize("name", [c["name"] for c in GOLDEN["cases"] if "brute" in c])
def test_induced_plans_match_brute_force_census(name):
    case = CASES[name]
    g = csr_of(case)
    census = O.census4(g)
    assert census == case["brute"]["census4"]
    got = [O.count(p, g)[0] for p in G.INDUCED] + [O.count("P13", O.orient(g))[0]]
    assert got == census


def _plan_multiplicities():
    """Embeddings / plan count per pattern, over every brute-forced graph with copies."""
    ratios = {p: set() for p in G.NONCLIQUE_PLANS}
    for case in GOLDEN["cases"]:
        if "brute" not in case:
            continue
        g = csr_of(case)
        for p in G.NONCLIQUE_PLANS:
            emb = case["brute"]["embeddings"][p]
            c = O.count(p, g)[0]
            if c == 0:
                assert emb == 0, (p, case["name"])
            else:
                ratios[p].add(emb / c)
    return ratios


def test_reference_plans_count_a_fixed_multiple_of_embeddings():
    """Each reference plan counts every copy of its pattern the same number of times: the
    number of injective edge-preserving maps is a constant multiple of the plan's count."""
    ratios = _plan_multiplicities()
    expected = {}
    for p, (k, edges) in G.PATTERN_EDGES.items():
        aut = G.automorphisms(k, edges)
        assert len(ratios[p]) == 1, (p, ratios[p])
        r = ratios[p].pop()
        # the plan counts each subgraph aut/r times; r must divide |Aut|
        assert float(r).is_integer() and aut % int(r) == 0, (p, r, aut)
        expected[p] = aut // int(r)
    # every reference plan counts each edge-induced copy of its pattern exactly once, so
    # count = embeddings / |Aut(H)| (the number of subgraphs isomorphic to H)
    assert all(v == 1 for v in expected.values()), expected


@pytest.mark.parametrize("name,n", [("K6", 6), ("K9", 9)])
def test_cliques_closed_form(name, n):
    dag = O.orient(G.named_csr(name))
    for k, p in ((3, "P0"), (4, "P13"), (5, "P14"), (6, "P15"), (7, "P16")):
        assert O.count(p, dag)[0] == math.comb(n, k)


def test_closed_forms_cycles_stars_bipartite_wheel():
    assert O.count("P1", G.named_csr("C4"))[0] == 1
    assert O.count("P1", G.named_csr("K34"))[0] == math.comb(3, 2) * math.comb(4, 2)
    assert O.count("induced-3-star", G.named_csr("S5"))[0] == math.comb(5, 3)
    assert O.count("induced-4-path", G.named_csr("C7"))[0] == 7
    w = G.named_csr("W6")
    assert O.count("P0", O.orient(w))[0] == 6
    assert O.count("P1", w)[0] == 6  # 4-cycles of W6: hub + 3 consecutive rim vertices
    assert O.census4(G.named_csr("petersen"))[:2] == [10, 60]


def noninduced_closed_forms(g):
    deg = g.degrees().astype(object)
    dag = O.orient(g)
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    # triangles per undirected edge and per vertex
    adj = [set(g.col[g.rowptr[v]:g.rowptr[v + 1]].tolist()) for v in range(g.n)]
    te = {}
    for u, v in zip(src.tolist(), g.col.tolist()):
        if u < v:
            te[(u, v)] = len(adj[u] & adj[v])
    T = sum(te.values()) // 3
    tv = [0] * g.n
    for (u, v), t in te.items():
        tv[u] += t
        tv[v] += t
    tv = [x // 2 for x in tv]
    n_star = sum(math.comb(int(d), 3) for d in deg)
    n_tt = sum(tv[v] * (int(deg[v]) - 2) for v in range(g.n) if deg[v] >= 2)
    n_p4 = sum((int(deg[u]) - 1) * (int(deg[v]) - 1) for (u, v) in te) - 3 * T
    n_d = sum(math.comb(t, 2) for t in te.values())
    return {"star": n_star, "tt": n_tt, "p4": n_p4, "diamond": n_d,
            "c4": O.count("P1", g)[0], "k4": O.count("P13", dag)[0]}


@pytest.mark.parametrize("name", ["W6", "petersen", "K34", "rmat-n64-ef4-s1", "rmat-n100-ef8-s2",
                                  "rmat-n256-ef8-s3", "rmat-n1000-ef16-s4"])
def test_induced_noninduced_identities(name):
    """N(.) edge-induced, I(.) vertex-induced 4-vertex counts obey the standard identities;
    the GPU census uses exactly these to obtain I(.) at scale."""
    g = csr_of(CASES[name])
    N = noninduced_closed_forms(g)
    I = {p: O.count(p, g)[0] for p in G.INDUCED}
    iS, iP, iT, iC, iD = (I["induced-3-star"], I["induced-4-path"],
                          I["induced-tailed-triangle"], I["induced-4-cycle"],
                          I["induced-diamond"])
    iK = N["k4"]
    assert N["diamond"] == iD + 6 * iK
    assert N["diamond"] == O.count("P2", g)[0]
    assert N["c4"] == iC + iD + 3 * iK
    assert N["tt"] == iT + 4 * iD + 12 * iK
    assert N["star"] == iS + iT + 2 * iD + 4 * iK
    assert N["p4"] == iP + 2 * iT + 4 * iC + 6 * iD + 12 * iK


def test_oracle_elements_accounting():
    """Set-op elements of the canonical plans: level-1 ops add d+(u)+d+(v) for every arc."""
    g = G.named_csr("K6")
    dag = O.orient(g)
    deg = dag.degrees()
    src = np.repeat(np.arange(dag.n), deg)
    lvl1 = int(sum(deg[u] + deg[v] for u, v in zip(src, dag.col)))
    assert O.count("P0", dag)[1] == lvl1
    # P13 adds, for every triangle-edge candidate v2 in W, |W| + d+(v2)
    c, e = O.count("P13", dag)
    assert c == 15 and e > lvl1


def test_rmat_generator_restatements_agree():
    """The oracle's R-MAT restatement and the library's host generator give identical edges."""
    import jupiter_b200 as J
    for (n, ef, a, b, c, seed) in [(64, 4, 0.57, 0.19, 0.19, 1), (1000, 16, 0.45, 0.1375,
                                                                 0.1375, 7),
                                   (3000, 8, 0.6, 0.1, 0.1, 3), (1 << 12, 4, 0.57, 0.19, 0.19, 1)]:
        s1, d1 = O.rmat_edges(n, ef * n, a, b, c, seed)
        s2, d2 = J.rmat_edges(n, ef * n, a, b, c, seed)
        assert np.array_equal(s1, s2) and np.array_equal(d1, d2)
        assert s1.max() < n and d1.max() < n


def _split_cases(seed=3):
    rng = np.random.default_rng(seed)
    cases = []
    for na in (0, 1, 5, 31, 32, 33, 200, 3000):
        for nb in (0, 1, 7, 32, 65, 1000):
            u = max(3 * (na + nb), 4)
            cases.append((np.unique(rng.integers(0, u, na)).astype(np.int32),
                          np.unique(rng.integers(0, u, nb)).astype(np.int32)))
    x = np.arange(0, 500, 2, dtype=np.int32)
    cases += [(x, x), (x, x + 1), (x[:10], x), (x, x[-3:])]
    return cases


def test_oracle_fused_splits_match_set_algebra():
    """fuse_set and dif_int_set as restated: the set algebra on non-empty operands, and the
    reference's count 0 with nothing written when an operand is empty."""
    for i, (a, b) in enumerate(_split_cases()):
        r, c, d, e = O.fuse_set(a, b)
        if len(a) == 0 or len(b) == 0:
            assert r == 0 and c is None
        else:
            assert r == len(np.intersect1d(a, b))
            assert np.array_equal(c, np.setdiff1d(a, b))
            assert np.array_equal(d, np.intersect1d(a, b))
            assert np.array_equal(e, np.setdiff1d(b, a))
        for up in (None, int(a[len(a) // 2]) if len(a) else 0, 0):
            r, c, d = O.dif_int_set(a, b, up)
            if len(a) == 0 or len(b) == 0:
                assert r == 0 and c is None
                continue
            lim = np.iinfo(np.int32).max if up is None else up
            keep = (a < lim) & ~np.isin(a, b)
            assert r == keep.sum() and np.array_equal(c, a[keep]), (i, up)
            assert np.array_equal(d, a[~keep]), (i, up)


def test_reference_search_variants_are_exact():
    """The reference's search variants, restated, against a plain lookup: the cached two-phase
    search with 32 pivots (warp) and 256 (CTA) finds exactly the keys a list holds, at their
    positions (the index the map form marks), for every list size from 1 to 700 and several
    large ones; binary_search_bound is the lower bound on non-empty lists; the hash-bin
    intersection counts |A & B| while no bin overflows.  So the plain lookups here (binary
    lifting, merge path) give the same intersections and differences."""
    rng = np.random.default_rng(17)
    sizes = list(range(1, 701)) + [1000, 1023, 1024, 1025, 4096, 100_000, 1_000_000]
    for n in sizes:
        lst = np.unique(rng.integers(0, 3 * n + 8, 2 * n).astype(np.int32))[:n]
        keys = np.concatenate([lst, lst - 1, lst + 1, [lst[0] - 5, lst[-1] + 5]]).astype(np.int32)
        pos = np.searchsorted(lst, keys)
        want = (pos < len(lst)) & (lst[np.minimum(pos, len(lst) - 1)] == keys)
        for width in (32, 256):
            found, marked = O.search_2phase(lst, keys, width)
            assert np.array_equal(found, want), (n, width)
            assert np.array_equal(marked[want], pos[want]) and (marked[~want] == -1).all(), n
        assert np.array_equal(O.search_bound(lst, keys), pos), n
    # on an empty list binary_search_bound returns 1 for a positive key, not 0
    assert list(O.search_bound(np.zeros(0, np.int32), [5, 0, -3])) == [1, 0, 0]
    for na, nb in ((0, 10), (1, 1), (50, 3000), (3000, 50), (20000, 20000), (100000, 7)):
        a = np.unique(rng.integers(0, 4 * (na + nb) + 8, na)).astype(np.int32)
        b = np.unique(rng.integers(0, 4 * (na + nb) + 8, nb)).astype(np.int32)
        assert O.hindex_count(a, b) == len(np.intersect1d(a, b)), (na, nb)
    # more than 1,024 keys of one residue mod 128 overflow a bin
    assert O.hindex_count(np.arange(0, 128 * 1100, 128, dtype=np.int32),
                          np.arange(0, 128 * 1200, 128, dtype=np.int32)) == -1


def test_reference_count_smaller_is_exact_for_member_bounds():
    """The reference's count_smaller, restated: for a bound in the list it is the bound's rank, so
    the P2/P9 sum over every member of W is |W| (|W| - 1) / 2, the closed form the plans here
    use; for bounds not in the list its narrowing step (end = mid - 1) can miss one element."""
    rng = np.random.default_rng(23)
    off_by_one = 0
    for n in list(range(1, 400)) + [513, 1000, 2048, 5000]:
        w = np.unique(rng.integers(0, 3 * n + 8, 2 * n).astype(np.int32))[:n]
        ranks = [O.count_smaller(int(x), w) for x in w]
        assert ranks == list(range(len(w))), n
        assert sum(ranks) == len(w) * (len(w) - 1) // 2
        for x in rng.integers(-1, 3 * n + 9, 8):
            got, want = O.count_smaller(int(x), w), int(np.searchsorted(w, x))
            assert got in (want, want - 1), (n, x)
            off_by_one += got != want
    assert off_by_one > 0  # the quirk for bounds outside the list is real
