"""GPU parity tests: every count through the C-ABI equals the reference-code / brute-force
golden values and the oracle, bit for bit.  Run on a B200 with `pytest -m gpu`."""
import json
import os
import tempfile

import numpy as np
import pytest

import graphs as G
import oracle_api as O

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_counts.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}
SMALL = [c["name"] for c in GOLDEN["cases"] if c["n"] <= 5000]
PLAN_CASES = [c["name"] for c in GOLDEN["cases"] if c["n"] <= 1000]


def oracle_csr(case):
    if case["kind"] == "named":
        return G.named_csr(case["name"])
    return G.rmat_csr((case["name"], case["n"], case["edge_factor"], case["a"], case["b"],
                       case["c"], case["seed"]))


def gpu_graph(J, case):
    if case["kind"] == "named":
        e = np.array(case["edges"], dtype=np.int32).reshape(-1, 2)
        return J.Graph.from_edges(e[:, 0], e[:, 1], case["n"])
    return J.Graph.rmat(case["n"], case["edge_factor"], case["a"], case["b"], case["c"],
                        case["seed"])


@pytest.fixture(scope="module")
def graphs(gpu):
    out = {}
    for name in SMALL:
        out[name] = gpu_graph(gpu, CASES[name])
    yield out
    for g in out.values():
        g.close()


def digest(rowptr, col):
    return G.csr_digest(O.Csr(len(rowptr) - 1, rowptr, col))


@pytest.mark.parametrize("name", SMALL + [G.RMAT_TRIANGLE[0]])
def test_device_csr_and_orientation_match_reference(gpu, graphs, name):
    case = CASES[name]
    g = graphs[name] if name in graphs else gpu_graph(gpu, case)
    assert digest(*g.csr()) == case["sym_digest"]
    assert digest(*g.csr(dag=True)) == case["ref"]["dag_digest"]


@pytest.mark.parametrize("name", SMALL)
def test_cliques_match_reference_code(gpu, graphs, name):
    g = graphs[name]
    ref = CASES[name]["ref"]
    for k in (3, 4, 5, 6, 7):
        if f"clique{k}" in ref:
            assert g.count(f"k-clique:{k}") == ref[f"clique{k}"], (name, k)
    assert g.count("triangle") == ref["clique3"]
    assert g.count("P13") == ref["clique4"]
    assert g.count("P14") == ref["clique5"]


@pytest.mark.parametrize("name", SMALL)
def test_clique_literal_plans_and_elements(gpu, graphs, name):
    g = graphs[name]
    dag = O.orient(oracle_csr(CASES[name]))
    for p in ("P0", "P13", "P14", "P15", "P16"):
        oc, oe = O.count(p, dag)
        c, st = g.count(p, stats=True)
        assert c == oc and st["setop_elements"] == oe, (name, p, c, oc, st, oe)
        c2, st2 = g.count(p, stats=True, flags=gpu.COUNT_FORCE_PLAN)
        assert c2 == oc and st2["setop_elements"] == oe and st2["method"] == "plan"


@pytest.mark.parametrize("name", PLAN_CASES)
def test_reference_plans_match_oracle(gpu, graphs, name):
    g = graphs[name]
    sym = oracle_csr(CASES[name])
    for p in G.NONCLIQUE_PLANS:
        oc, oe = O.count(p, sym)
        c, st = g.count(p, stats=True)
        assert c == oc and st["setop_elements"] == oe, (name, p, c, oc, st["setop_elements"], oe)
        assert g.count(p, flags=gpu.COUNT_FORCE_PLAN) == oc


@pytest.mark.parametrize("name", SMALL)
def test_p1_p2_and_induced_match_reference_code(gpu, graphs, name):
    g = graphs[name]
    ref = CASES[name]["ref"]
    assert g.count("4-cycle") == ref["P1"]
    assert g.count("P2") == ref["P2"]
    for p in G.INDUCED:
        short = p.replace("induced-", "")
        assert g.count(short, induced=True) == ref[p], (name, p)
        assert g.count(short, induced=True, flags=gpu.COUNT_FORCE_ENUM) == ref[p], (name, p)


@pytest.mark.parametrize("name", SMALL)
def test_census4(gpu, graphs, name):
    g = graphs[name]
    ref = CASES[name]["ref"]
    want = [ref[p] for p in G.INDUCED] + [ref["clique4"]]
    assert g.census4() == want
    if "brute" in CASES[name]:
        assert want == CASES[name]["brute"]["census4"]


@pytest.mark.parametrize("name", ["W6", "petersen", "rmat-n100-ef8-s2", "rmat-n1000-ef16-s4"])
def test_edge_induced_closed_forms(gpu, graphs, name):
    from test_oracle import noninduced_closed_forms
    N = noninduced_closed_forms(oracle_csr(CASES[name]))
    g = graphs[name]
    assert g.count("3-star") == N["star"]
    assert g.count("tailed-triangle") == N["tt"]
    assert g.count("4-path") == N["p4"]
    assert g.count("diamond") == N["diamond"]
    assert g.count("4-cycle") == N["c4"]


def complete_graph(J, n):
    iu = np.triu_indices(n, 1)
    return J.Graph.from_edges(iu[0].astype(np.int32), iu[1].astype(np.int32), n)


def test_large_roots_complete_graph(gpu):
    """K_1101: every degree ties, so the DAG orders by id and roots 0..75 have out-degree
    above 1024 (the edge-rooted list tier); the other roots fill every bitmap tier.  All
    counts have closed forms."""
    from math import comb
    n = 1101
    with complete_graph(gpu, n) as g:
        assert g.count("triangle") == comb(n, 3)
        assert g.info()["max_out_degree"] == n - 1
        assert g.count("k-clique:3") == comb(n, 3)
        assert g.count("4-clique") == comb(n, 4)
        assert g.count("diamond") == comb(n, 2) * comb(n - 2, 2)
        assert g.count("4-cycle") == 3 * comb(n, 4)
        assert g.count("tailed-triangle") == n * comb(n - 1, 2) * (n - 3)
        assert g.count("3-star") == n * comb(n - 1, 3)
        assert g.count("4-path") == 12 * comb(n, 4)
        assert g.census4() == [0, 0, 0, 0, 0, comb(n, 4)]


def test_list_tier_crown(gpu):
    """Roots of out-degree above 4096 run on edge-rooted lists.  Crown graph: A = 5000
    vertices in 1250 disjoint K4s, B = 5001 vertices joined to all of A, and a hub h joined
    to all of A.  Degrees: a 5005, b 5000, h 5000, so h and every b point to all of A
    (out-degree 5000).  With g = 1250 groups: triangles 4g + 6g + 6g|B|, 4-cliques
    g + 4g + 4g|B|, 5-cliques g(1 + |B|), diamonds 3 (|A| + |A||B|) + 6g C(|B| + 3, 2)."""
    from math import comb
    na, nb, g = 5000, 5001, 1250
    a = np.arange(na, dtype=np.int64)
    b = np.arange(na, na + nb, dtype=np.int64)
    h = na + nb
    grp = a.reshape(g, 4)
    iu = np.triu_indices(4, 1)
    src = [np.repeat(a, nb), np.full(na, h), grp[:, iu[0]].ravel()]
    dst = [np.tile(b, na), a, grp[:, iu[1]].ravel()]
    s = np.concatenate(src).astype(np.int32)
    d = np.concatenate(dst).astype(np.int32)
    with gpu.Graph.from_edges(s, d, h + 1) as G_:
        assert G_.count("triangle") == 4 * g + 6 * g + 6 * g * nb
        assert G_.info()["max_out_degree"] == na
        assert G_.count("4-clique") == g + 4 * g + 4 * g * nb
        assert G_.count("5-clique") == g * (1 + nb)
        assert G_.count("diamond") == 3 * (na + na * nb) + 6 * g * comb(nb + 3, 2)


def test_large_roots_against_oracle(gpu):
    """A K_1040 planted on the first vertices of an R-MAT graph: large roots next to small
    ones, checked against the oracle."""
    base = G.rmat_csr(("plant", 3000, 8, 0.57, 0.19, 0.19, 7))
    src = np.repeat(np.arange(base.n, dtype=np.int64), np.diff(base.rowptr)).astype(np.int32)
    iu = np.triu_indices(1040, 1)
    s = np.concatenate([src, iu[0].astype(np.int32)])
    d = np.concatenate([base.col.astype(np.int32), iu[1].astype(np.int32)])
    with gpu.Graph.from_edges(s, d, base.n) as g:
        rowptr, col = g.csr()
        sym = O.Csr(len(rowptr) - 1, rowptr, col)
        dag = O.orient(sym)
        assert g.count("triangle") == O.count("P0", dag)[0]
        assert g.info()["max_out_degree"] > 1024
        # edge-triangle diamond count against the literal P2 plan (no large-root tiers)
        assert g.count("diamond") == g.count("P2", flags=gpu.COUNT_FORCE_PLAN)


def c4_slab_graphs():
    """R-MAT graphs whose large 4-cycle apexes cover the slab forms: 2^18 vertices (two and
    three slices, 8- and 16-bit counters) and 2^20 (up to eleven slices: the heavy top-ranked
    apexes sweep them, the light ones count in dense arrays)."""
    return [(1 << 18, 8, 0.6, 0.1, 0.1, 11), (1 << 20, 4, 0.6, 0.1, 0.1, 11)]


def bipartite_2n(J, N):
    """K_{2,N}: hubs 0 and 1 joined to the leaves 2 .. N+1."""
    leaves = np.arange(2, N + 2, dtype=np.int32)
    s = np.concatenate([np.zeros(N, np.int32), np.ones(N, np.int32)])
    return J.Graph.from_edges(s, np.concatenate([leaves, leaves]), N + 2)


def test_c4_slab_slices_and_dense_apexes(gpu):
    for spec in c4_slab_graphs():
        sym = O.rmat_graph(*spec)
        with gpu.Graph.rmat(*spec) as g:
            assert g.count("4-cycle") == O.count("P1", sym)[0], spec


def test_c4_slab_wide_counters(gpu):
    """K_{2,N} with N = 70000: the top hub has N lower-ranked neighbours (32-bit counters,
    69 blocks of 1024 neighbours, two slices, every wedge in the second).  C4 = C(N, 2)."""
    from math import comb
    N = 70000
    with bipartite_2n(gpu, N) as g:
        assert g.count("4-cycle") == comb(N, 2)


@pytest.mark.parametrize("pattern", ["triangle", "4-clique", "5-clique", "P1", "P2", "P7"])
def test_rounds_do_not_change_counts(gpu, graphs, pattern):
    g = graphs["rmat-n4096-ef8-s5"]
    base = g.count(pattern)
    for rounds in (2, 3, 7):
        assert g.count(pattern, chunk_size=rounds) == base


def test_triangle_workload_full_size(gpu):
    case = CASES[G.RMAT_TRIANGLE[0]]
    with gpu_graph(gpu, case) as g:
        ref = case["ref"]
        assert g.count("triangle") == ref["clique3"]
        assert g.count("4-clique") == ref["clique4"]
        assert g.count("5-clique") == ref["clique5"]
        assert g.count("diamond") == ref["P2"]
        assert g.count("diamond", induced=True) == ref["induced-diamond"]
        assert g.count("tailed-triangle", induced=True) == ref["induced-tailed-triangle"]
        # diamond = sum_e C(t_e, 2) also through the literal plan
        assert g.count("P2", flags=gpu.COUNT_FORCE_PLAN) == ref["P2"]


def test_clique_workload_full_size(gpu):
    """The k-clique workload (R-MAT scale 22, edge factor 4): counts equal the reference's
    own code, and the set-op elements of the canonical plan are self-consistent."""
    case = CASES[G.RMAT_CLIQUE[0]]
    with gpu_graph(gpu, case) as g:
        ref = case["ref"]
        assert digest(*g.csr(dag=True)) == ref["dag_digest"]
        assert g.count("triangle") == ref["clique3"]
        c4, st4 = g.count("4-clique", stats=True)
        c5, st5 = g.count("5-clique", stats=True)
        assert c4 == ref["clique4"] and c5 == ref["clique5"]
        assert st4["setop_elements"] < st5["setop_elements"]
        assert g.count("4-clique", chunk_size=5) == ref["clique4"]


def test_reference_file_round_trip(gpu):
    case = CASES["rmat-n1000-ef16-s4"]
    sym = oracle_csr(case)
    with tempfile.TemporaryDirectory() as d:
        prefix = os.path.join(d, "g")
        O.write_reference_files(sym, prefix)
        with gpu.Graph.load(prefix) as g:
            assert digest(*g.csr()) == case["sym_digest"]
            assert g.count("P13") == case["ref"]["clique4"]
            g.save(os.path.join(d, "h"))
        for ext in (".vertex.bin", ".edge.bin"):
            assert open(prefix + ext, "rb").read() == open(os.path.join(d, "h") + ext, "rb").read()
        with gpu.Graph.load(os.path.join(d, "h"), use_dag=True) as g2:
            assert g2.count("triangle") == case["ref"]["clique3"]


def test_malformed_csr_rejected(gpu):
    ok_rowptr = np.array([0, 2, 4, 6], dtype=np.int64)
    ok_col = np.array([1, 2, 0, 2, 0, 1], dtype=np.int32)
    with gpu.Graph.from_csr(ok_rowptr, ok_col) as g:
        assert g.count("triangle") == 1
    bad = [
        (ok_rowptr, np.array([2, 1, 0, 2, 0, 1], dtype=np.int32)),      # unsorted row
        (ok_rowptr, np.array([1, 2, 0, 2, 0, 3], dtype=np.int32)),      # id out of range
        (ok_rowptr, np.array([0, 2, 0, 2, 0, 1], dtype=np.int32)),      # self-loop
        (np.array([0, 2, 3, 4], dtype=np.int64), np.array([1, 2, 0, 1], dtype=np.int32)),
        # ^ asymmetric: 2 lists 1, but 1 does not list 2
        (np.array([0, 3, 2, 6], dtype=np.int64), ok_col),               # decreasing rowptr
        (np.array([0, 2, 4, 5], dtype=np.int64), ok_col),               # rowptr[n] != m
        (ok_rowptr, np.array([1, 2, 0, 2, 1, 1], dtype=np.int32)),      # duplicate / asymmetric
    ]
    for rp, col in bad:
        with pytest.raises(gpu.JgpmError) as e:
            gpu.Graph.from_csr(rp, col)
        assert e.value.code == -1
    with pytest.raises(gpu.JgpmError) as e:
        gpu.Graph.from_edges(np.array([0, 5]), np.array([1, 1]), 3)
    assert e.value.code == -1


def test_unknown_pattern(gpu, graphs):
    g = graphs["K6"]
    for p, ind in (("P17", 0), ("hexagon", 0), ("P5", 1), ("k-clique:9", 0)):
        with pytest.raises(gpu.JgpmError) as e:
            g.count(p, induced=ind)
        assert e.value.code == -5


def _np_setop(op, a, b, upper, exclude, J):
    a = np.asarray(a)
    b = np.asarray(b)
    ap = a[a < upper]
    bp = b[b < upper]
    if op in (J.OP_INTERSECT, J.OP_INTERSECT_COUNT):
        r = np.intersect1d(ap, bp)
        if op == J.OP_INTERSECT_COUNT:
            r = r[r != exclude]
    else:
        r = np.setdiff1d(ap, bp)
        r = r[r != exclude]
    return r


def test_setops_match_numpy(gpu):
    J = gpu
    rng = np.random.default_rng(7)
    sizes = [0, 1, 31, 32, 33, 100, 1000, 100000]
    cases = []
    for na in sizes:
        for nb in sizes:
            if na * nb > 2_000_000_000:
                continue
            universe = max(4 * (na + nb), 8)
            a = np.unique(rng.integers(0, universe, na)).astype(np.int32)
            b = np.unique(rng.integers(0, universe, nb)).astype(np.int32)
            cases.append((a, b))
    # extreme ratio 1 : 10^4 and identical lists
    big = np.unique(rng.integers(0, 10**6, 200000)).astype(np.int32)
    cases.append((big[::10000].copy(), big))
    cases.append((big, big))
    for op in (J.OP_INTERSECT, J.OP_INTERSECT_COUNT, J.OP_DIFFERENCE, J.OP_DIFFERENCE_COUNT):
        a_l = [c[0] for c in cases]
        b_l = [c[1] for c in cases]
        ups = np.array([rng.integers(0, 2 * (int(c[0].max(initial=1)) + 1)) if i % 3 == 0
                        else np.iinfo(np.int32).max for i, c in enumerate(cases)], dtype=np.int32)
        exs = np.array([int(c[0][len(c[0]) // 2]) if (len(c[0]) and i % 2) else -1
                        for i, c in enumerate(cases)], dtype=np.int32)
        res = J.setop_batch(op, a_l, b_l, upper=ups, exclude=exs)
        for i, (a, b) in enumerate(cases):
            ex = exs[i] if op != J.OP_INTERSECT else -1
            want = _np_setop(op, a, b, ups[i], ex, J)
            if op in (J.OP_INTERSECT, J.OP_DIFFERENCE):
                assert res[0][i] == len(want) and np.array_equal(res[1][i], want), (op, i)
            else:
                assert res[i] == len(want), (op, i, len(a), len(b))
        # single-op entry point agrees
        a, b = cases[len(cases) // 2]
        one = J.setop(op, a, b)
        want = _np_setop(op, a, b, np.iinfo(np.int32).max, -1, J)
        if op in (J.OP_INTERSECT_COUNT, J.OP_DIFFERENCE_COUNT):
            assert one == len(want)
        else:
            assert np.array_equal(one, want)


def _split_pairs(rng):
    sizes = [0, 1, 31, 32, 33, 100, 1000, 100000]
    cases = []
    for na in sizes:
        for nb in sizes:
            universe = max(4 * (na + nb), 8)
            cases.append((np.unique(rng.integers(0, universe, na)).astype(np.int32),
                          np.unique(rng.integers(0, universe, nb)).astype(np.int32)))
    big = np.unique(rng.integers(0, 10**6, 200000)).astype(np.int32)
    cases += [(big[::10000].copy(), big), (big, big[::10000].copy()), (big, big)]
    return cases


def test_fused_splits_match_oracle(gpu):
    """fuse_set / dif_int_set through the C-ABI against the oracle's restatement.  Where an
    operand is empty the reference returns 0 and writes nothing; the entry points give the
    set algebra there (documented in the header), checked against numpy."""
    J = gpu
    rng = np.random.default_rng(11)
    cases = _split_pairs(rng)
    a_l = [c[0] for c in cases]
    b_l = [c[1] for c in cases]
    counts, out = J.setop_split_batch(J.SPLIT_FUSE, a_l, b_l)
    for i, (a, b) in enumerate(cases):
        c, d, e = out[i]
        if len(a) and len(b):
            r, oc, od, oe = O.fuse_set(a, b)
        else:
            r, oc, od, oe = 0, a, np.zeros(0, np.int32), b
        assert counts[i] == r, (i, len(a), len(b))
        assert np.array_equal(c, oc) and np.array_equal(d, od) and np.array_equal(e, oe), i
    ups = np.array([np.iinfo(np.int32).max if i % 3 == 0 else
                    int(rng.integers(0, 2 * (int(a.max(initial=1)) + 1)))
                    for i, (a, _) in enumerate(cases)], dtype=np.int32)
    counts, out = J.setop_split_batch(J.SPLIT_DIF_INT, a_l, b_l, upper=ups)
    for i, (a, b) in enumerate(cases):
        c, d, e = out[i]
        up = None if ups[i] == np.iinfo(np.int32).max else int(ups[i])
        if len(a) and len(b):
            r, oc, od = O.dif_int_set(a, b, up)
        else:
            keep = (a < ups[i]) if up is not None else np.ones(len(a), bool)
            r, oc, od = int(keep.sum()), a[keep], a[~keep]
        assert counts[i] == r and e is None, (i, len(a), len(b))
        assert np.array_equal(c, oc) and np.array_equal(d, od), i
    # the single-pair entry point agrees with the batch
    a, b = cases[len(cases) // 2 + 3]
    r, c, d, e = J.setop_split(J.SPLIT_FUSE, a, b)
    r0, oc, od, oe = O.fuse_set(a, b)
    assert r == r0 and np.array_equal(c, oc) and np.array_equal(d, od) and np.array_equal(e, oe)


def test_fused_split_device_arrays_and_untouched_entries(gpu):
    """Device operands and outputs are used in place; entries the sizes leave unwritten keep
    their contents, for host and device outputs alike."""
    import ctypes
    import torch
    J = gpu
    rng = np.random.default_rng(5)
    a = np.unique(rng.integers(0, 5000, 1500)).astype(np.int32)
    b = np.unique(rng.integers(0, 5000, 900)).astype(np.int32)
    P32 = ctypes.POINTER(ctypes.c_int32)
    P64 = ctypes.POINTER(ctypes.c_int64)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    ao = torch.tensor([0, len(a)], dtype=torch.int64, device="cuda")
    bo = torch.tensor([0, len(b)], dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    dc = torch.full((len(a),), -7, dtype=torch.int32, device="cuda")
    dd = torch.full((len(a),), -7, dtype=torch.int32, device="cuda")
    de = torch.full((len(b),), -7, dtype=torch.int32, device="cuda")
    ptr = lambda t, p: ctypes.cast(t.data_ptr(), p)  # noqa: E731
    rc = J.lib().jgpm_setop_split_batch(J.SPLIT_FUSE, ptr(da, P32), ptr(ao, P64), ptr(db, P32),
                                        ptr(bo, P64), 1, None, ptr(cnt, P32), ptr(dc, P32),
                                        ptr(dd, P32), ptr(de, P32))
    assert rc == 0
    torch.cuda.synchronize()
    r, oc, od, oe = O.fuse_set(a, b)
    assert int(cnt.item()) == r
    c, d, e = dc.cpu().numpy(), dd.cpu().numpy(), de.cpu().numpy()
    assert np.array_equal(c[: len(oc)], oc) and (c[len(oc):] == -7).all()
    assert np.array_equal(d[:r], od) and (d[r:] == -7).all()
    assert np.array_equal(e[: len(oe)], oe) and (e[len(oe):] == -7).all()
    hc = np.full(len(a), -9, np.int32)
    hd = np.full(len(a), -9, np.int32)
    n = ctypes.c_int32()
    rc = J.lib().jgpm_setop_split(J.SPLIT_DIF_INT, a.ctypes.data_as(P32), len(a),
                                  b.ctypes.data_as(P32), len(b), 2500, hc.ctypes.data_as(P32),
                                  hd.ctypes.data_as(P32), None, ctypes.byref(n))
    assert rc == 0
    r, oc, od = O.dif_int_set(a, b, 2500)
    assert n.value == r and np.array_equal(hc[:r], oc) and (hc[r:] == -9).all()
    assert np.array_equal(hd[: len(od)], od) and (hd[len(od):] == -9).all()
