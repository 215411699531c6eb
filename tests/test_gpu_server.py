"""GPU tests of the serving layer: exact counts through continuous batching, the same alone
and in the mix; admission and the memory-budgeted pool (eviction and re-upload)."""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

PATTERNS = ["triangle", "4-clique", "5-clique", "diamond", "4-cycle"]
ORACLE = {"triangle": ("P0", True), "4-clique": ("P13", True), "5-clique": ("P14", True),
          "diamond": ("P2", False), "4-cycle": ("P1", False)}
SPECS = [(1 << 12, 8, 7), (3000, 16, 8), (1 << 13, 4, 9), (1500, 32, 10)]


@pytest.fixture(scope="module")
def expected():
    want = {}
    for gi, (n, ef, seed) in enumerate(SPECS):
        sym = O.rmat_graph(n, ef, 0.57, 0.19, 0.19, seed)
        dag = O.orient(sym)
        for p in PATTERNS:
            name, use_dag = ORACLE[p]
            want[(gi, p)] = O.count(name, dag if use_dag else sym)[0]
    return want


def make_server(J, budget=8 << 30, inflight=3, batch=16):
    s = J.Server(memory_budget_bytes=budget, max_inflight=inflight, max_batch=batch)
    ids = [s.add_graph(J.Graph.rmat(n, ef, 0.57, 0.19, 0.19, seed)) for (n, ef, seed) in SPECS]
    return s, ids


def test_served_counts_exact_alone_and_in_mix(gpu, expected):
    s, ids = make_server(gpu)
    with s:
        # alone: one query at a time
        alone = {}
        for gi in ids:
            for p in PATTERNS:
                c, lat = s.wait(s.submit(gi, p))
                assert c == expected[(gi, p)]
                alone[(gi, p)] = c
        # in the mix: many queries in flight at once, in an interleaved order
        rng = np.random.default_rng(1)
        qs = [(int(rng.integers(len(ids))), PATTERNS[int(rng.integers(len(PATTERNS)))])
              for _ in range(120)]
        tickets = [s.submit(g, p) for g, p in qs]
        for (g, p), t in zip(qs, tickets):
            c, lat = s.wait(t)
            assert c == alone[(g, p)] and lat >= 0.0
        st = s.stats()
        assert st["completed"] == len(ids) * len(PATTERNS) + 120
        assert st["mean_batch"] > 1.0  # queries were actually packed together


def test_pool_evicts_and_restores_under_a_tight_budget(gpu, expected):
    J = gpu
    sizes = []
    for (n, ef, seed) in SPECS:
        with J.Graph.rmat(n, ef, 0.57, 0.19, 0.19, seed) as g:
            g.count("triangle")  # builds the DAG and root tiers, as the pool does
            sizes.append(g.info()["device_bytes"])
    # room for the two largest graphs, not for all four
    budget = sum(sorted(sizes)[-2:]) + 4096
    s = J.Server(memory_budget_bytes=budget, max_inflight=2, max_batch=4)
    ids = [s.add_graph(J.Graph.rmat(n, ef, 0.57, 0.19, 0.19, seed)) for (n, ef, seed) in SPECS]
    with s:
        for rep in range(2):
            for gi in ids:
                for p in ("triangle", "diamond", "4-clique"):
                    c, _ = s.wait(s.submit(gi, p))
                    assert c == expected[(gi, p)]
        st = s.stats()
        assert st["evictions"] > 0 and st["restores"] > 0


def test_admission_rejects_what_can_never_fit(gpu):
    J = gpu
    s = J.Server(memory_budget_bytes=64 << 20, max_inflight=1, max_batch=4)
    with s:
        gid = s.add_graph(J.Graph.rmat(1 << 15, 16, 0.57, 0.19, 0.19, 3))
        with pytest.raises(J.JgpmError) as e:
            s.submit(gid, "4-cycle")  # dense 4-cycle counters exceed the budget
        assert e.value.code == -11
        assert s.stats()["rejected"] == 1
        c, _ = s.wait(s.submit(gid, "triangle"))
        assert c > 0


def test_wait_timeout_and_unknown_ticket(gpu):
    s, ids = make_server(gpu)
    with s:
        with pytest.raises(gpu.JgpmError) as e:
            s.wait(123456, timeout_ms=10)
        assert e.value.code == -12
        with pytest.raises(gpu.JgpmError) as e:
            s.submit(ids[0], "P99")
        assert e.value.code == -5


def test_replay_server_and_plain_agree(gpu, expected):
    s, ids = make_server(gpu)
    with s:
        rng = np.random.default_rng(5)
        n = 200
        arr = np.cumsum(rng.exponential(1.0 / 2000.0, n))
        gids = rng.integers(len(ids), size=n)
        pats = [PATTERNS[int(x)] for x in rng.integers(len(PATTERNS), size=n)]
        c1, lat1, w1 = s.replay(gids, pats, arr)
        c2, lat2, w2 = s.replay(gids, pats, arr, plain=True)
        assert c1 == c2
        for g, p, c in zip(gids, pats, c1):
            assert c == expected[(int(g), p)]
        assert (lat1 >= 0).all() and (lat2 >= 0).all()


def test_plain_lane_patterns(gpu):
    """Non-batchable patterns (vertex-induced diamond, reference P3..P12) run on the plain
    lane, concurrently with batches (which also carry the batchable vertex-induced tailed
    triangle), and give the plain counts."""
    n, ef, seed = SPECS[0]
    sym = O.rmat_graph(n, ef, 0.57, 0.19, 0.19, seed)
    want_tt = O.count("induced-tailed-triangle", sym)[0]
    want_d = O.count("induced-diamond", sym)[0]
    want_p7 = O.count("P7", sym)[0]
    want_tri = O.count("P0", O.orient(sym))[0]
    s, ids = make_server(gpu)
    with s:
        ts = []
        for _ in range(5):
            ts.append(("tt", s.submit(ids[0], "induced:tailed-triangle")))
            ts.append(("d", s.submit(ids[0], "induced:diamond")))
            ts.append(("tri", s.submit(ids[0], "triangle")))
            ts.append(("p7", s.submit(ids[0], "P7")))
        for kind, t in ts:
            c, _ = s.wait(t)
            assert c == {"tt": want_tt, "d": want_d, "tri": want_tri, "p7": want_p7}[kind]
        with pytest.raises(gpu.JgpmError) as e:
            s.submit(ids[0], "induced:P7")
        assert e.value.code == -5


def test_plain_lane_budget_covers_literal_plan_scratch(gpu):
    """A literal-plan query (P3) on a graph with a hub allocates per-warp candidate lists of
    the maximum degree (up to 2 GiB) while it runs.  Admission counts them: with a budget
    that holds the graph but not those lists the query is refused, with room for them it runs
    and the admitted frontier covers them."""
    J = gpu
    hub = 60000
    src = np.concatenate([np.zeros(hub, np.int32), np.arange(1, hub, dtype=np.int32)])
    dst = np.concatenate([np.arange(1, hub + 1, dtype=np.int32),
                          np.arange(2, hub + 1, dtype=np.int32)])
    lists = 2 << 30  # 2 GiB: the literal kernel's cap for a maximum degree of 60,000
    tight = J.Server(memory_budget_bytes=1 << 30, max_inflight=1, max_batch=4)
    with tight:
        gid = tight.add_graph(J.Graph.from_edges(src, dst, hub + 1))
        with pytest.raises(J.JgpmError) as e:
            tight.submit(gid, "P3")
        assert e.value.code == -11
    roomy = J.Server(memory_budget_bytes=4 << 30, max_inflight=1, max_batch=4)
    with roomy:
        gid = roomy.add_graph(J.Graph.from_edges(src, dst, hub + 1))
        resident = roomy.stats()["resident_bytes"]  # at admission (the lists come later)
        c, _ = roomy.wait(roomy.submit(gid, "P3"))
        sym = O.build_csr(hub + 1, src, dst)
        assert c == O.count("P3", sym)[0]
        st = roomy.stats()
        assert st["peak_frontier_bytes"] >= lists
        assert st["peak_frontier_bytes"] + resident <= 4 << 30


def test_light_queries_do_not_wait_behind_heavy_ones(gpu, expected):
    """Shortest estimated work first: with one slot and one query per batch, a heavy query
    (4-cycle on the largest graph) queued behind a blocker and ahead of light ones (triangles
    on a small graph) runs after them; every count stays exact."""
    import time
    J = gpu
    s = J.Server(memory_budget_bytes=8 << 30, max_inflight=1, max_batch=1)
    with s:
        big = s.add_graph(J.Graph.rmat(1 << 16, 16, 0.57, 0.19, 0.19, 31))
        small = s.add_graph(J.Graph.rmat(1 << 11, 4, 0.57, 0.19, 0.19, 32))
        t0 = time.perf_counter()
        blocker = s.submit(big, "5-clique")
        heavy = s.submit(big, "4-cycle")
        light = [s.submit(small, "triangle") for _ in range(6)]
        c_heavy, lat_heavy = s.wait(heavy)
        done_heavy = lat_heavy  # latencies are measured from each query's own submission
        lights = [s.wait(t) for t in light]
        s.wait(blocker)
        sym = O.rmat_graph(1 << 11, 4, 0.57, 0.19, 0.19, 32)
        want = O.count("P0", O.orient(sym))[0]
        assert all(c == want for c, _ in lights)
        assert c_heavy == O.count("P1", O.rmat_graph(1 << 16, 16, 0.57, 0.19, 0.19, 31))[0]
        # submissions were microseconds apart: compare completion order through latencies
        assert max(lat for _, lat in lights) < done_heavy, (lights, done_heavy)
        assert time.perf_counter() - t0 < 60


def test_graph_pool_split_over_two_servers(gpu, expected):
    """The multi-GPU pool's placement and routing (jupiter_b200.pools) with two servers on one
    device standing in for two GPUs (the servers never wait on each other): each serves the
    queries of its own graphs, and the merged results equal the oracle for every query."""
    from jupiter_b200 import pools
    J = gpu
    loads = [n * ef for n, ef, _ in SPECS]
    owner = pools.place_graphs(loads, [16 * n * ef for n, ef, _ in SPECS], 2, 8 << 30)
    assert sorted(set(owner.tolist())) == [0, 1]
    rng = np.random.default_rng(2)
    gids = rng.integers(len(SPECS), size=80)
    pats = [PATTERNS[int(x)] for x in rng.integers(len(PATTERNS), size=80)]
    arr = np.cumsum(rng.exponential(1e-3, 80))
    parts = []
    for r in range(2):
        s = J.Server(memory_budget_bytes=8 << 30, max_inflight=3, max_batch=16)
        with s:
            for g in pools.local_ids(owner, r):
                n, ef, seed = SPECS[g]
                s.add_graph(J.Graph.rmat(n, ef, 0.57, 0.19, 0.19, seed))
            idx, loc = pools.local_queries(gids, owner, r)
            c, lat, wall = s.replay(loc, [pats[i] for i in idx], arr[idx])
            parts.append((idx, c, lat, wall))
    counts, lat, wall = pools.merge_results(len(gids), parts)
    assert counts == [expected[(int(g), p)] for g, p in zip(gids, pats)]
    assert not np.isnan(lat).any() and wall == max(p[3] for p in parts)
