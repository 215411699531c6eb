"""CPU tests of the multi-GPU graph pool (jupiter_b200.pools): placement is deterministic,
balanced and within budget; with world_size 2 over gloo each rank serves the queries of its own
graphs (counted here by the oracle, on CPU), and the gathered per-query results equal the
one-process results of the whole trace."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GRAPHS = [(400 + 150 * i, 6, 100 + i) for i in range(7)]  # (n, edge factor, seed)
PATTERNS = [("P0", True), ("P13", True), ("P1", False), ("P2", False)]  # (plan, on the DAG)


def _trace(nq=60, seed=4):
    rng = np.random.default_rng(seed)
    w = np.arange(1, len(GRAPHS) + 1, dtype=np.float64) ** -1.1
    gids = rng.choice(len(GRAPHS), size=nq, p=w / w.sum())
    pats = [int(x) for x in rng.integers(len(PATTERNS), size=nq)]
    return gids, pats, w / w.sum()


def _placement(world):
    from jupiter_b200 import pools
    _, _, share = _trace()
    loads = [s * n * ef for s, (n, ef, _) in zip(share, GRAPHS)]
    nbytes = [n * ef * 16 for n, ef, _ in GRAPHS]
    return pools.place_graphs(loads, nbytes, world, budget_bytes=1 << 30)


def _serve(O, graphs, local_gids, pats):
    counts = []
    for g, p in zip(local_gids, pats):
        name, on_dag = PATTERNS[p]
        csr, dag = graphs[g]
        counts.append(O.count(name, dag if on_dag else csr, nthreads=1)[0])
    return counts


def _build(O, ids):
    out = []
    for i in ids:
        n, ef, seed = GRAPHS[i]
        g = O.rmat_graph(n, ef, 0.57, 0.19, 0.19, seed)
        out.append((g, O.orient(g)))
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    for p in (ROOT, os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle_api as O
        from jupiter_b200 import pools
        owner = _placement(world)
        gids, pats, _ = _trace()
        idx, local = pools.local_queries(gids, owner, rank)
        graphs = _build(O, pools.local_ids(owner, rank))
        counts = _serve(O, graphs, local, [pats[i] for i in idx])
        lat = [float(i) for i in idx]  # stands in for latencies: checks the merge order
        all_counts, all_lat, wall = pools.gather_results(len(gids), idx, counts, lat,
                                                         1.0 + rank)
        q.put((rank, list(map(int, owner)), len(idx), all_counts, list(all_lat), wall))
    finally:
        dist.destroy_process_group()


def test_placement_balanced_deterministic_and_within_budget():
    from jupiter_b200 import pools
    loads = [9.0, 7.0, 6.0, 5.0, 4.0, 3.0, 1.0]
    owner = pools.place_graphs(loads, [10] * 7, 2, budget_bytes=100)
    assert list(owner) == list(pools.place_graphs(loads, [10] * 7, 2, budget_bytes=100))
    per = [sum(l for l, o in zip(loads, owner) if o == r) for r in range(2)]
    assert abs(per[0] - per[1]) <= 1.0  # greedy longest-first: 17.5 each at best
    # the budget overrides the load: rank 0 holds at most 3 graphs of 10 bytes
    owner = pools.place_graphs(loads, [10] * 7, 3, budget_bytes=30)
    assert all((owner == r).sum() <= 3 for r in range(3))
    with pytest.raises(ValueError):
        pools.place_graphs([1.0, 1.0], [20, 20], 1, budget_bytes=30)
    idx, local = pools.local_queries([0, 3, 3, 6, 1], np.array([0, 1, 0, 1, 0, 0, 1]), 1)
    # rank 1 owns graphs 1, 3, 6, which its server numbers 0, 1, 2
    assert list(idx) == [1, 2, 3, 4] and list(local) == [1, 1, 2, 0]


def test_pool_two_ranks_gloo():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gids, pats, _ = _trace()
    want = _serve(O, _build(O, range(len(GRAPHS))), gids, pats)
    assert res[0][1] == res[1][1]  # both ranks placed the graphs alike
    assert 0 < res[0][2] < len(gids) and res[0][2] + res[1][2] == len(gids)
    for rank, owner, nmine, counts, lat, wall in res:
        assert counts == want  # every query answered once, by its graph's owner
        assert lat == [float(i) for i in range(len(gids))] and wall == 2.0
