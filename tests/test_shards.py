"""CPU tests of the multi-GPU split with world_size 2 over gloo: each rank counts its shard of
the root arcs (here with the oracle, on CPU: root arcs rank, rank + 2, ..., the split rule of
jgpm_count_shard's nested-loop plans), one all-reduce sums the partial counts, and the sum
equals the one-process count; the time is the maximum over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle_api as O
        from jupiter_b200 import shards
        assert shards.world_and_rank() == (world, rank)
        g = O.rmat_graph(2000, 8, 0.57, 0.19, 0.19, 3)
        dag = O.orient(g)
        parts = [O.count("P0", dag, rank, dag.m, world, nthreads=1)[0],
                 O.count("P13", dag, rank, dag.m, world, nthreads=1)[0],
                 O.count("P1", g, rank, g.m, world, nthreads=1)[0]]
        total = shards.reduce_counts(parts, torch.device("cpu"))
        ms = shards.max_over_ranks(10.0 * (rank + 1), torch.device("cpu"))
        full = [O.count("P0", dag, nthreads=1)[0], O.count("P13", dag, nthreads=1)[0],
                O.count("P1", g, nthreads=1)[0]]
        q.put((rank, total, full, parts, ms))
    finally:
        dist.destroy_process_group()


def test_shards_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, full, parts, ms in res:
        assert total == full  # the shards' partial counts add up to the whole count
        assert ms == 20.0
    # each rank did a real share of the work (no rank counted everything)
    assert all(0 < a < f for a, f in zip(res[0][3], res[0][2]))


def test_overflowing_count_is_refused():
    import torch
    from jupiter_b200 import shards
    with pytest.raises(OverflowError):
        shards.reduce_counts([1 << 63], torch.device("cpu"))
