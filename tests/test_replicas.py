"""CPU tests of the multi-GPU replica protocol with world_size 2 over gloo: each rank counts a
full replica (here with the oracle, on CPU), the counts are summed by one all-reduce and the
time is the maximum over ranks."""
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
        from jupiter_b200 import replicas
        g = O.rmat_graph(2000, 8, 0.57, 0.19, 0.19, 3)
        dag = O.orient(g)
        c3 = O.count("P0", dag, nthreads=1)[0]
        c4 = O.count("P13", dag, nthreads=1)[0]
        total = replicas.check_replicas([c3, c4], torch.device("cpu"))
        ms = replicas.max_over_ranks(10.0 * (rank + 1), torch.device("cpu"))
        bad = None  # a replica that disagrees is detected on every rank
        try:
            replicas.check_replicas([c3 + rank, c4], torch.device("cpu"))
        except RuntimeError as e:
            bad = str(e)
        q.put((rank, total, ms, c3, c4, bad))
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, ms, c3, c4, bad in res:
        assert total == [2 * c3, 2 * c4]
        assert ms == 20.0
        assert bad is not None and "disagree" in bad


def test_overflowing_count_is_refused():
    import torch
    from jupiter_b200 import replicas
    with pytest.raises(OverflowError):
        replicas.reduce_counts([1 << 63], torch.device("cpu"))
