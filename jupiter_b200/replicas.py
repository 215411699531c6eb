"""Multi-GPU replica protocol: one process per GPU, each holding a full replica of the graph.

Every rank counts the whole workload on its own GPU (weak scaling: per-GPU work is fixed as
the number of GPUs grows), then the ranks exchange exactly one thing: the u64 counts, summed
with one all-reduce, which is the reference's final MPI_Reduce of the counts
(src/jupiter_gpm.cu:880-904).  Timing is the maximum over ranks.  The same functions run
over NCCL on GPUs and over gloo on CPU (the tests).
"""
import torch
import torch.distributed as dist


def _world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size()
    return 1


def reduce_counts(counts, device):
    """Sums a list of per-rank counts over all ranks with one all-reduce.  int64 carries every
    count below 2^63; a larger count raises OverflowError."""
    for c in counts:
        if c >= (1 << 63):
            raise OverflowError("count does not fit the int64 all-reduce")
    t = torch.tensor(list(counts), dtype=torch.int64, device=device)
    if _world() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [int(x) for x in t.tolist()]


def max_over_ranks(value, device):
    """The maximum of a float (a time in ms, say) over all ranks."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if _world() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def check_replicas(local_counts, device):
    """Every replica must produce the same counts: the summed counts equal world x local."""
    world = _world()
    total = reduce_counts(local_counts, device)
    if total != [world * c for c in local_counts]:
        raise RuntimeError(f"replica counts disagree: {total} vs {world} x {local_counts}")
    return total
