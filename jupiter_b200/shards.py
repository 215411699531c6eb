"""Multi-GPU split of a count: one process per GPU, each holding the whole graph.

Rank r of w counts only its shard of the work (jgpm_count_shard: for k-cliques the roots of
every out-degree tier with index = r mod w, for the other patterns the root arcs r, r + w,
...), so the work per GPU shrinks as the number of GPUs grows (strong scaling).  The ranks
then exchange exactly one thing per count, a u64 partial sum, added up by one all-reduce:
the reference's split of the root edges over ranks (src/jupiter_gpm.cu:91-150) and its final
MPI_Reduce of the counts (:880-904).  Timing is the maximum over ranks.  The same functions
run over NCCL on GPUs and over gloo on CPU (the tests).
"""
import torch
import torch.distributed as dist


def world_and_rank():
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def count_local(graph, pattern, induced=False, details=False):
    """This rank's shard of the count of `pattern` on `graph` (a jupiter_b200.Graph)."""
    world, rank = world_and_rank()
    return graph.count_shard(pattern, rank, world, induced=induced, details=details)


def reduce_counts(partials, device):
    """Sums a list of per-rank partial counts over all ranks with one all-reduce.  int64
    carries every sum below 2^63; a larger partial raises OverflowError, and a total that
    wraps past 2^63 is caught by the check on the result."""
    for c in partials:
        if c < 0 or c >= (1 << 63):
            raise OverflowError("partial count does not fit the int64 all-reduce")
    t = torch.tensor(list(partials), dtype=torch.int64, device=device)
    if world_and_rank()[0] > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = [int(x) for x in t.tolist()]
    if any(x < 0 for x in out):
        raise OverflowError("summed count does not fit the int64 all-reduce")
    return out


def max_over_ranks(value, device):
    """The maximum of a float (a time in ms, say) over all ranks."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world_and_rank()[0] > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
