"""Multi-GPU serving: the graph pool spread over one server per GPU.

One process per GPU, each with its own server (jupiter_b200.Server) on its own device.  Every
rank computes the same placement of the pool's graphs from the same inputs, so placing them
takes no message: the graphs go, heaviest expected load first, each to the rank with the least
load so far that still has memory for it (greedy longest-first).  A query runs on the rank that
owns its graph, since a query needs all of its graph and the graphs are independent.  For a
replayed open-loop trace every rank takes the queries of its own graphs, keeps their arrival
times, and replays them through its own server; one all-gather then brings the per-query
results to every rank.  This is the served counterpart of the reference's split of work over
ranks (src/jupiter_gpm.cu:91-150): there one graph's root edges are split, here whole graphs are
placed.  The same functions run over NCCL on GPUs and over gloo on CPU (the tests).
"""
import numpy as np
import torch.distributed as dist

from .shards import world_and_rank


def place_graphs(loads, nbytes, world, budget_bytes):
    """Owner rank of every graph.  loads[i]: expected work of graph i (its share of the queries
    x the work of one query); nbytes[i]: its resident bytes; budget_bytes: what one rank may
    hold.  Deterministic: ties go to the lower graph index and the lower rank.  Raises
    ValueError when a graph fits no rank."""
    loads = np.asarray(loads, dtype=np.float64)
    nbytes = np.asarray(nbytes, dtype=np.int64)
    if world < 1 or len(loads) != len(nbytes):
        raise ValueError("place_graphs: bad arguments")
    order = sorted(range(len(loads)), key=lambda i: (-loads[i], i))
    load = np.zeros(world, dtype=np.float64)
    held = np.zeros(world, dtype=np.int64)
    owner = np.full(len(loads), -1, dtype=np.int32)
    for i in order:
        fits = [r for r in range(world) if held[r] + nbytes[i] <= budget_bytes]
        if not fits:
            raise ValueError(f"graph {i} ({int(nbytes[i])} bytes) fits no rank's budget")
        r = min(fits, key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += loads[i]
        held[r] += nbytes[i]
    return owner


def local_ids(owner, rank):
    """The global ids of the graphs `rank` owns, in ascending order; a rank's server numbers
    them 0, 1, ... in this order."""
    return [int(g) for g in np.flatnonzero(np.asarray(owner) == rank)]


def local_queries(graph_ids, owner, rank):
    """Indices of the trace's queries whose graph `rank` owns, and those queries' graph ids
    renumbered to the rank's server."""
    gids = np.asarray(graph_ids)
    idx = np.flatnonzero(np.asarray(owner)[gids] == rank)
    remap = {g: i for i, g in enumerate(local_ids(owner, rank))}
    return idx, np.array([remap[int(g)] for g in gids[idx]], dtype=np.int32)


def merge_results(n, parts):
    """Per-query counts and latencies of the whole trace (n queries) from the ranks' shares,
    each (query indices, counts, latencies in ms, wall seconds), and the longest wall time."""
    all_counts = [None] * n
    all_lat = np.full(n, np.nan, dtype=np.float64)
    wall = 0.0
    for pidx, pc, pl, pw in parts:
        for j, c, l in zip(pidx, pc, pl):
            if all_counts[j] is not None:
                raise RuntimeError(f"query {j} was served by two ranks (placements differ)")
            all_counts[j] = c
            all_lat[j] = l
        wall = max(wall, pw)
    if any(c is None for c in all_counts):
        raise RuntimeError("a query has no result (placements differ)")
    return all_counts, all_lat, wall


def gather_results(n, idx, counts, latency_ms, wall_s):
    """merge_results over every rank's share, gathered by one all-gather (every rank takes
    the same collective step and gets the whole result)."""
    world, _ = world_and_rank()
    mine = (list(map(int, idx)), list(map(int, counts)), list(map(float, latency_ms)),
            float(wall_s))
    parts = [mine]
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, mine)
    return merge_results(n, parts)
