"""Parity at the workloads' own sizes.

* The vertex-induced workload (R-MAT scale 24, edge factor 16, seed 1: 16.8 M vertices,
  521 M arcs): the set-difference enumeration plans and the edge-induced 4-cycle plan P1,
  run by jgpm_count_roots over a seeded, degree-stratified sample of root vertices (each
  counted over its whole slot range), equal the reference's own host code (oracle/_ref:
  its loader and its SetIntersection / VertexSet set operations) driving the same plans
  over the same roots.  The sample spans degrees 1 to several thousand, and every root's
  neighbourhood reaches the graph's hubs (degrees up to 406,787).  The plans' cost grows as
  d^2 .. d^3 per root vertex, so the dearest patterns sample fewer of the heavy roots.
* The batched workload (4,096 jobs): one batched launch over the full mix; a seeded subset of
  64 jobs is recounted by the oracle from the same seeded R-MAT definition.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

INDUCED_SCALE = 24
# degree bands [lo, hi) of the root vertices and the vertices drawn per band
BANDS = [(1, 16, 400), (16, 128, 150), (128, 1024, 24), (1024, 8192, 2)]
# (pattern, induced, reference-driver name, roots kept per band)
INDUCED_PLANS = [
    ("P1", 0, "P1", (400, 150, 24, 2)),
    ("4-cycle", 1, "induced-4-cycle", (400, 150, 24, 2)),
    ("diamond", 1, "induced-diamond", (400, 150, 24, 2)),
    ("tailed-triangle", 1, "induced-tailed-triangle", (400, 150, 24, 2)),
    ("4-path", 1, "induced-4-path", (400, 150, 8, 0)),
    ("3-star", 1, "induced-3-star", (400, 150, 24, 1)),
]


def stratified_roots(rowptr, seed=24):
    deg = np.diff(rowptr)
    rng = np.random.default_rng(seed)
    out = []
    for lo, hi, k in BANDS:
        idx = np.flatnonzero((deg >= lo) & (deg < hi))
        out.append(sorted(int(v) for v in rng.choice(idx, size=min(k, len(idx)),
                                                      replace=False)))
    return out


def test_induced_workload_sampled_roots_match_reference_code(gpu):
    if O.ref_lib() is None:
        pytest.fail("oracle/_ref/libjref.so (the reference's host code) is not built")
    n = 1 << INDUCED_SCALE
    with gpu.Graph.rmat(n, 16, 0.57, 0.19, 0.19, 1) as g:
        rowptr, col = g.csr()
        bands = stratified_roots(rowptr)
        with tempfile.TemporaryDirectory() as tmp:
            prefix = os.path.join(tmp, "g")
            O.write_reference_files(O.Csr(n, rowptr, col), prefix)
            del col
            rg = O.RefGraph(prefix, use_dag=False)
            try:
                for name, induced, rname, keep in INDUCED_PLANS:
                    want = got = 0
                    for roots, k in zip(bands, keep):
                        for v in roots[:k]:
                            b, e = int(rowptr[v]), int(rowptr[v + 1])
                            w = rg.count(rname, b, e, 1)[0]
                            c = g.count_roots(name, b, e, 1, induced=bool(induced))
                            assert c == w, (name, induced, v, e - b, c, w)
                            want += w
                            got += c
                    assert got == want and want > 0, (name, got, want)
            finally:
                rg.close()


BATCH_ORACLE = {"triangle": ("P0", True), "4-clique": ("P13", True),
                "5-clique": ("P14", True), "diamond": ("P2", False), "4-cycle": ("P1", False)}


def test_batched_workload_full_mix_matches_oracle_subset(gpu):
    import bench
    specs = bench.batched_specs(4096)
    graphs = [gpu.Graph.rmat(n, ef, a, b, c, sd) for (n, ef, a, b, c, sd, _) in specs]
    try:
        jobs = [(g, sp[6]) for g, sp in zip(graphs, specs)]
        counts, st = gpu.batch_count(jobs)
        assert len(counts) == len(jobs) and st["launches"] >= 1
        rng = np.random.default_rng(64)
        for j in sorted(rng.choice(len(specs), size=64, replace=False)):
            n, ef, a, b, c, sd, pat = specs[j]
            sym = O.rmat_graph(n, ef, a, b, c, sd)
            oname, dag = BATCH_ORACLE[pat]
            want = O.count(oname, O.orient(sym) if dag else sym)[0]
            assert counts[j] == want, (j, n, ef, pat, counts[j], want)
    finally:
        for g in graphs:
            g.close()


# (oracle name, runs on the DAG, largest graph the oracle recounts in the test)
SERVED_ORACLE = {"triangle": ("P0", True, 3 << 20), "4-clique": ("P13", True, 3 << 20),
                 "diamond": ("P2", False, 3 << 20), "5-clique": ("P14", True, 450000),
                 "4-cycle": ("P1", False, 130000),
                 "induced:tailed-triangle": ("induced-tailed-triangle", False, 130000)}


def test_served_workload_matches_oracle_subset(gpu):
    """The served workload: the 64-graph pool and an open-loop trace at 1,000 queries/s,
    replayed through the server (continuous batching, plain lanes for the heavy graphs).  A
    seeded subset of the answered queries is recounted by the oracle.  The subset takes the
    queries whose graph the oracle's nested-loop plan recounts in seconds: up to 3 M vertices
    for triangles, 4-cliques and diamonds, fewer for the dearer plans."""
    import bench
    specs = bench.served_setup(gpu)
    srv = gpu.Server(memory_budget_bytes=150 << 30, max_inflight=4, max_batch=256)
    try:
        for (n, ef, sd) in specs:
            srv.add_graph(gpu.Graph.rmat(n, ef, 0.57, 0.19, 0.19, sd))
        gids, pats, arr = bench.served_trace(1000, 400)
        counts, lat, wall = srv.replay(gids, pats, arr)
        assert len(counts) == 400 and wall > 0
        eligible = [q for q in range(len(gids))
                    if specs[int(gids[q])][0] <= SERVED_ORACLE[pats[q]][2]]
        rng = np.random.default_rng(5)
        pick = sorted(int(q) for q in rng.choice(eligible, size=16, replace=False))
        by_graph = {}
        for q in pick:
            by_graph.setdefault(int(gids[q]), []).append(q)
        for gi, qs in sorted(by_graph.items()):
            n, ef, sd = specs[gi]
            sym = O.rmat_graph(n, ef, 0.57, 0.19, 0.19, sd)
            dag = None
            for q in qs:
                oname, on_dag, _ = SERVED_ORACLE[pats[q]]
                if on_dag and dag is None:
                    dag = O.orient(sym)
                want = O.count(oname, dag if on_dag else sym)[0]
                assert counts[q] == want, (q, gi, n, pats[q], counts[q], want)
    finally:
        srv.close()
