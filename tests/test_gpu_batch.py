"""GPU tests of the batched persistent kernel: every job's count equals its plain count and
the oracle, alone and in the mix, under every tuning the autotuner can pick."""
import itertools

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

PATTERNS = ["triangle", "4-clique", "5-clique", "diamond", "4-cycle"]
ORACLE = {"triangle": ("P0", True), "4-clique": ("P13", True), "5-clique": ("P14", True),
          "diamond": ("P2", False), "4-cycle": ("P1", False), "6-clique": ("P15", True)}


def mixed_graphs(J, count=12, seed=3):
    rng = np.random.default_rng(seed)
    specs = []
    for j in range(count):
        n = int(round(2 ** rng.uniform(np.log2(200), np.log2(6000))))
        ef = int(rng.choice([4, 8, 16, 32]))
        a = float(rng.uniform(0.45, 0.65))
        b = c = (1 - a) / 4
        specs.append((n, ef, a, b, c, 100 + j))
    return specs, [J.Graph.rmat(n, ef, a, b, c, s) for (n, ef, a, b, c, s) in specs]


@pytest.fixture(scope="module")
def mixed(gpu):
    specs, gs = mixed_graphs(gpu)
    want = {}
    for i, (n, ef, a, b, c, s) in enumerate(specs):
        sym = O.rmat_graph(n, ef, a, b, c, s)
        dag = O.orient(sym)
        for p in PATTERNS + ["6-clique"]:
            name, use_dag = ORACLE[p]
            want[(i, p)] = O.count(name, dag if use_dag else sym)[0]
    yield specs, gs, want
    for g in gs:
        g.close()


def test_plain_counts_match_oracle(gpu, mixed):
    specs, gs, want = mixed
    for i, g in enumerate(gs):
        for p in PATTERNS:
            assert g.count(p) == want[(i, p)], (i, p)


def test_batch_matches_plain_and_oracle(gpu, mixed):
    specs, gs, want = mixed
    jobs = [(g, p) for g in gs for p in PATTERNS]
    counts, st = gpu.batch_count(jobs)
    assert st["launches"] in (1, 2, 3) and st["tasks"] > 0
    for (g, p), c in zip(jobs, counts):
        assert c == want[(gs.index(g), p)], (gs.index(g), p)


def test_each_job_same_alone_and_in_mix(gpu, mixed):
    specs, gs, want = mixed
    jobs = [(gs[i % len(gs)], PATTERNS[(i * 7) % len(PATTERNS)]) for i in range(40)]
    counts, _ = gpu.batch_count(jobs)
    for (g, p), c in zip(jobs, counts):
        alone, _ = gpu.batch_count([(g, p)])
        assert alone == [c]
        assert c == want[(gs.index(g), p)]


def test_graph_replay_and_direct_launches_agree(gpu, mixed):
    """A batch's launches are captured in a CUDA graph and replayed while its launch plan
    repeats; a changed job set recaptures (updating the executable graph in place).  Replayed,
    recaptured and directly launched batches give the oracle's counts."""
    specs, gs, want = mixed
    sets = [[(g, p) for g in gs for p in PATTERNS],
            [(g, p) for g in gs[:5] for p in ("triangle", "4-cycle")],
            [(g, "diamond") for g in gs[3:9]]]
    for jobs in sets + sets[:1]:
        for graphs in (1, 1, 0):  # capture (or update), replay, direct
            t = gpu.Tuning(8, 128, 256, 0, graphs)
            counts, st = gpu.batch_count(jobs, t)
            assert st["tuning"]["graphs"] == graphs
            for (g, p), c in zip(jobs, counts):
                assert c == want[(gs.index(g), p)], (gs.index(g), p, graphs)


@pytest.mark.parametrize("min_group,split,rpt,isect",
                         list(itertools.product([4, 8, 32], [32, 128], [8, 256], [0, 1])))
def test_every_tuning_gives_the_same_counts(gpu, mixed, min_group, split, rpt, isect):
    specs, gs, want = mixed
    jobs = [(g, p) for g in gs[:6] for p in PATTERNS + ["6-clique"]]
    t = gpu.Tuning(min_group, split, rpt, isect)
    counts, st = gpu.batch_count(jobs, t)
    assert st["tuning"]["min_group"] == min_group
    for (g, p), c in zip(jobs, counts):
        assert c == want[(gs.index(g), p)], (gs.index(g), p, t.as_dict())


def test_autotune_returns_valid_tuning(gpu, mixed):
    specs, gs, want = mixed
    jobs = [(g, p) for g in gs for p in PATTERNS]
    t = gpu.autotune(jobs, sample_jobs=20)
    assert t.min_group in (4, 8, 16, 32) and t.intersect in (0, 1)
    counts, _ = gpu.batch_count(jobs, t)
    for (g, p), c in zip(jobs, counts):
        assert c == want[(gs.index(g), p)]


def test_batch_rejects_unbatchable_pattern(gpu, mixed):
    specs, gs, want = mixed
    with pytest.raises(gpu.JgpmError) as e:
        gpu.batch_count([(gs[0], "P7")])
    assert e.value.code == -5


@pytest.mark.parametrize("min_group,split", [(4, 128), (8, 64), (32, 32), (16, 128)])
def test_plain_tiers_any_split(gpu, mixed, min_group, split):
    """The plain kernels' tier boundaries (lane groups, warp roots, CTA roots) do not change
    counts on the large-degree triangle workload graph."""
    specs, gs, want = mixed
    g = gs[-1]
    g.set_tuning(gpu.Tuning(min_group, split, 0, 0))
    try:
        for p in ("triangle", "4-clique", "5-clique"):
            assert g.count(p) == want[(len(gs) - 1, p)]
    finally:
        g.set_tuning(gpu.Tuning(4, 128, 0, 0))


def test_batch_large_roots_complete_graph(gpu, mixed):
    """K_1101 (out-degrees up to 1100, so every root tier including the edge-rooted one)
    batched with the small graphs: closed-form counts."""
    from math import comb
    specs, gs, want = mixed
    n = 1101
    iu = np.triu_indices(n, 1)
    with gpu.Graph.from_edges(iu[0].astype(np.int32), iu[1].astype(np.int32), n) as k:
        closed = {"triangle": comb(n, 3), "4-clique": comb(n, 4),
                  "diamond": comb(n, 2) * comb(n - 2, 2), "4-cycle": 3 * comb(n, 4)}
        jobs = [(k, p) for p in closed] + [(g, p) for g in gs[:4] for p in PATTERNS]
        counts, _ = gpu.batch_count(jobs)
        for (g, p), c in zip(jobs, counts):
            if g is k:
                assert c == closed[p], p
            else:
                assert c == want[(gs.index(g), p)], (gs.index(g), p)


def test_batch_c4_slab_and_dense(gpu, mixed):
    """Large 4-cycle apexes in the batch's side kernel: slabs over several slices with 8-, 16-
    and 32-bit counters, and dense arrays for the apexes past the slice cap, next to small
    graphs.  Against the oracle and the K_{2,N} closed form."""
    from math import comb
    from test_gpu_parity import bipartite_2n, c4_slab_graphs
    specs, gs, want = mixed
    N = 70000
    big = [gpu.Graph.rmat(*spec) for spec in c4_slab_graphs()]
    try:
        with bipartite_2n(gpu, N) as kb:
            jobs = [(g, "4-cycle") for g in big] + [(kb, "4-cycle")] + \
                [(g, "4-cycle") for g in gs[:4]]
            exp = [O.count("P1", O.rmat_graph(*spec))[0] for spec in c4_slab_graphs()] + \
                [comb(N, 2)] + [want[(i, "4-cycle")] for i in range(4)]
            counts, st = gpu.batch_count(jobs)
            assert counts == exp
            assert st["launches"] == 2
            # without the 2^20 graph every large apex fits the narrow slab form (two CTAs of
            # 512 threads per SM)
            keep = [0, 2, 3, 4, 5, 6]
            counts, _ = gpu.batch_count([jobs[i] for i in keep])
            assert counts == [exp[i] for i in keep]
    finally:
        for g in big:
            g.close()


def test_batch_list_roots_crown(gpu, mixed):
    """Roots of out-degree 5000 (above the batched bitmap limits) run on edge-rooted lists in
    the batch: the crown graph of test_gpu_parity (closed forms), batched with small graphs."""
    from math import comb
    specs, gs, want = mixed
    na, nb, g = 5000, 5001, 1250
    a = np.arange(na, dtype=np.int64)
    b = np.arange(na, na + nb, dtype=np.int64)
    h = na + nb
    grp = a.reshape(g, 4)
    iu = np.triu_indices(4, 1)
    s = np.concatenate([np.repeat(a, nb), np.full(na, h), grp[:, iu[0]].ravel()]).astype(np.int32)
    d = np.concatenate([np.tile(b, na), a, grp[:, iu[1]].ravel()]).astype(np.int32)
    with gpu.Graph.from_edges(s, d, h + 1) as crown:
        closed = {"triangle": 4 * g + 6 * g + 6 * g * nb, "4-clique": g + 4 * g + 4 * g * nb,
                  "5-clique": g * (1 + nb),
                  "diamond": 3 * (na + na * nb) + 6 * g * comb(nb + 3, 2)}
        jobs = [(crown, p) for p in closed] + [(gg, "4-clique") for gg in gs[:3]]
        counts, _ = gpu.batch_count(jobs)
        for (gg, p), c in zip(jobs, counts):
            if gg is crown:
                assert c == closed[p], p
            else:
                assert c == want[(gs.index(gg), p)]


def test_batch_induced_tailed_triangle(gpu, mixed):
    """Vertex-induced tailed triangles in the batch (one k = 4 pass: 12 K4 - 4 N(diamond) +
    N(tailed triangle)) equal the plain fused count and the census (an independent method),
    alone and mixed with other jobs."""
    specs, gs, want = mixed
    jobs = [(g, "induced:tailed-triangle") for g in gs] + [(g, "4-clique") for g in gs[:4]]
    counts, _ = gpu.batch_count(jobs)
    for (g, p), c in zip(jobs, counts):
        if p == "4-clique":
            assert c == want[(gs.index(g), p)]
            continue
        assert c == g.count("tailed-triangle", induced=True)
        assert c == g.census4()[2]
    n = 1101
    iu = np.triu_indices(n, 1)
    with gpu.Graph.from_edges(iu[0].astype(np.int32), iu[1].astype(np.int32), n) as k:
        assert gpu.batch_count([(k, "induced:tailed-triangle")])[0] == [0]
        assert k.count("tailed-triangle", induced=True) == 0


def test_batch_induced_tailed_triangle_crown(gpu):
    """Crown graph (see test_batch_list_roots_crown): the tailed triangles are the
    triangles h + A-edge and b + A-edge, each with the |A| - 4 vertices of other groups as the
    tail: 6 g (|A| - 4)(1 + |B|)."""
    na, nb, g = 5000, 5001, 1250
    a = np.arange(na, dtype=np.int64)
    b = np.arange(na, na + nb, dtype=np.int64)
    h = na + nb
    grp = a.reshape(g, 4)
    iu = np.triu_indices(4, 1)
    s = np.concatenate([np.repeat(a, nb), np.full(na, h), grp[:, iu[0]].ravel()]).astype(np.int32)
    d = np.concatenate([np.tile(b, na), a, grp[:, iu[1]].ravel()]).astype(np.int32)
    want = 6 * g * (na - 4) * (1 + nb)
    with gpu.Graph.from_edges(s, d, h + 1) as crown:
        assert crown.count("tailed-triangle", induced=True) == want
        assert gpu.batch_count([(crown, "induced:tailed-triangle")])[0] == [want]
