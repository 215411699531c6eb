"""Generates tests/golden/golden_counts.json (run in the build container, where the reference
tree is present):

    python tests/golden/make_golden.py

For every test graph it records
  * the CSR digest of the symmetric graph and of the degree-oriented DAG, where the DAG is
    produced by the REFERENCE's own loader and orientation (Graph(prefix, use_dag=true),
    common/graph.cc:8-124, 210-401) reading the reference's on-disk format;
  * counts produced by the reference's own compiled host set-operation code
    (SetIntersection / VertexSet, common/intersect.cc, common/VertexSet.cc) driving the plans
    (oracle/ref/ref_plans.cc) -- the "ref" block;
  * brute-force counts for small graphs: the vertex-induced 4-vertex census over all
    4-subsets, and the number of injective edge-preserving maps (embeddings) of each
    reference pattern -- the "brute" block.
The tests check the oracle restatement (and through it the GPU path) against these values.
"""
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_api as O  # noqa: E402
import graphs as G  # noqa: E402

REF_PATTERNS_SYM = ["P1", "P2"] + G.INDUCED
BRUTE_MAX_N = 128


def ref_block(g, dag, tmp, name, big, cliques_only=False):
    prefix = os.path.join(tmp, name)
    O.write_reference_files(g, prefix)
    out = {}
    rg = O.RefGraph(prefix, use_dag=True)
    d = rg.csr()
    out["dag_digest"] = G.csr_digest(d)
    out["dag_matches_oracle_orientation"] = G.csr_digest(d) == G.csr_digest(dag)
    for k in (3, 4, 5, 6, 7):
        if big and k > 5:
            continue
        out[f"clique{k}"] = rg.count(f"clique{k}")[0]
    rg.close()
    if cliques_only:
        return out
    rs = O.RefGraph(prefix, use_dag=False)
    for p in REF_PATTERNS_SYM:
        if big and p in ("P1", "induced-4-cycle", "induced-3-star", "induced-4-path"):
            continue
        out[p] = rs.count(p)[0]
    rs.close()
    return out


def brute_block(g):
    out = {"census4": O.census4(g)}
    emb = {}
    for p, (k, edges) in G.PATTERN_EDGES.items():
        emb[p] = O.count_embeddings(k, edges, g)
    out["embeddings"] = emb
    out["automorphisms"] = {p: G.automorphisms(k, e) for p, (k, e) in G.PATTERN_EDGES.items()}
    return out


def main():
    cases = []
    specs = [("named", n) for n in G.NAMED] + [("rmat", s) for s in G.RMAT_SMALL] + \
        [("rmat", G.RMAT_TRIANGLE), ("rmat-cliques", G.RMAT_CLIQUE)]
    with tempfile.TemporaryDirectory() as tmp:
        for kind, spec in specs:
            t0 = time.time()
            if kind == "named":
                name = spec
                g = G.named_csr(name)
                entry = {"name": name, "kind": "named", "n": g.n,
                         "edges": [list(e) for e in G.NAMED[name][1]]}
            elif kind == "rmat-cliques":
                name = spec[0]
                g = G.rmat_csr(spec)
                entry = {"name": name, "kind": "rmat", "n": g.n, "edge_factor": spec[2],
                         "a": spec[3], "b": spec[4], "c": spec[5], "seed": spec[6],
                         "cliques_only": True}
            else:
                name = spec[0]
                g = G.rmat_csr(spec)
                entry = {"name": name, "kind": "rmat", "n": g.n, "edge_factor": spec[2],
                         "a": spec[3], "b": spec[4], "c": spec[5], "seed": spec[6]}
            dag = O.orient(g)
            big = g.n > 20000
            entry["arcs"] = g.m
            entry["dag_arcs"] = dag.m
            entry["sym_digest"] = G.csr_digest(g)
            entry["ref"] = ref_block(g, dag, tmp, name, big, kind == "rmat-cliques")
            if g.n <= BRUTE_MAX_N:
                entry["brute"] = brute_block(g)
            cases.append(entry)
            print(f"{name}: n={g.n} arcs={g.m} ({time.time() - t0:.1f}s)", flush=True)
    with open(os.path.join(HERE, "golden_counts.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
