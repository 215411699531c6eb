"""Benchmark of the plain k-clique counting path (4-clique and 5-clique) on the citation-graph
shaped workload: R-MAT scale 22 (4,194,304 vertices), edge factor 4, a/b/c/d =
0.57/0.19/0.19/0.05, seed 1, degree-oriented DAG resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl jgpm|reference]

A step is one exact 4-clique count plus one exact 5-clique count of the whole graph, each a
plain single-query call of the library.  The metric is set-op elements per second: the
set-op operand elements of the canonical edge-rooted plan (every level-1 arc intersection
N+(u) & N+(v) adds d+(u)+d+(v), every deeper "W & N+(v)" adds |W|+d+(v)), counted exactly
by the library's accounting pass and cross-checked against the oracle in the tests.
Between timed steps L2 is flushed by writing a 512 MiB buffer (the graph is ~100 MB, below
the 126 MB L2).  Multi-GPU (torchrun): every rank holds the whole graph and counts its shard
of each count (jgpm_count_shard: the roots of every out-degree tier with index = rank mod
world), so the total work is fixed (strong scaling); the partial counts are summed with one
NCCL all-reduce, and times are the maximum over ranks.

The kernels are bound by instruction issue, not by memory (the DAG stays in L2): `roofline`
reports the dominant count's issue-slot use (warp instructions per second, from the ncu
counters committed in profiles/counters.json, over 4 issue slots x SMs x the sampled SM
clock), with its DRAM and L2 traffic beside it.

The reference arm (--impl reference) times the reference's own host code (its AVX2
set-intersection and graph loader, compiled from its sources into oracle/_ref/) driving the
same plans on all host cores, over a bounded sample of root arcs of the same workload.
"""
import argparse
import atexit
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {"workload": "k-clique (k=4,5) on R-MAT scale 22, edge factor 4, "
                        "a/b/c/d=0.57/0.19/0.19/0.05, seed 1, degree-oriented DAG",
            "scale": 22, "edge_factor": 4, "a": 0.57, "b": 0.19, "c": 0.19, "seed": 1,
            "patterns": ["4-clique", "5-clique"], "l2": "flushed between steps (512 MiB write)"}
METRIC = "matches/s + set-op elems/s (% HBM roofline); served vs plain queries/s, p50/p99"
UNIT = "set-op elems/s"
N_VERT = 1 << 22
EDGE_FACTOR = 4


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            atexit.register(self.__exit__, None, None, None)  # never outlives the bench
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler is running: samples taken before that
            # (nvidia-smi's start-up) are not counted
            t_end = time.perf_counter() + 5.0
            while not self.lines and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.first = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc and self.proc.poll() is None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:] or self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), \
        int(os.environ.get("WORLD_SIZE", 1))


# ----------------------------------------------------------------------------- our arm
def counters():
    """Per-count ncu counters of the tier kernels (profiles/counters.json): warp instructions,
    DRAM and L2 bytes of one 4-clique and one 5-clique count of this workload."""
    p = os.path.join(ROOT, "profiles", "counters.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def roofline_of(name, ms, elems, ctr, sm_mhz, sms, hbm, hbm_kind):
    """Issue-slot roofline of one count: the tier kernels run from L2 and are bound by
    instruction issue.  achieved = warp instructions (ncu) / the count's event-timed
    duration; peak = 4 issue slots x SMs x the median SM clock sampled during the run."""
    c = ctr.get(name)
    t = ms / 1e3
    out = {"bound": "issue", "kernel": f"{name} count (bitmap clique tiers)", "unit": "warp-inst/s",
           "peak": 4.0 * sms * sm_mhz * 1e6,
           "peak_kind": f"4 issue slots x {sms} SMs x {sm_mhz:.0f} MHz (median sampled SM clock)",
           "algorithmic_gbs": 4.0 * elems / t / 1e9,
           "algorithmic_note": "canonical plan's set-op operand bytes per second: a work rate, "
                               "not memory traffic (the bitmap kernels read far fewer bytes)"}
    if c:
        out.update({"achieved": c["warp_inst"] / t, "frac": c["warp_inst"] / t / out["peak"],
                    "warp_inst_per_launch": c["warp_inst"], "traffic": c["dram_bytes"],
                    "dram_gbs": c["dram_bytes"] / t / 1e9,
                    "dram_frac": c["dram_bytes"] / t / 1e9 / hbm, "dram_peak_gbs": hbm,
                    "dram_peak_kind": hbm_kind, "l2_bytes": c["l2_bytes"],
                    "l2_gbs": c["l2_bytes"] / t / 1e9, "counters": "profiles/counters.json"})
    else:
        out.update({"achieved": None, "frac": None, "traffic": None})
    return out


def run_jgpm(args):
    import ctypes

    import numpy as np
    import torch

    import jupiter_b200 as J
    from jupiter_b200 import shards

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    J.lib().jgpm_set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count

    g = J.Graph.rmat(N_VERT, EDGE_FACTOR, 0.57, 0.19, 0.19, 1, use_dag=True)
    info = g.info()
    stream = torch.cuda.ExternalStream(g.stream(), device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    # untimed: exact counts and the canonical plan's set-op elements
    c4, st4 = g.count("4-clique", stats=True)
    c5, st5 = g.count("5-clique", stats=True)
    elems4, elems5 = st4["setop_elements"], st5["setop_elements"]
    elems_step = elems4 + elems5
    matches_step = c4 + c5

    def count(pattern):
        if world > 1:
            return g.count_shard(pattern, rank, world, details=True)
        return g.count(pattern, details=True)

    if world > 1:  # the shards add up to the whole count on every rank
        parts = [count("4-clique")[0], count("5-clique")[0]]
        if shards.reduce_counts(parts, dev) != [c4, c5]:
            raise RuntimeError("sharded counts do not add up to the whole counts")
    want = None

    def step(events):
        nonlocal want
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e2 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        a, sa = count("4-clique")
        with torch.cuda.stream(stream):
            e1.record(stream)
        b, sb = count("5-clique")
        with torch.cuda.stream(stream):
            e2.record(stream)
        if want is None:
            want = (a, b)
        if (a, b) != want:
            raise RuntimeError(f"count changed between runs: {a} {b} vs {want}")
        events.append((e0, e1, e2, sa["launches"] + sb["launches"]))

    for _ in range(args.warmup):
        step([])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    events = []
    # clocks are sampled over both timed regions: the device-timed steps and the e2e steps
    clk = ClockSampler(local).__enter__()
    for _ in range(args.steps):
        step(events)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t4 = [e0.elapsed_time(e1) for e0, e1, e2, _ in events]
    t5 = [e1.elapsed_time(e2) for e0, e1, e2, _ in events]
    total_ms = sum(a + b for a, b in zip(t4, t5))
    launches = sum(x[3] for x in events)
    k4_ms, k5_ms = sum(t4) / len(t4), sum(t5) / len(t5)
    if world > 1:
        total_ms = shards.max_over_ranks(total_ms, dev)
        k4_ms = shards.max_over_ranks(k4_ms, dev)
        k5_ms = shards.max_over_ranks(k5_ms, dev)
    ms_per_step = total_ms / args.steps
    value = elems_step / (ms_per_step / 1e3)

    # e2e: through the public API with host buffers (pinned): upload of the CSR, orientation,
    # both counts (this rank's shards), the counts read back (and summed over the ranks)
    rowptr, col = g.csr()
    h_rowptr = torch.from_numpy(rowptr).pin_memory()
    h_col = torch.from_numpy(col).pin_memory()
    P64 = ctypes.POINTER(ctypes.c_int64)
    P32 = ctypes.POINTER(ctypes.c_int32)
    rp_ptr = ctypes.cast(h_rowptr.data_ptr(), P64)
    col_ptr = ctypes.cast(h_col.data_ptr(), P32)

    def e2e_step():
        h = ctypes.c_void_p()
        rc = J.lib().jgpm_graph_from_csr(rp_ptr, col_ptr, len(rowptr) - 1, len(col), 1,
                                         ctypes.byref(h))
        if rc:
            raise RuntimeError(J.lib().jgpm_last_error().decode())
        gg = J.Graph(h.value)
        if world > 1:
            parts = [gg.count_shard("4-clique", rank, world),
                     gg.count_shard("5-clique", rank, world)]
            a, b = shards.reduce_counts(parts, dev)
        else:
            a, b = gg.count("4-clique"), gg.count("5-clique")
        gg.close()
        if a != c4 or b != c5:
            raise RuntimeError("e2e count mismatch")

    # each e2e step is timed on its own (host clock around a synchronous call) and the median
    # over all timed steps is reported: the host-side part varies from step to step
    e2e_step()
    torch.cuda.synchronize()
    e2e_times = []
    for _ in range(args.steps):
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        e2e_step()
        torch.cuda.synchronize()
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    clk.__exit__(None, None, None)
    e2e_ms = statistics.median(e2e_times)
    if world > 1:
        e2e_ms = shards.max_over_ranks(e2e_ms, dev)
    h2d = rowptr.nbytes + col.nbytes
    d2h = 2 * 8

    hbm, hbm_kind = peaks()
    ck = clk.summary()
    sm_mhz = ck["sm_mhz"] or 1965.0
    ctr = counters()
    roof = roofline_of("5-clique", k5_ms, elems5, ctr, sm_mhz, sms, hbm, hbm_kind)
    roof["other"] = {"4-clique": roofline_of("4-clique", k4_ms, elems4, ctr, sm_mhz, sms, hbm,
                                             hbm_kind)}
    roof["kernel_share_of_step"] = k5_ms / ms_per_step

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT stands in for the absent citation dataset)",
        "config": dict(WORKLOAD, parallelism=f"root shards x{world}" if world > 1 else "single",
                       num_vertices=info["num_vertices"], num_arcs=info["num_arcs"],
                       num_dag_arcs=info["num_dag_arcs"],
                       max_out_degree=info["max_out_degree"]),
        "matches_per_s": matches_step / (ms_per_step / 1e3),
        "counts": {"4-clique": c4, "5-clique": c5},
        "setop_elements": {"4-clique": elems4, "5-clique": elems5},
        "ms": {"4-clique": k4_ms, "5-clique": k5_ms},
        "roofline": roof,
        "e2e": {"value": elems_step / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "steps": len(e2e_times), "ms_min": min(e2e_times), "ms_max": max(e2e_times),
                "stat": "median of per-step times"},
        "gpu_launches": launches,
        "clocks": ck,
    }
    g.close()
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ CPU reference / baseline
def _cpu_graph():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    g = O.rmat_graph(N_VERT, EDGE_FACTOR, 0.57, 0.19, 0.19, 1)
    return O, g


def _sample_stride(total_arcs, target_arcs):
    return max(1, total_arcs // max(1, target_arcs))


def cpu_baseline(seconds=15.0, O=None, g=None, rg=None):
    """The reference's host code (oracle/_ref) on a strided sample of root arcs, all cores."""
    if O is None:
        O, g = _cpu_graph()
    dag = O.orient(g)
    threads = os.cpu_count() or 1
    tmp = None
    if rg is None:
        tmp = tempfile.TemporaryDirectory()
        prefix = os.path.join(tmp.name, "g")
        O.write_reference_files(g, prefix)
        rg = O.RefGraph(prefix, use_dag=True)
    # calibrate the stride so the sample runs ~`seconds`
    stride = _sample_stride(dag.m, 20000)
    c, t = rg.count("P13", 0, dag.m, stride, threads)
    c5, t5 = rg.count("P14", 0, dag.m, stride, threads)
    per = (t + t5) / max(1, (dag.m + stride - 1) // stride)
    want = max(1, int(seconds / max(per, 1e-9)))
    stride = max(1, dag.m // want)
    c, t = rg.count("P13", 0, dag.m, stride, threads)
    c5, t5 = rg.count("P14", 0, dag.m, stride, threads)
    _, e4 = O.count("P13", dag, 0, dag.m, stride, threads)
    _, e5 = O.count("P14", dag, 0, dag.m, stride, threads)
    if tmp is not None:
        rg.close()
        tmp.cleanup()
    return {"value": (e4 + e5) / (t + t5), "unit": UNIT, "cores": threads,
            "kind": "reference", "seconds": t + t5,
            "sample": f"every {stride}th root arc of the DAG ({(dag.m + stride - 1) // stride} of "
                      f"{dag.m}), 4-clique + 5-clique plans over the reference's AVX2 "
                      f"SetIntersection (common/intersect.cc)",
            "cpu": _cpu_model()}


def _cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    O, g = _cpu_graph()
    dag = O.orient(g)
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "g")
        O.write_reference_files(g, prefix)
        rg = O.RefGraph(prefix, use_dag=True)
        threads = os.cpu_count() or 1
        per_step = max(1.0, args.cpu_seconds / max(1, args.steps + args.warmup))
        stride = _sample_stride(dag.m, 20000)
        _, t4 = rg.count("P13", 0, dag.m, stride, threads)
        _, t5 = rg.count("P14", 0, dag.m, stride, threads)
        per = (t4 + t5) / max(1, (dag.m + stride - 1) // stride)
        stride = max(1, dag.m // max(1, int(per_step / max(per, 1e-9))))
        _, e4 = O.count("P13", dag, 0, dag.m, stride, threads)
        _, e5 = O.count("P14", dag, 0, dag.m, stride, threads)
        for _ in range(args.warmup):
            rg.count("P13", 0, dag.m, stride, threads)
            rg.count("P14", 0, dag.m, stride, threads)
        secs = 0.0
        for i in range(args.steps):
            off = i % stride
            _, a = rg.count("P13", off, dag.m, stride, threads)
            _, b = rg.count("P14", off, dag.m, stride, threads)
            secs += a + b
        rg.close()
    ms_per_step = secs * 1e3 / args.steps
    value = (e4 + e5) / (ms_per_step / 1e3)
    sample = (f"every {stride}th root arc of the DAG per step (offset varies by step), "
              f"4-clique + 5-clique plans over the reference's AVX2 SetIntersection")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic (seeded R-MAT stands in for the absent citation dataset)",
           "config": dict(WORKLOAD, parallelism="host cores"),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                            "sample": sample, "cpu": _cpu_model()},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ other workloads
BATCH_PATTERNS = ["triangle", "4-clique", "5-clique", "diamond", "4-cycle"]


def batched_specs(njobs=4096, seed=4096):
    """Job j: graph seed 1 + j; n log-uniform in [1K, 256K]; edge factor uniform in
    {4, 8, 16, 32}; a ~ U[0.45, 0.65], b = c = (1 - a) / 4; pattern uniform over the five."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for j in range(njobs):
        n = int(round(2 ** rng.uniform(10.0, 18.0)))
        ef = int(rng.choice([4, 8, 16, 32]))
        a = float(rng.uniform(0.45, 0.65))
        b = (1.0 - a) / 4.0
        pat = BATCH_PATTERNS[int(rng.integers(len(BATCH_PATTERNS)))]
        out.append((n, ef, a, b, b, 1 + j, pat))
    return out


def run_batched(args):
    import numpy as np
    import torch

    import jupiter_b200 as J
    torch.cuda.set_device(0)
    specs = batched_specs(args.jobs)
    t0 = time.time()
    graphs = [J.Graph.rmat(n, ef, a, b, c, sd) for (n, ef, a, b, c, sd, _) in specs]
    jobs = [(g, sp[6]) for g, sp in zip(graphs, specs)]
    gen_s = time.time() - t0
    # plain: each job as its own jgpm_count call (also prepares DAGs and tiers)
    plain_counts = [g.count(p) for g, p in jobs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_dev_ms = 0.0
    for _ in range(args.plain_passes):
        res = [g.count(p, details=True) for g, p in jobs]
        plain_counts = [c for c, _ in res]
        plain_dev_ms += sum(st["kernel_ms"] for _, st in res)
    torch.cuda.synchronize()
    plain_s = (time.perf_counter() - t0) / args.plain_passes
    plain_dev_s = plain_dev_ms / 1e3 / args.plain_passes
    # plain device time of the jobs that take at least a millisecond of device time alone: their
    # launches fill the GPU, so batching can remove little of it
    big_dev_s = sum(st["kernel_ms"] for _, st in res if st["kernel_ms"] >= 1.0) / 1e3
    tuning = J.autotune(jobs, sample_jobs=256)
    for _ in range(args.warmup):
        J.batch_count(jobs, tuning)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    kms = []
    launches = 0
    for _ in range(args.steps):
        counts, st = J.batch_count(jobs, tuning)
        kms.append(st["kernel_ms"])
        launches += st["launches"]
        if counts != plain_counts:
            raise RuntimeError("batched counts differ from the plain counts")
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    dev_ms = sum(kms) / len(kms)
    out = {"metric": METRIC, "workload": "batched",
           "value": len(jobs) / (dev_ms / 1e3), "unit": "queries/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic R-MAT jobs",
           "config": {"workload": f"{len(jobs)} (graph, pattern) jobs in one persistent launch: "
                      "n log-uniform [1K,256K], ef in {4,8,16,32}, a~U[.45,.65], b=c=(1-a)/4, "
                      "pattern uniform over triangle/4-clique/5-clique/diamond/4-cycle",
                      "jobs": len(jobs), "tuning": tuning.as_dict(), "tasks": st["tasks"]},
           "batched_wall_queries_per_s": len(jobs) / wall,
           "plain_queries_per_s": len(jobs) / plain_s,
           "speedup_vs_plain": (len(jobs) / (dev_ms / 1e3)) / (len(jobs) / plain_s),
           "speedup_vs_plain_wall": plain_s / wall,
           "counts_identical_to_plain": True, "graph_generation_s": gen_s,
           "gpu_launches": launches,
           "amdahl": {"plain_wall_s": plain_s, "plain_device_s": plain_dev_s,
                      "plain_host_share": 1.0 - plain_dev_s / plain_s,
                      "plain_device_s_in_jobs_of_1ms_or_more": big_dev_s,
                      "bound_if_batching_removed_all_host_time": plain_s / plain_dev_s,
                      "batched_vs_plain_device": plain_dev_s / (dev_ms / 1e3),
                      "note": "the batch can remove the plain calls' host time and the tails "
                              "of small launches, not the device work of jobs that fill the GPU"}}
    for g in graphs:
        g.close()
    print(json.dumps(out), flush=True)


def served_setup(J, ngraphs=64, seed=5):
    import numpy as np
    rng = np.random.default_rng(seed)
    scales = rng.uniform(14.0, 23.0, ngraphs)
    return [(int(round(2 ** sc)), 8, 1001 + i) for i, sc in enumerate(scales)]


def served_shares(ngraphs=64):
    """Each graph's share of the queries: Zipf(1.1) over the graph ids."""
    import numpy as np
    pz = np.arange(1, ngraphs + 1, dtype=np.float64) ** -1.1
    return pz / pz.sum()


def served_trace(rate, nq, ngraphs=64, seed=11):
    import numpy as np
    rng = np.random.default_rng(seed + int(rate))
    gids = rng.choice(ngraphs, size=nq, p=served_shares(ngraphs))
    pats = ["triangle", "4-clique", "5-clique", "diamond", "4-cycle", "induced:tailed-triangle"]
    pp = [pats[int(x)] for x in rng.integers(len(pats), size=nq)]
    arr = np.cumsum(rng.exponential(1.0 / rate, nq))
    return gids, pp, arr


def run_served(args):
    """The served workload.  Under torchrun the graph pool is spread over one server per GPU
    (jupiter_b200.pools): every rank places the graphs alike, builds and serves only its own,
    replays the queries of its graphs with their arrival times, and one all-gather per arm
    brings all per-query results to rank 0.  Both arms (served and plain) run on every GPU."""
    import numpy as np
    import torch

    import jupiter_b200 as J
    from jupiter_b200 import pools

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    J.lib().jgpm_set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    specs = served_setup(J)
    budget = 150 << 30
    loads = [sh * n * ef for sh, (n, ef, _) in zip(served_shares(len(specs)), specs)]
    nbytes = [12 * n * ef + 16 * n for n, ef, _ in specs]  # symmetric CSR + DAG, estimated
    owner = pools.place_graphs(loads, nbytes, world, budget)
    srv = J.Server(memory_budget_bytes=budget, max_inflight=4, max_batch=256, device=local)
    t0 = time.time()
    for gid in pools.local_ids(owner, rank):
        n, ef, sd = specs[gid]
        srv.add_graph(J.Graph.rmat(n, ef, 0.57, 0.19, 0.19, sd))
    gen_s = time.time() - t0

    def replay(gids, pats, arr, plain=False):
        idx, loc = pools.local_queries(gids, owner, rank)
        c, lat, wall = srv.replay(loc, [pats[i] for i in idx], np.asarray(arr)[idx],
                                  plain=plain)
        return pools.gather_results(len(gids), idx, c, lat, wall)

    # warm every (graph, pattern) once so first-use costs are outside the measurement
    g0, p0, a0 = served_trace(1000, 200)
    replay(g0, p0, a0)
    rows = []
    for rate in args.rates:
        nq = int(min(args.max_queries, max(50, rate * args.seconds)))
        gids, pats, arr = served_trace(rate, nq)
        c1, lat1, w1 = replay(gids, pats, arr)
        c2, lat2, w2 = replay(gids, pats, arr, plain=True)
        if c1 != c2:
            bad = [(int(g), p, int(a), int(b)) for g, p, a, b in zip(gids, pats, c1, c2) if a != b]
            raise RuntimeError(f"served counts differ from the plain counts at {rate} q/s: "
                               f"{len(bad)} of {nq}, e.g. (graph, pattern, served, plain) "
                               f"{bad[:6]}")
        rows.append({"offered_qps": rate, "queries": nq,
                     "served": {"qps": nq / w1, "p50_ms": float(np.percentile(lat1, 50)),
                                "p99_ms": float(np.percentile(lat1, 99))},
                     "plain": {"qps": nq / w2, "p50_ms": float(np.percentile(lat2, 50)),
                               "p99_ms": float(np.percentile(lat2, 99))}})
    st = srv.stats()
    srv.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    best = max(rows, key=lambda r: r["served"]["qps"])
    out = {"metric": METRIC, "workload": "served", "value": best["served"]["qps"],
           "unit": "queries/s", "n_gpus": world, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "int32", "data": "synthetic R-MAT graph pool",
           "config": {"workload": "open-loop Poisson queries over 64 resident R-MAT graphs "
                      "(scale U[14,23], ef 8, .57/.19/.19/.05, seeds 1001..1064), graph ~ "
                      "Zipf(1.1), pattern uniform over triangle/4-clique/5-clique/diamond/"
                      "4-cycle/vertex-induced tailed triangle, 150 GB budget per GPU",
                      "max_inflight": 4, "max_batch": 256,
                      "parallelism": f"graph pool over {world} GPUs" if world > 1 else "single",
                      "graphs_per_gpu": [len(pools.local_ids(owner, r)) for r in range(world)]},
           "rates": rows, "server_stats_rank0": st, "graph_generation_s": gen_s,
           "counts_identical_to_plain": True}
    print(json.dumps(out), flush=True)


def run_induced(args):
    import torch

    import jupiter_b200 as J
    torch.cuda.set_device(0)
    n = 1 << args.scale
    t0 = time.time()
    g = J.Graph.rmat(n, 16, 0.57, 0.19, 0.19, 1)
    gen_s = time.time() - t0
    info = g.info()
    names = ["3-star", "4-path", "tailed-triangle", "4-cycle", "diamond", "4-clique"]
    t0 = time.perf_counter()
    census = g.census4()
    torch.cuda.synchronize()
    census_s = time.perf_counter() - t0
    per = {}
    for p in names[:5]:
        c, st = g.count(p, induced=True, details=True)
        per[p] = {"count": c, "ms": st["kernel_ms"], "method": st["method"]}
        if c != census[names.index(p)]:
            raise RuntimeError("census and per-pattern counts differ")
    out = {"metric": METRIC, "workload": "induced-4-vertex",
           "value": 5 / census_s, "unit": "patterns/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "int64", "data": "synthetic R-MAT",
           "config": {"workload": f"vertex-induced 4-cycle/diamond/tailed triangle/4-path/3-star "
                      f"on R-MAT scale {args.scale}, ef 16, .57/.19/.19/.05, seed 1",
                      "num_vertices": info["num_vertices"], "num_arcs": info["num_arcs"],
                      "max_degree": info["max_degree"]},
           "census": dict(zip(names, census)), "census_s": census_s, "per_pattern": per,
           "graph_generation_s": gen_s}
    g.close()
    print(json.dumps(out), flush=True)


def run_count(args):
    """One pattern on one seeded R-MAT graph, timed per count (device events): the command the
    per-kernel profiles run.  --rmat n,ef,a,b,c,seed."""
    import torch

    import jupiter_b200 as J
    torch.cuda.set_device(0)
    f = args.rmat.split(",")
    spec = (int(f[0]), int(f[1]), float(f[2]), float(f[3]), float(f[4]), int(f[5]))
    with J.Graph.rmat(*spec) as g:
        for _ in range(args.warmup):
            c = g.count(args.pattern, induced=args.induced)
        ms = []
        for _ in range(args.steps):
            c, st = g.count(args.pattern, induced=args.induced, details=True)
            ms.append(st["kernel_ms"])
        print(json.dumps({"workload": "count", "pattern": args.pattern, "induced": args.induced,
                          "rmat": list(spec), "count": c, "kernel_ms": ms, "method": st["method"],
                          "graph": g.info()}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="jgpm", choices=["jgpm", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="clique",
                    choices=["clique", "batched", "served", "induced", "count"])
    ap.add_argument("--pattern", default="4-cycle")
    ap.add_argument("--induced", action="store_true", help="count workload: vertex-induced")
    ap.add_argument("--rmat",
                    default="258730,32,0.471263918196369,0.13218402045090777,0.13218402045090777,2958",
                    help="count workload: n,ef,a,b,c,seed (default: the heaviest 4-cycle job "
                    "of the batched workload)")
    ap.add_argument("--jobs", type=int, default=4096)
    ap.add_argument("--plain-passes", type=int, default=1)
    ap.add_argument("--rates", type=float, nargs="+", default=[100, 300, 1000, 3000, 5000])
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--max-queries", type=int, default=4000)
    ap.add_argument("--scale", type=int, default=24)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "induced":
        run_induced(args)
    elif args.workload == "count":
        run_count(args)
    else:
        run_jgpm(args)


if __name__ == "__main__":
    main()
