"""CPU tests of bench.py's reporting arithmetic: the issue-slot roofline of a count, the clock
record (samples before the sampler's first reading are not counted; throttle reasons are
reported), and the served workload's placement of the graph pool."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_issue_roofline_arithmetic(bench):
    ctr = {"5-clique": {"warp_inst": 11_632_800_000, "dram_bytes": 400_000_000,
                        "l2_bytes": 13_000_000_000}}
    r = bench.roofline_of("5-clique", 20.0, 1e11, ctr, 1965.0, 148, 6650.0, "fallback")
    peak = 4 * 148 * 1965e6
    assert r["bound"] == "issue" and r["peak"] == pytest.approx(peak)
    assert r["achieved"] == pytest.approx(11_632_800_000 / 0.02)
    assert r["frac"] == pytest.approx(11_632_800_000 / 0.02 / peak)
    assert r["traffic"] == 400_000_000 and r["dram_gbs"] == pytest.approx(20.0)
    assert r["dram_frac"] == pytest.approx(20.0 / 6650.0)
    assert r["algorithmic_gbs"] == pytest.approx(4e11 / 0.02 / 1e9)
    none = bench.roofline_of("4-clique", 5.0, 1e9, ctr, 1965.0, 148, 6650.0, "fallback")
    assert none["achieved"] is None and none["frac"] is None


def test_clock_record_skips_start_up_samples_and_reports_reasons(bench):
    c = bench.ClockSampler(0)
    line = "0, {sm}, 1965, 700.0, 0x0, Not Active, Not Active, {th}, {pc}"
    c.lines = [line.format(sm=345, th="Not Active", pc="Not Active")]  # before the region
    c.first = 1
    c.lines += [line.format(sm=1965, th="Not Active", pc="Not Active"),
                line.format(sm=1950, th="Not Active", pc="Active"),
                line.format(sm=1965, th="Active", pc="Not Active"), "garbage"]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    c.first = 4  # no sample inside the region: all samples are used
    c.lines = c.lines[:4]
    assert c.summary()["samples"] == 4


def test_served_placement_uses_every_gpu(bench):
    from jupiter_b200 import pools
    specs = bench.served_setup(None)
    share = bench.served_shares(len(specs))
    assert abs(share.sum() - 1.0) < 1e-12 and share[0] > share[-1]
    loads = [sh * n * ef for sh, (n, ef, _) in zip(share, specs)]
    nbytes = [12 * n * ef + 16 * n for n, ef, _ in specs]
    for world in (1, 2, 4, 8):
        owner = pools.place_graphs(loads, nbytes, world, 150 << 30)
        per = [sum(l for l, o in zip(loads, owner) if o == r) for r in range(world)]
        assert sorted(set(owner.tolist())) == list(range(world))
        # greedy longest-first: no rank exceeds the mean by more than the largest load
        assert max(per) <= sum(loads) / world + max(loads)
