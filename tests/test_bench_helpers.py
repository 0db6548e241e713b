"""CPU checks of bench.py's reporting helpers: the clock record taken during the timed region
(median SM clock, max clock, throttle reasons), the latency percentiles, the algorithmic
bytes behind the roofline, and the measured HBM peak it is divided by."""
import json
import os

import numpy as np

import bench


def test_clock_summary_reads_clocks_and_throttle_reasons():
    s = bench.ClockSampler(0)
    s.lines = [
        "0, 1965, 1965, 700.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 800.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    out = s.summary()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    s.lines = ["0, 1200, 1965, 500, 0x8, Active, Not Active, Active, Not Active"]
    assert s.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    s.lines = []
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_latency_percentiles_in_ms():
    ns = np.arange(1, 1001) * 1_000_000  # 1 .. 1000 ms
    p = bench.percentiles_ms(ns)
    assert p["max"] == 1000.0 and abs(p["p50"] - 500.5) < 1e-9
    assert abs(p["p99"] - np.percentile(np.arange(1, 1001), 99)) < 1e-9
    assert p["p50"] <= p["p99"] <= p["p99.9"] <= p["max"]


def test_algorithmic_bytes_weight_each_function_by_its_bytes():
    stats = {"fn0_evals": 10, "fn1_evals": 5, "fn2_evals": 2}
    assert bench.algorithmic_bytes(stats, bench.BYTES_PER_CALL["photon"]) == 10 * 93 + 5 * 68 + 2 * 32
    assert bench.algorithmic_bytes({}, [32, 32]) == 0


def test_peak_comes_from_the_measured_file():
    p = bench.peaks()
    path = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        assert p["source"] == "measured" and p["hbm_gbs"] == float(json.load(open(path))["hbm_gbs"])
    else:
        assert p["source"] == "fallback"


def _args(**kw):
    import argparse
    d = dict(workload="photon", photons=10_000_000, grid=128, scale=22, program="async", variant=-1)
    d.update(kw)
    return argparse.Namespace(**d)


def test_both_arms_report_the_same_workload_config():
    """The config names the workload only; how it is run (program type, tuning variant, the
    reference's launch shape) is reported beside it, so both arms print equal configs."""
    for wl in ("photon", "bfs", "collatz"):
        a = bench.workload_config(_args(workload=wl, program="async"), 1)
        b = bench.workload_config(_args(workload=wl, program="event", variant=3), 1)
        assert a == b and "program" not in a and "variant" not in a
    assert bench.workload_config(_args(), 1)["workload"] == "photon_walk_1e+07_photons_128^3"


def test_reference_side_scripts_do_not_load_the_product():
    """The reference arm, the reference sweep and the golden-fixture script build their inputs
    with the oracle's own generators, so their processes map no library of the product."""
    for rel in ("oracle/reference_bench.py", "oracle/ref_sweep.py", "tests/golden/make_golden.py"):
        src = open(os.path.join(bench.ROOT, rel)).read()
        assert "harmonize_b200" not in src, rel


def test_reference_arm_names_resolve():
    """Every oracle name the reference arm of bench.py uses is exported by the oracle package
    (the arm only runs on a GPU box; a missing export would end it there)."""
    import re
    import oracle
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "oracle", "reference_bench.py")).read()
    names = set(re.findall(r"\boracle\.([A-Za-z_][A-Za-z0-9_]*)", src))
    assert names, "no oracle names found"
    missing = [n for n in sorted(names) if not hasattr(oracle, n)]
    assert not missing, missing


def test_collatz_plain_leg_passes_the_whole_range_as_one_plain_job(monkeypatch):
    """The Collatz bench line's plain_kernel leg: one plain job over the bench's start values
    (1 .. 2^20) through hrm_plain_run on one stream, best of three, its outputs compared with
    the timed run's. The device is faked here; the leg's C entry point runs in the GPU tests."""
    import ctypes
    import types

    import harmonize_b200 as hrm
    from harmonize_b200 import jobs

    seen = []

    class FakeJobsLib:
        def hrm_plain_run(self, arr_ref, njobs, nstreams, done_ptr, total_ref):
            j = arr_ref._obj[0]
            seen.append((j.kind, j.first, j.count, j.out, njobs, nstreams))
            total_ref._obj.value = 2.0 + len(seen)  # 3, 4, 5 ms: best of three is 3
            return 0

    class FakeTensor:
        def data_ptr(self):
            return 0x1000

        def pin_memory(self):
            return self

    fake_torch = types.SimpleNamespace(empty=lambda *a, **k: FakeTensor(), int32="int32",
                                       equal=lambda a, b: True, cuda=types.SimpleNamespace(synchronize=lambda: None))
    monkeypatch.setattr(jobs, "_bind", lambda: FakeJobsLib())
    monkeypatch.setattr(bench, "flush_l2", lambda buf: None)
    args = types.SimpleNamespace(program="async", variant=2, workload="collatz")
    wl = bench.run_collatz(args, hrm, 0, 1, None, fake_torch)
    ms, info = wl["plain_arm"](None)
    assert ms == 3.0
    assert info["same_outputs"] is True and "one thread per start value" in info["what"]
    assert seen == [(jobs.JOB_COLLATZ, 1, 1 << 20, 0x1000, 1, 1)] * 3


def test_photon_plain_leg_passes_the_photons_as_one_plain_job(monkeypatch):
    """The photon bench line's plain_kernel leg: one plain photon job (the bench's photons and
    medium) through hrm_plain_run on one stream, best of three, its tallies compared with the
    timed run's; the leg reports its own description for the line. Device faked, as above."""
    import types

    import harmonize_b200 as hrm
    from harmonize_b200 import jobs

    seen = []

    class FakeJobsLib:
        def hrm_plain_run(self, arr_ref, njobs, nstreams, done_ptr, total_ref):
            j = arr_ref._obj[0]
            seen.append((j.kind, j.first, j.count, j.n, j.seed, njobs, nstreams))
            total_ref._obj.value = 10.0 - len(seen)  # 9, 8, 7 ms: best of three is 7
            return 0

    class FakeTensor:
        def data_ptr(self):
            return 0x2000

        def cuda(self):
            return self

        def pin_memory(self):
            return self

    fake_torch = types.SimpleNamespace(from_numpy=lambda a: FakeTensor(), zeros=lambda *a, **k: FakeTensor(),
                                       int64="int64", equal=lambda a, b: False,
                                       cuda=types.SimpleNamespace(synchronize=lambda: None))
    monkeypatch.setattr(jobs, "_bind", lambda: FakeJobsLib())
    monkeypatch.setattr(bench, "flush_l2", lambda buf: None)
    args = types.SimpleNamespace(program="async", variant=2, workload="photon", grid=8, photons=100)
    wl = bench.run_photon(args, hrm, 0, 1, None, fake_torch)
    ms, info = wl["plain_arm"](None)
    assert ms == 7.0
    assert info["same_tallies"] is False and "one thread per source photon" in info["what"]
    assert seen == [(jobs.JOB_PHOTON, 0, 100, 8, 0x5EED0123456789, 1, 1)] * 3


def test_plain_record_of_the_line():
    rec = bench.plain_record(385.6843, 16119494612, {"same_tallies": True, "what": "w"})
    assert rec == {"ms": 385.684, "equivalent_calls_per_s": round(16119494612 / 0.3856843, 1),
                   "same_tallies": True, "what": "w"}
