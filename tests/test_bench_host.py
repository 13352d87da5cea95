"""Host-side pieces of bench.py that run without a GPU: argument defaults,
the workload cells, the clock-record parsing, the profiled-traffic scaling
and the JSON config block."""
import importlib
import sys

import pytest


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ".")
    return importlib.import_module("bench")


def test_defaults_and_helpers_present(bench, monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.impl, a.workload, a.batch, a.queue) == (1, "ours", "c3", 64, 4096)
    assert a.warmup >= 3
    for name in ("ClockSampler", "measured_peaks", "dgemm_peak_tflops", "cpu_rounds", "run_reference",
                 "run_ours", "profiled_traffic", "workload_config", "metric_name", "make_cells", "Waves"):
        assert hasattr(bench, name), name


def test_c3_waves_walk_the_cost_sharded_queue(bench, monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--queue", "40", "--batch", "8", "--npix", "16"])
    a = bench.parse()
    w = bench.Waves(a, 0, 1)
    assert len(w.queue) == 40
    first, second = w.next(), w.next()
    assert len(first) == 8 and first[0] is w.queue[0] and second[0] is w.queue[8]
    sizes = {d["nx"] for d in w.queue}
    assert sizes <= {7, 9, 11, 13, 15} and len(sizes) >= 3  # uneven truncations
    # two ranks split the queue by cost, disjointly
    q0, q1 = bench.Waves(a, 0, 2).queue, bench.Waves(a, 1, 2).queue
    assert len(q0) + len(q1) == 40
    key = lambda d: (d["nx"], d["lam"], d["r0"])
    assert not ({key(d) for d in q0} & {key(d) for d in q1})
    cfg = bench.workload_config(a, a.batch)
    assert "4096" not in cfg["workload"] and "40 cells" in cfg["workload"]


def test_cells_are_seeded_and_rank_disjoint(bench):
    c0 = bench.make_cells("c2", 3, 0, 16)
    c1 = bench.make_cells("c2", 3, 1, 16)
    assert len(c0) == 3 and all(d["nx"] == 11 and d["ny"] == 11 for d in c0)
    assert bench.make_cells("c2", 3, 0, 16)[1]["r0"] == c0[1]["r0"]  # deterministic
    assert [d["r0"] for d in c0] != [d["r0"] for d in c1]


def test_clock_record_parsing(bench):
    cs = bench.ClockSampler(0)
    cs.proc = type("P", (), {"terminate": lambda s: None, "wait": lambda s, timeout=None: 0})()
    cs.lines = ["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
                "0, 1900, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
                "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    clk = cs.stop()
    assert clk["sm_mhz"] == 1965.0 and clk["sm_max_mhz"] == 1965.0
    assert clk["reasons"] == ["sw_power_cap"] and clk["samples"] == 3


def test_profiled_traffic_scales_by_matrices(bench):
    per_launch_one = bench.profiled_traffic("schur_qr", 40 * 242 ** 3)
    assert per_launch_one is not None and per_launch_one > 0
    assert bench.profiled_traffic("schur_qr", 2 * 40 * 242 ** 3) == pytest.approx(2 * per_launch_one)
    assert bench.profiled_traffic("no_such_family", 1.0) is None


def test_roofline_uses_union_time_and_launched_families(bench):
    """The dominant family is chosen among launched kernels (host_alloc is
    host time) by its busy time, the union of its launch intervals, which
    is also the denominator of the achieved rate."""
    stats = {
        "host_alloc": {"ms": 9000.0, "busy_ms": 9000.0, "launches": 0, "flops": 0.0, "bytes": 0.0},
        "schur_qr": {"ms": 3000.0, "busy_ms": 1000.0, "launches": 6, "flops": 4.0e12, "bytes": 0.0},
        "zgemm": {"ms": 900.0, "busy_ms": 800.0, "launches": 100, "flops": 2.4e13, "bytes": 0.0},
        "assembly": {"ms": 100.0, "busy_ms": 90.0, "launches": 50, "flops": 0.0, "bytes": 1e9},
    }
    r = bench.roofline_of(stats, 35.0)
    assert r["kernel"] == "schur_qr" and r["bound"] == "tensor"
    assert r["achieved"] == pytest.approx(4.0)           # 4e12 flops over 1.0 s busy
    assert r["frac"] == pytest.approx(4.0 / 35.0)
    assert r["avg_launch_ms"] == pytest.approx(500.0)    # summed durations per launch
    assert r["busy_ms"] == 1000.0
