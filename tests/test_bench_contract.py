"""bench.py's reference arm runs on the CPU (the reference's own flow step under Numba's CUDA
simulator when it is installed into baseline/_ref, else the oracle on bounded stripes of the
workload) and prints one JSON line with the keys the driver reads; checked here without a GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("chiral magnet 4096x4096")
    cb = d["cpu_baseline"]
    installed = os.path.isdir(os.path.join(ROOT, "baseline", "_ref", "soliton_solver"))
    assert cb["kind"] == ("reference" if installed else "port")
    assert cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_clock_summary_keeps_only_the_timed_region():
    """bench.Clocks.summary(): the median SM clock, the max power and the union of the
    clock-event reasons of the samples between the first and last mark()."""
    sys.path.insert(0, ROOT)
    import bench

    c = bench.Clocks(0)
    c.thread = object()  # as if the NVML poller had run
    c.marks = [10.0, 10.02]
    c.samples = [(9.99, 1000.0, 1965.0, 500.0, {"sw_power_cap"}),   # before the timed region
                 (10.005, 1965.0, 1965.0, 270.0, set()),
                 (10.010, 1950.0, 1965.0, 275.0, {"sw_power_cap"}),
                 (10.015, 1965.0, 1965.0, 272.0, set()),
                 (10.03, 900.0, 1965.0, 100.0, {"hw_slowdown"})]    # after it
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["power_w_max"] == 275.0 and s["reasons"] == ["sw_power_cap"]
    empty = bench.Clocks(0)
    assert empty.summary()["sm_mhz"] is None
