"""The host-side arithmetic of bench.py's JSON line (CPU): the FP-pipe
fraction, the clock summary (median SM clock and the throttle reasons seen)
and the contract keys of the reference arm's line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_fp_pipe_fractions():
    import bench
    peak = {"f64": 34.0, "f32": 72.0, "f32x2": 74.0}
    cell_steps = 256 ** 3 * 20
    out = bench.fp_pipe("learned", 172.0, {"f32": 143.4, "f64": 1036.0}, cell_steps, peak)
    assert out["flops_per_cell_step"] == bench.FLOPS_PER_CELL_STEP
    for p_, ms in (("learned", 172.0), ("f32", 143.4), ("f64", 1036.0)):
        a = bench.FLOPS_PER_CELL_STEP * cell_steps / (ms / 1e3) / 1e12
        pk = 34.0 if p_ == "f64" else 74.0
        assert out[p_]["achieved"] == pytest.approx(a)
        assert out[p_]["peak"] == pk
        assert out[p_]["frac"] == pytest.approx(a / pk)


def test_clock_summary_reports_median_and_reasons():
    import bench
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1935, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "garbage line", "0, [N/A], 1965, 1, 0, a, b, c, d"]
    s = c.summary()
    assert s == {"sm_mhz": 1935.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    c.lines.append("0, 1200, 1965, 500, 0x40, Not Active, Active, Not Active, Not Active")
    assert bench.ClockSampler.summary(c)["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


@pytest.mark.timeout(600)
def test_reference_arm_line_keeps_the_contract():
    """`bench.py --impl reference` (the oracle on the host cores) prints one
    JSON line with the metric of the GPU arm and a cpu_baseline / e2e block."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--n", "64"], capture_output=True, text=True, timeout=580)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
