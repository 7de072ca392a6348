"""bench.py's host-side pieces on the CPU: the clock-sample parser, the per-kernel DRAM
traffic read from the committed ncu summaries, the peak-bandwidth lookup, and the
reference arm's JSON line (the oracle timed on the host, no GPU)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_sampler_reports_the_median_under_load_and_the_reasons(tmp_path):
    path = tmp_path / "clocks.csv"
    rows = [
        "0, 345, 1965, 150.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 810.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    path.write_text("\n".join(rows) + "\n")
    s = bench.ClockSampler(0)
    s.proc = _Done()
    s.path = str(path)
    out = s.stop()
    assert out["sm_mhz"] == 1965.0  # the idle 345 MHz sample is not under load
    assert out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    assert out["samples"] == 4
    assert not path.exists()


def test_clock_sampler_without_nvidia_smi():
    s = bench.ClockSampler(0)
    assert s.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_profiled_traffic_covers_the_tile_kernels():
    traffic = bench.profiled_traffic()
    for k in ("tile_fwd", "tile_x", "tile_inv"):  # the names the roofline entry reads
        assert k in traffic, k
    assert all(v > 0 for v in traffic.values())


def test_peaks_fall_back_without_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, 1590.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6546.9, "bf16_tflops": 1500.0}))
    assert bench.peaks() == (6546.9, 1500.0, "measured")


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is True
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == bench.WORKLOAD
