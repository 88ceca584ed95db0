"""The measurement plumbing of bench.py that needs no GPU: the algorithmic
bytes of each kernel, the committed DRAM traffic it reports beside them, and
the JSON line of the reference arm (the reference's own CPU code)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, str(ROOT))
    import bench as b
    return b


def test_algorithmic_bytes_per_kernel(bench):
    Np, Nc = 512 ** 3, 512 ** 3
    assert bench.algorithmic_bytes("gather_kick_drift_deposit", Np, Nc, False) == 60 * Np + 4 * Nc
    assert bench.algorithmic_bytes("gather_kick", Np, Nc, False) == 48 * Np + 4 * Nc
    assert bench.algorithmic_bytes("deposit", Np, Nc, False) == 12 * Np + 4 * Nc
    assert bench.algorithmic_bytes("gather_kick_drift_deposit", Np, Nc, True) == 2 * (60 * Np + 4 * Nc)
    assert bench.algorithmic_bytes("fd_grad", Np, Nc, False) is None


def test_dram_traffic_of_the_dominant_kernel_is_committed(bench):
    w = bench.workload_name(9, 1)
    t = bench.dram_traffic("gather_kick_drift_deposit", w)
    assert t is not None and t > bench.algorithmic_bytes("gather_kick_drift_deposit", 512 ** 3, 512 ** 3, False)
    assert bench.dram_traffic("no_such_kernel", w) is None


def test_reference_arm_prints_one_json_line():
    # a 64^3 box keeps the reference's two timed steps short here (the
    # default is the full 512^3 box)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--mbits", "6"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "particle-steps/s" and d["higher_is_better"] is True
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    if d["cpu_baseline"]["kind"] == "reference":  # one step at all threads and one at a single thread
        assert "1" in d["cpu_baseline"]["seconds_per_step_by_threads"]


class _FakeNVML:
    """Read-only NVML stand-in: a fixed SM clock and the power-cap reason."""
    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonHwSlowdown = 1
    nvmlClocksEventReasonHwThermalSlowdown = 2
    nvmlClocksEventReasonSwThermalSlowdown = 4
    nvmlClocksEventReasonSwPowerCap = 8

    def nvmlInit(self):
        pass

    def nvmlDeviceGetHandleByIndex(self, i):
        return i

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        return 1900

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return 8


@pytest.mark.parametrize("seconds", [0.0, 0.1])
def test_clock_sampler_reports_short_and_long_regions(bench, monkeypatch, seconds):
    """Clocks and throttle reasons are sampled during the timed region; a
    region shorter than the sampling thread's start-up still gets a reading."""
    import time
    monkeypatch.setitem(sys.modules, "pynvml", _FakeNVML())
    with bench.Clocks(0) as clk:
        time.sleep(seconds)
    s = clk.summary()
    assert s["samples"] >= 1 and s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["source"] == "nvml 10 ms"


class _SilentNVML(_FakeNVML):
    def nvmlDeviceGetClockInfo(self, h, kind):
        raise RuntimeError("no reading")


def test_clock_sampler_survives_an_nvml_without_readings(bench, monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", _SilentNVML())
    with bench.Clocks(0) as clk:
        pass
    s = clk.summary()
    assert s["samples"] == 0 or s["source"].startswith("nvidia-smi")


def test_nvidia_smi_lines_are_parsed(bench):
    clk = bench.Clocks(0)
    clk._parse_smi("0, 1900, 1965, 712.40, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
                   "garbage line\n")
    assert clk.samples == [(1900.0, 1965.0, {"sw_power_cap"})]


def test_clock_records_that_reject_a_timing(bench):
    ok = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    assert not bench.clocks_disturbed(ok)
    assert not bench.clocks_disturbed({"sm_mhz": 1300.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"]})
    assert bench.clocks_disturbed({"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["hw_slowdown"]})
    assert bench.clocks_disturbed({"sm_mhz": 1200.0, "sm_max_mhz": 1965.0, "reasons": []})
    assert not bench.clocks_disturbed({"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0})
