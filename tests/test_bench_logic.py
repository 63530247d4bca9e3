"""Host-side logic of bench.py on the CPU: the clock record's summary (with
a stand-in for the NVML sampling thread), the figures the roofline takes
from committed files, the workload name both arms print and the ensemble's
column tiling."""
import threading

import numpy as np

import bench
from gitm_b200 import synthetic


class _Joined:
    def join(self, timeout=None):
        return None


def _sampler_with(samples, smax=1965.0):
    s = bench.ClockSampler(0)
    s.thread = _Joined()
    s.stop_flag = threading.Event()
    s.smax = smax
    s.samples = list(samples)
    return s


def test_clock_summary_reads_reasons_power_and_temperature():
    # (SM MHz, clock-event reason bits, W, deg C)
    samples = [(1965.0, 0, 500.0, 40), (1965.0, 0x4, 990.0, 52), (1800.0, 0x4 | 0x20, 700.0, 61)]
    out = _sampler_with(samples).stop()
    assert out["sm_mhz"] == 1965.0 and out["sm_min_mhz"] == 1800.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    assert out["samples"] == 3
    assert out["power_w_max"] == 990.0 and out["temp_c_max"] == 61


def test_clock_summary_without_samples():
    out = _sampler_with([]).stop()
    assert out["sm_mhz"] is None and out["samples"] == 0 and out["reasons"] == []
    assert out["power_w_max"] is None and out["temp_c_max"] is None


def test_roofline_inputs_come_from_the_committed_files():
    # the oracle's operation count and the ncu summary's DRAM bytes
    assert bench.opcount(50) == 616627.0
    assert bench.opcount(50, "ausm") == 1391515.0
    assert bench.profile_traffic() == 25284.0
    # compulsory bytes per column and launch: the state read once, written once
    assert 20e3 < bench.algorithmic_bytes_per_column_step(50) < 30e3


def test_workload_name_is_one_string_for_both_arms():
    assert bench.workload_name(1.0, 64800, 50, "rusanov") == "globe 1 deg, 64800 columns x 50 alts, Rusanov RK4, dt 2 s"
    assert bench.workload_name(2.5, 10368, 50, "ausm").endswith("AUSM RK4, dt 2 s")


def test_tile_member_repeats_columns_and_keeps_the_grid():
    m = synthetic.make_member(7, 20, seed=3)
    t = bench.tile_member(m, 18)
    assert t.n_cols == 18
    idx = np.arange(18) % 7
    np.testing.assert_array_equal(t.ndensity_s, m.ndensity_s[..., idx])
    np.testing.assert_array_equal(t.temperature, m.temperature[..., idx])
    np.testing.assert_array_equal(t.altitude, m.altitude)


def test_reference_arm_prints_the_contract_line():
    """bench.py --impl reference on a small globe: one JSON line with the
    reference arm's keys, its e2e moving no bytes between host and device."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--deg", "10", "--cpu-seconds", "1"],
                       capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "column-steps/s" and line["value"] > 0
    assert line["config"]["workload"] == bench.workload_name(10.0, 648, 50, "rusanov")
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "column-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 of the reference arm works and prints."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--deg", "10", "--cpu-seconds", "1"],
                       capture_output=True, text=True, timeout=300, cwd=root, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
