"""Host-side pieces of bench.py that need no GPU: the clock-record summary
(against a fake NVML sample stream), the roofline traffic read from the
committed ncu summaries, and the flop constants the metric uses."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from spearhed_b200 import flops  # noqa: E402


def test_clock_summary_reads_reason_bits():
    s = bench.ClockSampler(0)
    s.nvml = object()  # NVML path taken; samples supplied by hand
    s.max_mhz = 1965.0
    s.samples = [(1965.0, 0x0), (1950.0, 0x4), (1965.0, 0x1), (1800.0, 0x4 | 0x8)]
    d = s.summary()
    assert d["samples"] == 4
    assert d["sm_max_mhz"] == 1965.0
    assert d["sm_mhz"] == 1957.5
    # 0x1 (GPU idle) is not a reason the record keeps; 0x4 and 0x8 are
    assert d["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_clock_summary_without_samples():
    s = bench.ClockSampler(0)
    s.nvml = object()
    d = s.summary()
    assert d["samples"] == 0 and d["sm_mhz"] is None and d["reasons"] == []


def test_traffic_lines_of_committed_profiles():
    dens = bench.traffic_from_profiles("density_fp32_orszag_tang.txt")
    force = bench.traffic_from_profiles("force_mhd_fp32_orszag_tang.txt")
    assert dens is not None and 1e8 < dens < 5e9
    assert force is not None and 1e8 < force < 5e9
    assert bench.traffic_from_profiles("no_such_profile.txt") is None


def test_flop_constants():
    assert flops.PASSES_PER_STEP["mhd"] == 3
    assert flops.FORCE_FLOPS["mhd"] > flops.FORCE_FLOPS["hydro"] > flops.DENSITY_FLOPS["cubic"]
    assert flops.CULL_FLOPS_PER_CANDIDATE == 9


def test_hbm_view_of_a_launch():
    v = bench.hbm_view({"traffic": 6.5e8, "ms_per_launch": 1.0}, 6500.0)
    assert v["unit"] == "GB/s" and abs(v["achieved"] - 650.0) < 1e-9 and abs(v["frac"] - 0.1) < 1e-12
    assert bench.hbm_view({"traffic": None, "ms_per_launch": 1.0}, 6500.0) is None
    assert bench.hbm_view({"traffic": 6.5e8, "ms_per_launch": 1.0}, None) is None


def test_traffic_only_for_the_profiled_configuration():
    import argparse
    a = argparse.Namespace(workload="orszag_tang", nx=512, nz=4)
    assert bench.profiled_config(a)
    a.nx = 256
    assert not bench.profiled_config(a)
    assert not bench.profiled_config(argparse.Namespace(workload="mhd_rotor", nx=512, nz=4))
