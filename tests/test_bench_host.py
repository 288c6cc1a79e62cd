"""Host-side logic of bench.py (no GPU): the committed DRAM-traffic data covers every kernel
of the step and is used only for the workload it was captured on, the field-error summary,
and the clock summary reports throttle reasons from any sample."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_traffic_data_covers_every_kernel():
    import json
    d = json.load(open(bench.TRAFFIC_DATA))
    kb = bench.kernel_bytes(*bench.GRID, bench.NPART)
    assert set(d["kernels"]) == set(kb)
    assert tuple(d["workload"]["grid"]) == bench.GRID and d["workload"]["particles"] == bench.NPART
    # x-pair gather: coordinates in, E out, the x-pair grid once
    n = bench.GRID[0] * bench.GRID[1] * bench.GRID[2]
    assert kb["interp_f32"] == 48 * bench.NPART + 32 * n


def test_profiled_traffic_of_the_dominant_kernel():
    t = bench.profiled_traffic("interp_f32", bench.GRID, bench.NPART, "random")
    a = bench.kernel_bytes(*bench.GRID, bench.NPART)["interp_f32"]
    # the measured DRAM traffic is the algorithmic bytes to within 3% (no re-reads)
    assert t is not None and abs(t - a) <= 0.03 * a
    assert bench.profiled_traffic("no_such_kernel", bench.GRID, bench.NPART, "random") is None
    # a capture of another workload is not used
    assert bench.profiled_traffic("interp_f32", (64, 64, 64), bench.NPART, "random") is None
    assert bench.profiled_traffic("interp_f32", bench.GRID, bench.NPART, "sorted") is None


def test_field_errors():
    import numpy as np
    ref = np.random.default_rng(0).standard_normal((100, 3))
    e = bench.field_errors(ref * (1 + 1e-7), ref)
    assert e["max"] <= 1.1e-7 and e["rms"] <= 1.1e-7 and len(e["max_per_component"]) == 3


def test_clock_summary_reasons():
    c = bench.ClockSampler(0)
    c.samples = [(1965.0, 1965.0, set()), (1950.0, 1965.0, {"sw_power_cap"}), (1965.0, 1965.0, set())]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    c.samples = []
    assert c.summary()["samples"] == 0


@pytest.mark.parametrize("np_", [1, 1000, 10 ** 7])
def test_kernel_bytes_scale_with_particles(np_):
    kb0 = bench.kernel_bytes(64, 64, 128, 0)
    kb1 = bench.kernel_bytes(64, 64, 128, np_)
    assert kb1["deposit_f32"] - kb0["deposit_f32"] == 24 * np_
    assert kb1["interp_f32"] - kb0["interp_f32"] == 48 * np_
    assert kb1["fft_z_conv"] == kb0["fft_z_conv"]
