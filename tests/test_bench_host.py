"""Host-side logic of bench.py (no GPU): the algorithmic bytes per kernel agree with the
committed DRAM-traffic table, the table parser returns the dominant kernel's traffic, and
the clock summary reports throttle reasons from any sample."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_kernel_bytes_match_traffic_table():
    kb = bench.kernel_bytes(*bench.GRID, bench.NPART)
    rows = {}
    for line in open(bench.TRAFFIC_TABLE):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 6 and cells[0] in kb:
            rows[cells[0]] = int(cells[5])
    assert set(rows) == set(kb)
    for name, b in kb.items():
        assert rows[name] == b, name
    # x-pair gather: coordinates in, E out, the x-pair grid once
    n = bench.GRID[0] * bench.GRID[1] * bench.GRID[2]
    assert kb["interp_f32"] == 48 * bench.NPART + 32 * n


def test_profiled_traffic_of_the_dominant_kernel():
    t = bench.profiled_traffic("interp_f32")
    a = bench.kernel_bytes(*bench.GRID, bench.NPART)["interp_f32"]
    # the measured DRAM traffic is the algorithmic bytes to within 3% (no re-reads)
    assert t is not None and abs(t - a) <= 0.03 * a
    assert bench.profiled_traffic("no_such_kernel") is None


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
